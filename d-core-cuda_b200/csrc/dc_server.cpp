// Serving loop: streams of edge-update requests against many device-resident
// graphs, admitted under an HBM budget, with continuous batching.
//
//   - every graph has a FIFO of pending requests; a worker that picks a graph
//     takes all of its pending requests at once and applies them as one
//     maintenance batch (their concatenation, in arrival order, has the same
//     sequential meaning as applying them one after another, because a batch
//     reduces to its net effect per edge in order)
//   - workers run different graphs at the same time, each graph on its own
//     CUDA stream with stream-ordered allocations, so their kernels overlap
//     on the device
//   - a graph is resident (device handle + decomposition) only while the
//     budget holds it; each resident graph is charged an upper bound of its
//     device footprint (maintenance transients included), and to admit
//     another the least recently used idle graph is evicted (its current
//     edges are kept on the host, and it is rebuilt and decomposed again when
//     a request needs it)
//   - a request's latency runs from submission to the end of the batch that
//     contained it
//
// No counterpart in the reference (its driver handles one graph,
// main.cu:1784-2218).
#include <algorithm>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "dc_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id;
    uint32_t graph;
    std::vector<uint32_t> pairs;
    std::vector<uint8_t> del;
    Clock::time_point t_submit;
};

struct Completion {
    uint64_t id;
    uint32_t graph;
    double latency_ms;
    uint32_t batch_requests;  // requests coalesced into the batch
    uint64_t batch_updates;
    int32_t status;
};

struct GraphSlot {
    uint32_t V = 0;
    std::vector<uint32_t> src, dst;  // current edges while not resident
    dc_graph* h = nullptr;
    std::deque<Request> pending;
    bool busy = false;
    uint64_t bytes = 0;     // charged to the budget while resident
    uint64_t measured = 0;  // dc_graph_device_bytes after the last batch
    uint64_t E = 0;         // live edges
    Clock::time_point last_used;
    uint64_t batches = 0;
};

}  // namespace

struct dc_server {
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<GraphSlot> graphs;  // deque: slots keep their address while graphs are added
    std::vector<Completion> done;
    std::vector<std::thread> workers;
    uint64_t budget = 0, used = 0, peak = 0;
    uint64_t next_id = 1, submitted = 0, completed = 0;
    uint64_t admissions = 0, evictions = 0, batches = 0;
    int method = DC_MAINT_AUTO;
    int device = 0;
    int row_repair = 1;
    uint64_t sms = 148;
    bool stop = false;
    dc_graph_opts opts;
};

namespace {

// Upper bound on the device bytes a handle of V vertices and E edges can
// hold, transients of maintenance included: slack adjacency under the
// rebuild rule (len + len/8 + 2 per list) with its kmax-sort working copies,
// offsets and lengths, kmax/row 0, the skyline twice (old and merged during a
// batch), per-vertex scratch, the vertex ring and ticket ring (powers of two),
// the corner log (at most E + V corners) and rebuild staging.
uint64_t footprint_bound(uint64_t V, uint64_t E, uint64_t sms) {
    const uint64_t cap = E + E / 8 + 2 * V + 64;
    uint64_t b = 2 * 4 * cap * 2;
    b += 4 * 4 * (V + 1);
    b += 4 * 3 * (V + 1) + 3 * (8 * (E + 2 * V) + 4 * (V + 1));  // skyline and its two spares
    b += 4 * 20 * (V + 2) + 8 * (V + 2) + 8 * (sms * 64 + 64);
    b += 8 * (V + sms * 64 * 32 + 64);
    b += 12 * (E + V + 1);
    b += 16 * (2 * V + 2 * cap / 32 + sms * 64 + 4096);
    b += 8 * E + 2 * 4 * cap;
    b += 4 * 7 * (V + 1) + 2 * 4 * ((E + 8) + (E + 8) / 8 + 7);  // the row kernel's relabeled graph
    return b + (1ull << 20);
}

// Bytes charged to the budget for a resident graph: the bound with room for
// E/8 (at least 4096) more edges, so batches rarely need a new reservation.
uint64_t reserve_bytes(uint64_t V, uint64_t E, uint64_t sms) {
    return footprint_bound(V, E + std::max<uint64_t>(E / 8, 4096), sms);
}

void charge(dc_server* s, GraphSlot& g, uint64_t bytes) {
    s->used = s->used - g.bytes + bytes;
    g.bytes = bytes;
    s->peak = std::max(s->peak, s->used);
}

// Evicts idle resident graphs (least recently used first) until `need` more
// bytes fit.  Called with the lock held; the victim is marked busy and its
// edges are downloaded with the lock released, so other workers keep going.
// False when nothing is left to evict.
bool make_room(dc_server* s, uint64_t need, const GraphSlot* keep, std::unique_lock<std::mutex>& lk) {
    while (s->used + need > s->budget) {
        GraphSlot* victim = nullptr;
        for (auto& g : s->graphs) {
            if (&g == keep || !g.h || g.busy) continue;
            if (!victim || g.last_used < victim->last_used) victim = &g;
        }
        if (!victim) return false;
        GraphSlot& g = *victim;
        g.busy = true;
        dc_graph* h = g.h;
        lk.unlock();
        uint64_t E = 0;
        dc_graph_info(h, nullptr, &E);
        std::vector<uint32_t> src(E), dst(E);
        dc_graph_get_edges(h, src.data(), dst.data(), E, &E);
        dc_graph_free(h);
        lk.lock();
        g.src.swap(src);
        g.dst.swap(dst);
        g.h = nullptr;
        g.busy = false;
        charge(s, g, 0);
        s->evictions++;
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
    return true;
}

// Makes g resident: reserves its bytes (evicting idle graphs; a graph larger
// than the whole budget waits until nothing else is resident), then builds
// and decomposes it with the lock released.  Lock held on entry and exit;
// g.busy must be set by the caller.  A waiting admission holds no charge, so
// the graphs it waits for always finish.
int admit(dc_server* s, GraphSlot& g, std::unique_lock<std::mutex>& lk) {
    if (g.h) return DC_OK;
    const uint64_t need = reserve_bytes(g.V, g.src.size(), s->sms);
    while (!make_room(s, need, &g, lk) && s->used != 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(2));
    charge(s, g, need);
    s->admissions++;
    std::vector<uint32_t> src, dst;
    src.swap(g.src);
    dst.swap(g.dst);
    lk.unlock();
    dc_graph* h = nullptr;
    int rc = dc_graph_create(g.V, src.size(), src.data(), dst.data(), &s->opts, &h);
    if (rc == DC_OK) rc = dc_set_row_repair(h, s->row_repair);
    if (rc == DC_OK) rc = dc_decompose(h, DC_METHOD_INCREMENTAL, nullptr, nullptr);
    uint64_t bytes = 0;
    if (rc == DC_OK) dc_graph_device_bytes(h, &bytes);
    lk.lock();
    if (rc != DC_OK) {
        if (h) dc_graph_free(h);
        g.src.swap(src);
        g.dst.swap(dst);
        charge(s, g, 0);
        return rc;
    }
    g.h = h;
    g.measured = bytes;
    g.E = src.size();
    return DC_OK;
}

// Grows a resident graph's charge before a batch of n_ins insertions when
// its bound no longer fits the charge: idle graphs are evicted for it; when
// none is left the batch runs over budget (it cannot wait for busy graphs
// without risking that they wait for it).
void grow_charge(dc_server* s, GraphSlot& g, uint64_t n_ins, std::unique_lock<std::mutex>& lk) {
    const uint64_t bound = footprint_bound(g.V, g.E + n_ins, s->sms);
    if (bound <= g.bytes) return;
    const uint64_t need = reserve_bytes(g.V, g.E + n_ins, s->sms);
    make_room(s, need - g.bytes, &g, lk);
    charge(s, g, need);
}

void worker(dc_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // the graph whose oldest pending request is oldest
        GraphSlot* pick = nullptr;
        for (;;) {
            if (s->stop) return;
            for (auto& g : s->graphs) {
                if (g.busy || g.pending.empty()) continue;
                if (!pick || g.pending.front().t_submit < pick->pending.front().t_submit) pick = &g;
            }
            if (pick) break;
            s->cv_work.wait(lk);
        }
        GraphSlot& g = *pick;
        g.busy = true;
        std::vector<Request> batch(std::make_move_iterator(g.pending.begin()),
                                   std::make_move_iterator(g.pending.end()));
        g.pending.clear();
        int rc = admit(s, g, lk);
        if (rc != DC_OK)
            fprintf(stderr, "dc_server: admitting graph %u failed (%d): %s\n", batch.front().graph, rc,
                    dc_last_error());
        // one maintenance batch for all coalesced requests
        std::vector<uint32_t> pairs;
        std::vector<uint8_t> del;
        uint64_t updates = 0, n_ins = 0;
        for (auto& r : batch) {
            pairs.insert(pairs.end(), r.pairs.begin(), r.pairs.end());
            del.insert(del.end(), r.del.begin(), r.del.end());
            updates += r.del.size();
        }
        for (uint8_t x : del) n_ins += x == 0;
        if (rc == DC_OK) {
            grow_charge(s, g, n_ins, lk);
            lk.unlock();
            rc = dc_maintain(g.h, pairs.data(), del.data(), updates, s->method, nullptr);
            if (rc != DC_OK)  // the worker's error message is thread-local: report it here
                fprintf(stderr, "dc_server: batch of %llu updates on graph %u failed (%d): %s\n",
                        (unsigned long long)updates, batch.front().graph, rc, dc_last_error());
            uint64_t bytes = 0, E = 0;
            dc_graph_device_bytes(g.h, &bytes);
            dc_graph_info(g.h, nullptr, &E);
            lk.lock();
            g.measured = bytes;
            g.E = E;
        }
        Clock::time_point now = Clock::now();
        for (auto& r : batch) {
            Completion c;
            c.id = r.id;
            c.graph = r.graph;
            c.latency_ms = std::chrono::duration<double, std::milli>(now - r.t_submit).count();
            c.batch_requests = (uint32_t)batch.size();
            c.batch_updates = updates;
            c.status = rc;
            s->done.push_back(c);
        }
        s->completed += batch.size();
        s->batches++;
        g.batches++;
        g.busy = false;
        g.last_used = now;
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

using dc::set_error;

extern "C" int dc_server_create(uint64_t hbm_budget_bytes, int max_concurrent, int method, int device,
                                dc_server** out) {
    if (!out || max_concurrent < 1 || max_concurrent > 64 || hbm_budget_bytes == 0 || method < DC_MAINT_AUTO ||
        method > DC_MAINT_REPEEL)
        return set_error(DC_ERR_INVALID, "dc_server_create: bad argument");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(DC_ERR_NO_DEVICE, "dc_server_create: no CUDA device");
    }
    if (device < 0 || device >= n) return set_error(DC_ERR_INVALID, "dc_server_create: device %d out of range", device);
    dc_server* s = new dc_server();
    s->budget = hbm_budget_bytes;
    s->method = method;
    s->device = device;
    dc_graph_opts_default(&s->opts);
    s->opts.device = device;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
        s->sms = (uint64_t)sms;
    for (int i = 0; i < max_concurrent; ++i) s->workers.emplace_back(worker, s);
    *out = s;
    return DC_OK;
}

extern "C" int dc_server_add_graph(dc_server* s, uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                                   uint32_t* graph_id) {
    if (!s || !graph_id || (E && (!src || !dst))) return set_error(DC_ERR_INVALID, "dc_server_add_graph: bad argument");
    for (uint64_t e = 0; e < E; ++e)
        if (src[e] >= V || dst[e] >= V)
            return set_error(DC_ERR_INVALID, "dc_server_add_graph: edge %llu has an id >= V", (unsigned long long)e);
    std::lock_guard<std::mutex> lk(s->mu);
    s->graphs.emplace_back();
    GraphSlot& g = s->graphs.back();
    g.V = V;
    g.src.assign(src, src + E);
    g.dst.assign(dst, dst + E);
    g.last_used = Clock::now();
    *graph_id = (uint32_t)(s->graphs.size() - 1);
    return DC_OK;
}

extern "C" int dc_server_submit(dc_server* s, uint32_t graph_id, const uint32_t* pairs, const uint8_t* is_delete,
                                uint64_t b, uint64_t* request_id) {
    if (!s || (b && !pairs)) return set_error(DC_ERR_INVALID, "dc_server_submit: bad argument");
    Request r;
    r.graph = graph_id;
    r.pairs.assign(pairs, pairs + 2 * b);
    r.del.assign(b, 0);
    if (is_delete)
        for (uint64_t i = 0; i < b; ++i) r.del[i] = is_delete[i] ? 1 : 0;
    std::lock_guard<std::mutex> lk(s->mu);
    if (graph_id >= s->graphs.size()) return set_error(DC_ERR_INVALID, "dc_server_submit: unknown graph %u", graph_id);
    const uint32_t V = s->graphs[graph_id].V;
    for (uint64_t i = 0; i < 2 * b; ++i)
        if (pairs[i] >= V) return set_error(DC_ERR_INVALID, "dc_server_submit: vertex id %u >= V", pairs[i]);
    r.id = s->next_id++;
    r.t_submit = Clock::now();
    if (request_id) *request_id = r.id;
    s->graphs[graph_id].pending.push_back(std::move(r));
    s->submitted++;
    s->cv_work.notify_one();
    return DC_OK;
}

extern "C" int dc_server_drain(dc_server* s, uint64_t timeout_ms) {
    if (!s) return set_error(DC_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                  [&] { return s->completed == s->submitted; });
    return ok ? DC_OK
              : set_error(DC_ERR_TIMEOUT, "dc_server_drain: %llu requests still pending after %llu ms",
                          (unsigned long long)(s->submitted - s->completed), (unsigned long long)timeout_ms);
}

extern "C" int dc_server_completions(dc_server* s, uint64_t* ids, uint32_t* graphs, double* latency_ms,
                                     uint32_t* batch_requests, uint64_t* batch_updates, int32_t* status,
                                     uint64_t capacity, uint64_t* n) {
    if (!s || !n) return set_error(DC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (!ids) {
        *n = s->done.size();
        return DC_OK;
    }
    *n = std::min<uint64_t>(capacity, s->done.size());
    for (uint64_t i = 0; i < *n; ++i) {
        const Completion& c = s->done[i];
        ids[i] = c.id;
        if (graphs) graphs[i] = c.graph;
        if (latency_ms) latency_ms[i] = c.latency_ms;
        if (batch_requests) batch_requests[i] = c.batch_requests;
        if (batch_updates) batch_updates[i] = c.batch_updates;
        if (status) status[i] = c.status;
    }
    s->done.erase(s->done.begin(), s->done.begin() + *n);
    return DC_OK;
}

extern "C" int dc_server_info_get(dc_server* s, dc_server_info* info) {
    if (!s || !info) return set_error(DC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(info, 0, sizeof(*info));
    info->budget_bytes = s->budget;
    info->used_bytes = s->used;
    info->peak_bytes = s->peak;
    info->admissions = s->admissions;
    info->evictions = s->evictions;
    info->batches = s->batches;
    info->submitted = s->submitted;
    info->completed = s->completed;
    info->graphs = (uint32_t)s->graphs.size();
    for (auto& g : s->graphs) {
        info->resident += g.h != nullptr;
        if (g.h) info->measured_bytes += g.measured;
    }
    return DC_OK;
}

extern "C" int dc_server_graph_result(dc_server* s, uint32_t graph_id, int32_t* kmaxes, int32_t* rows,
                                      uint64_t rows_capacity, int32_t* kmax) {
    if (!s || !kmax) return set_error(DC_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (graph_id >= s->graphs.size()) return set_error(DC_ERR_INVALID, "unknown graph %u", graph_id);
    GraphSlot& g = s->graphs[graph_id];
    s->cv_done.wait(lk, [&] { return !g.busy && g.pending.empty(); });
    g.busy = true;
    int rc = admit(s, g, lk);
    if (rc == DC_OK) {
        lk.unlock();
        dc_decomp_info info;
        rc = dc_decomp_info_get(g.h, &info);
        if (rc == DC_OK) {
            *kmax = info.kmax;
            if (kmaxes) rc = dc_get_kmaxes(g.h, kmaxes);
            if (rc == DC_OK && rows) {
                if (rows_capacity < (uint64_t)(info.kmax + 1) * g.V)
                    rc = set_error(DC_ERR_CAPACITY, "dc_server_graph_result: rows need %llu values",
                                   (unsigned long long)(info.kmax + 1) * g.V);
                else
                    rc = dc_get_lmax_rows(g.h, 0, (uint32_t)info.kmax + 1, rows);
            }
        }
        lk.lock();
    }
    g.busy = false;
    g.last_used = Clock::now();
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    return rc;
}

extern "C" int dc_server_set_row_repair(dc_server* s, int on) {
    if (!s) return set_error(DC_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    s->row_repair = on ? 1 : 0;
    return DC_OK;
}

extern "C" int dc_server_free(dc_server* s) {
    if (!s) return DC_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    for (auto& t : s->workers) t.join();
    for (auto& g : s->graphs)
        if (g.h) dc_graph_free(g.h);
    delete s;
    return DC_OK;
}
