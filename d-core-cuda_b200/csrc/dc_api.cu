// C ABI of the engine: graph handles, decomposition and result access.
// Each function names the reference entry point it stands in for; the
// declarations with full documentation are in include/dcore_b200.h.
#include <atomic>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <cmath>
#include <vector>
#include <sys/stat.h>

#include "dc_engine.cuh"
#include "dc_internal.h"

using namespace dc;

#define API_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess)                                                               \
            return set_error(DC_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e));  \
    } while (0)

namespace {

int select_device(const dc_graph_opts* o) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(DC_ERR_NO_DEVICE,
                         "no CUDA device available (%s); the engine runs on the GPU only and has no CPU fallback",
                         e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
    }
    if (o && o->device >= 0) {
        if (o->device >= n) return set_error(DC_ERR_INVALID, "device %d out of range (%d devices)", o->device, n);
        API_CUDA(cudaSetDevice(o->device));
    }
    return DC_OK;
}

int new_handle(const dc_graph_opts* o, dc_graph** out) {
    if (!out) return set_error(DC_ERR_INVALID, "null output handle");
    *out = nullptr;
    if (int rc = select_device(o)) return rc;
    dc_graph* h = new dc_graph();
    dc_graph_opts def;
    dc_graph_opts_default(&def);
    if (!o) o = &def;
    h->gap_min = o->gap_min;
    h->gap_div = o->gap_div;
    if (int rc = init_handle(h)) {
        dc_graph_free(h);
        return rc;
    }
    *out = h;
    return DC_OK;
}

bool file_exists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

}  // namespace

extern "C" void dc_graph_opts_default(dc_graph_opts* o) {
    if (!o) return;
    o->gap_min = 1;  // OFFSET_GAP (src/common.h:36)
    o->gap_div = 0;
    o->device = -1;
}

extern "C" int dc_device_count(int* n) {
    if (!n) return set_error(DC_ERR_INVALID, "null argument");
    *n = 0;
    cudaError_t e = cudaGetDeviceCount(n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *n = 0;
    }
    return DC_OK;
}

extern "C" int dc_reserve_device_memory(int device, uint64_t bytes) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
        cudaGetLastError();
        return set_error(DC_ERR_NO_DEVICE, "dc_reserve_device_memory: no CUDA device");
    }
    if (device < 0 || device >= n) return set_error(DC_ERR_INVALID, "dc_reserve_device_memory: bad device %d", device);
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    int rc = DC_OK;
    cudaMemPool_t pool;
    uint64_t keep = ~0ull;
    cudaStream_t st = nullptr;
    void* p = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess ||
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        rc = set_error(DC_ERR_CUDA, "dc_reserve_device_memory: pool setup failed");
    } else if (bytes) {
        if (cudaMallocAsync(&p, bytes, st) != cudaSuccess) {
            rc = set_error(DC_ERR_NOMEM, "dc_reserve_device_memory: %llu bytes not available",
                           (unsigned long long)bytes);
        } else {
            cudaFreeAsync(p, st);
        }
        if (cudaStreamSynchronize(st) != cudaSuccess && rc == DC_OK)
            rc = set_error(DC_ERR_CUDA, "dc_reserve_device_memory: synchronisation failed");
    }
    if (st) cudaStreamDestroy(st);
    cudaGetLastError();
    cudaSetDevice(cur);
    return rc;
}

extern "C" int dc_graph_create_device(uint32_t V, uint64_t E, const uint32_t* d_src, const uint32_t* d_dst,
                                      const dc_graph_opts* opts, dc_graph** out) {
    if (E && (!d_src || !d_dst)) return set_error(DC_ERR_INVALID, "dc_graph_create_device: null edge arrays");
    dc_graph* h = nullptr;
    if (int rc = new_handle(opts, &h)) return rc;
    if (int rc = build_from_device_edges(h, V, E, d_src, d_dst)) {
        dc_graph_free(h);
        return rc;
    }
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        dc_graph_free(h);
        return set_error(DC_ERR_CUDA, "graph build: %s", cudaGetErrorString(e));
    }
    *out = h;
    return DC_OK;
}

extern "C" int dc_graph_create(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                               const dc_graph_opts* opts, dc_graph** out) {
    if (E && (!src || !dst)) return set_error(DC_ERR_INVALID, "dc_graph_create: null edge arrays");
    dc_graph* h = nullptr;
    if (int rc = new_handle(opts, &h)) return rc;
    uint32_t *d_src = nullptr, *d_dst = nullptr;
    size_t bytes = (E ? E : 1) * sizeof(uint32_t);
    if (cudaMallocAsync(&d_src, bytes, h->stream) != cudaSuccess ||
        cudaMallocAsync(&d_dst, bytes, h->stream) != cudaSuccess) {
        cudaGetLastError();
        if (d_src) cudaFreeAsync(d_src, h->stream);
        dc_graph_free(h);
        return set_error(DC_ERR_NOMEM, "dc_graph_create: cannot stage %llu edges on the device", (unsigned long long)E);
    }
    int rc = DC_OK;
    if (E) {
        if (cudaMemcpyAsync(d_src, src, E * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
            cudaMemcpyAsync(d_dst, dst, E * 4, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
            rc = set_error(DC_ERR_CUDA, "dc_graph_create: edge upload failed");
    }
    if (rc == DC_OK) rc = build_from_device_edges(h, V, E, d_src, d_dst);
    cudaFreeAsync(d_src, h->stream);
    cudaFreeAsync(d_dst, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (rc == DC_OK && e != cudaSuccess) rc = set_error(DC_ERR_CUDA, "graph build: %s", cudaGetErrorString(e));
    if (rc != DC_OK) {
        dc_graph_free(h);
        return rc;
    }
    *out = h;
    return DC_OK;
}

// Graph(const string&) (src/graph.cpp:381-395): use the binary cache
// "<path>-binary-g=<gap>" when present, else parse the text file.  A path
// that itself names a "-binary-g=" file is read as binary.
extern "C" int dc_graph_load(const char* path, int prune, const dc_graph_opts* opts, dc_graph** out) {
    if (!path || !out) return set_error(DC_ERR_INVALID, "dc_graph_load: null argument");
    dc_graph_opts def;
    dc_graph_opts_default(&def);
    const dc_graph_opts* o = opts ? opts : &def;
    std::string p(path);
    std::string cache = p + "-binary-g=" + std::to_string(o->gap_min);
    std::string bin;
    if (p.find("-binary-g=") != std::string::npos) bin = p;
    else if (file_exists(cache)) bin = cache;
    if (!bin.empty()) {
        BinaryGraph b;
        if (int rc = read_binary_graph(bin.c_str(), b)) return rc;
        std::vector<uint32_t> s(b.E), d(b.E);
        uint64_t e = 0;
        for (uint32_t v = 0; v < b.V; ++v)
            for (int32_t i = 0; i < b.out_deg[v]; ++i) {
                s[e] = v;
                d[e] = b.out_nbr[b.out_off[v] + i];
                ++e;
            }
        return dc_graph_create(b.V, b.E, s.data(), d.data(), o, out);
    }
    uint32_t V = 0;
    std::vector<uint32_t> s, d;
    if (int rc = parse_text_graph(path, prune, &V, s, d)) return rc;
    return dc_graph_create(V, s.size(), s.data(), d.data(), o, out);
}

extern "C" int dc_graph_load_text_device(const char* path, int prune, const dc_graph_opts* opts, dc_graph** out) {
    if (!path || !out) return set_error(DC_ERR_INVALID, "dc_graph_load_text_device: null argument");
    dc_graph* h = nullptr;
    if (int rc = new_handle(opts, &h)) return rc;
    uint32_t V = 0;
    uint64_t E = 0;
    uint32_t *src = nullptr, *dst = nullptr;
    int rc = parse_text_graph_device(path, prune, h->stream, h->geom.sms, &V, &E, &src, &dst);
    if (rc == DC_OK) rc = build_from_device_edges(h, V, E, src, dst);
    if (src) cudaFreeAsync(src, h->stream);
    if (dst) cudaFreeAsync(dst, h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (rc == DC_OK && e != cudaSuccess) rc = set_error(DC_ERR_CUDA, "graph build: %s", cudaGetErrorString(e));
    if (rc != DC_OK) {
        dc_graph_free(h);
        return rc;
    }
    *out = h;
    return DC_OK;
}

extern "C" int dc_write_decomp_cpu_device(dc_graph* h, const char* path) {
    if (!h || !path) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (!h->d.full())
        return set_error(DC_ERR_STATE, "the decomposition holds row 0 and rows %d..%d only (dc_decompose_rows)",
                         h->d.row_lo, h->d.row_hi);
    API_CUDA(cudaSetDevice(h->device));
    return write_decomp_cpu_device(h, path);
}

extern "C" int dc_set_trace(dc_graph* h, uint32_t max_steps, dc_trace_fn fn, void* user) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (h->trace_dev) cudaFree(h->trace_dev);
    if (h->trace_host) cudaFreeHost(h->trace_host);
    h->trace_dev = nullptr;
    h->trace_host = nullptr;
    h->trace_cap = 0;
    h->trace_cb = nullptr;
    if (max_steps == 0 || !fn) return DC_OK;
    if (cudaMalloc(&h->trace_dev, 64ull * max_steps) != cudaSuccess ||
        cudaHostAlloc(&h->trace_host, 64ull * max_steps, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "trace buffers");
    }
    h->trace_cap = max_steps;
    h->trace_cb = fn;
    h->trace_user = user;
    return DC_OK;
}

extern "C" int dc_graph_free(dc_graph* h) {
    if (!h) return DC_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    dc_set_trace(h, 0, nullptr, nullptr);
    free_graph_arrays(h->g, h->stream);
    free_decomp(h->d, h->stream);
    free_scratch(h);
    dc::free_captured_batches(h);
    if (h->ctl) cudaFreeAsync(h->ctl, h->stream);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return DC_OK;
}

extern "C" int dc_graph_info(const dc_graph* h, uint32_t* V, uint64_t* E) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (V) *V = h->g.V;
    if (E) *E = h->g.E;
    return DC_OK;
}

extern "C" int dc_graph_device_bytes(const dc_graph* h, uint64_t* bytes) {
    if (!h || !bytes) return set_error(DC_ERR_INVALID, "null argument");
    *bytes = device_footprint(h);
    return DC_OK;
}

extern "C" int dc_graph_degrees(dc_graph* h, int32_t* in_deg, int32_t* out_deg) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (in_deg) API_CUDA(cudaMemcpyAsync(in_deg, h->g.in_len, 4ull * h->g.V, cudaMemcpyDeviceToHost, h->stream));
    if (out_deg) API_CUDA(cudaMemcpyAsync(out_deg, h->g.out_len, 4ull * h->g.V, cudaMemcpyDeviceToHost, h->stream));
    API_CUDA(cudaStreamSynchronize(h->stream));
    return DC_OK;
}

// Live edges of the device graph as (src, dst) pairs, src ascending, each
// out-list in ascending dst order.
extern "C" int dc_graph_get_edges(dc_graph* h, uint32_t* src, uint32_t* dst, uint64_t capacity, uint64_t* n_edges) {
    if (!h || !n_edges) return set_error(DC_ERR_INVALID, "null argument");
    const uint32_t V = h->g.V;
    std::vector<uint32_t> off((size_t)V + 1), nbr(h->g.out_cap ? h->g.out_cap : 1);
    std::vector<int32_t> len(V ? V : 1);
    if (V) {
        API_CUDA(cudaMemcpyAsync(off.data(), h->g.out_off, 4ull * (V + 1), cudaMemcpyDeviceToHost, h->stream));
        API_CUDA(cudaMemcpyAsync(len.data(), h->g.out_len, 4ull * V, cudaMemcpyDeviceToHost, h->stream));
        if (h->g.out_cap)
            API_CUDA(cudaMemcpyAsync(nbr.data(), h->g.out_nbr, 4ull * h->g.out_cap, cudaMemcpyDeviceToHost, h->stream));
    }
    API_CUDA(cudaStreamSynchronize(h->stream));
    uint64_t E = 0;
    for (uint32_t v = 0; v < V; ++v) E += (uint64_t)len[v];
    *n_edges = E;
    if (!src || !dst) return DC_OK;
    if (capacity < E) return set_error(DC_ERR_CAPACITY, "dc_graph_get_edges: capacity too small");
    uint64_t e = 0;
    for (uint32_t v = 0; v < V; ++v) {
        uint32_t* a = nbr.data() + off[v];
        std::sort(a, a + len[v]);
        for (int32_t i = 0; i < len[v]; ++i) {
            src[e] = v;
            dst[e] = a[i];
            ++e;
        }
    }
    return DC_OK;
}

// Graph::writeBinary (src/graph.cpp:261-285).
extern "C" int dc_graph_write_binary(dc_graph* h, const char* path, uint32_t gap) {
    if (!h || !path) return set_error(DC_ERR_INVALID, "null argument");
    uint64_t E = 0;
    if (int rc = dc_graph_get_edges(h, nullptr, nullptr, 0, &E)) return rc;
    std::vector<uint32_t> s(E ? E : 1), d(E ? E : 1);
    if (int rc = dc_graph_get_edges(h, s.data(), d.data(), E, &E)) return rc;
    return write_binary_graph(path, h->g.V, E, s.data(), d.data(), gap);
}

// dcore(Graph&) (main.cu:197-262) / checkDCore (main.cu:276-293).
extern "C" int dc_decompose(dc_graph* h, int method, int32_t* kmax, int32_t* lmax) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (method != DC_METHOD_INCREMENTAL && method != DC_METHOD_PEEL)
        return set_error(DC_ERR_INVALID, "unknown decomposition method %d", method);
    API_CUDA(cudaSetDevice(h->device));
    if (int rc = decompose(h, method, 0)) return rc;
    if (kmax) *kmax = h->d.kmax;
    if (lmax) *lmax = h->d.lmax;
    return DC_OK;
}

extern "C" int dc_decompose_rows(dc_graph* h, uint32_t k_first, uint32_t k_last, int32_t* kmax, int32_t* lmax) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    API_CUDA(cudaSetDevice(h->device));
    const int32_t k0 = (int32_t)std::min<uint32_t>(k_first, 0x7FFFFFFF);
    const int32_t k1 = (int32_t)std::min<uint32_t>(k_last, 0x7FFFFFFF);
    if (int rc = decompose_range(h, k0, k1)) return rc;
    if (kmax) *kmax = h->d.kmax;
    if (lmax) *lmax = h->d.lmax;
    return DC_OK;
}

extern "C" int dc_row_weights(dc_graph* h, uint64_t* weights, uint64_t capacity) {
    if (!h || !weights) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.peel_valid) return set_error(DC_ERR_STATE, "no kmax on this graph (dc_decompose_rows first)");
    if (capacity < (uint64_t)h->d.kmax + 1)
        return set_error(DC_ERR_CAPACITY, "dc_row_weights: need kmax + 1 = %d values", h->d.kmax + 1);
    API_CUDA(cudaSetDevice(h->device));
    return row_weights(h, weights);
}

extern "C" int dc_graph_kmax_edge_batches(dc_graph* h, uint64_t B, const uint32_t* d_from, const uint32_t* d_to,
                                          int64_t* d_batch_of, int64_t* n_batches) {
    if (!h || !n_batches || (B && (!d_from || !d_to || !d_batch_of)))
        return set_error(DC_ERR_INVALID, "dc_graph_kmax_edge_batches: null argument");
    if (!h->d.peel_valid) return set_error(DC_ERR_STATE, "no kmax on this graph (dc_decompose first)");
    API_CUDA(cudaSetDevice(h->device));
    return kmax_edge_batches_device(h, B, d_from, d_to, d_batch_of, n_batches);
}

extern "C" int dc_maintain(dc_graph* h, const uint32_t* pairs, const uint8_t* is_delete, uint64_t b, int method,
                           dc_maint_stats* stats) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    API_CUDA(cudaSetDevice(h->device));
    return maintain(h, pairs, is_delete, b, method, stats);
}

extern "C" int dc_set_row_repair(dc_graph* h, int on) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (on < 0 || on > 3) return set_error(DC_ERR_INVALID, "dc_set_row_repair: mode must be 0, 1, 2 or 3");
    h->row_repair = on;
    return DC_OK;
}

extern "C" int dc_set_captured_batches(dc_graph* h, int on) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    h->captured_batches = on != 0;
    return DC_OK;
}

extern "C" int dc_graph_set_scheduler(dc_graph* h, dc_sched* s) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    h->sched = s;
    return DC_OK;
}

extern "C" int dc_maint_log_enable(dc_graph* h, int on) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    h->log_maint = on != 0;
    if (!on) h->maint_log.clear();
    return DC_OK;
}

// Records of the batches maintained since logging was enabled: features[16],
// method, and total / core / rows milliseconds.
extern "C" int dc_maint_log_get(dc_graph* h, float* features, int32_t* methods, float* times_ms, uint64_t capacity,
                                uint64_t* n) {
    if (!h || !n) return set_error(DC_ERR_INVALID, "null argument");
    *n = h->maint_log.size();
    if (!features || !methods || !times_ms) return DC_OK;
    if (capacity < *n) return set_error(DC_ERR_CAPACITY, "dc_maint_log_get: capacity too small");
    for (uint64_t i = 0; i < *n; ++i) {
        const dc::MaintLogRec& r = h->maint_log[i];
        memcpy(features + 16 * i, r.feat, sizeof(r.feat));
        methods[i] = r.method;
        times_ms[3 * i] = r.total_ms;
        times_ms[3 * i + 1] = r.core_ms;
        times_ms[3 * i + 2] = r.rows_ms;
    }
    return DC_OK;
}

extern "C" int dc_decomp_info_get(dc_graph* h, dc_decomp_info* info) {
    if (!h || !info) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    memset(info, 0, sizeof(*info));
    info->kmax = h->d.kmax;
    info->lmax = h->d.lmax;
    info->n_corners = h->d.n_corners;
    info->kmax_ms = h->times.kmax_ms;
    info->row0_ms = h->times.row0_ms;
    info->rows_ms = h->times.trans_ms;
    info->skyline_ms = h->times.sky_ms;
    info->expand_ms = h->times.expand_ms;
    info->evals = h->stat_evals;
    info->drops = h->stat_drops;
    info->entries = h->stat_entries;
    return DC_OK;
}

extern "C" int dc_get_kmaxes(dc_graph* h, int32_t* out) {
    if (!h || !out) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (h->g.V) API_CUDA(cudaMemcpyAsync(out, h->d.kmax_v, 4ull * h->g.V, cudaMemcpyDeviceToHost, h->stream));
    API_CUDA(cudaStreamSynchronize(h->stream));
    return DC_OK;
}

extern "C" int dc_get_lmax_rows_device(dc_graph* h, uint32_t k0, uint32_t n, int32_t* d_out) {
    if (!h || (n && !d_out)) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if ((uint64_t)k0 + n > (uint64_t)h->d.kmax + 1)
        return set_error(DC_ERR_INVALID, "rows [%u, %llu) outside 0..kmax=%d", k0, (unsigned long long)k0 + n, h->d.kmax);
    if (!h->d.holds(k0, n))
        return set_error(DC_ERR_STATE, "rows [%u, %llu) not held: the decomposition holds row 0 and rows %d..%d",
                         k0, (unsigned long long)k0 + n, h->d.row_lo, h->d.row_hi);
    if (h->d.rows_valid) {
        if (n)
            API_CUDA(cudaMemcpyAsync(d_out, h->d.rows + (uint64_t)k0 * h->g.V, 4ull * n * h->g.V,
                                     cudaMemcpyDeviceToDevice, h->stream));
        return DC_OK;
    }
    return expand_rows(h, k0, n, d_out);
}

// The rows of g.lmaxes (main.cu:226-247) copied to host memory.
extern "C" int dc_get_lmax_rows(dc_graph* h, uint32_t k0, uint32_t n, int32_t* out) {
    if (!h || (n && !out)) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if ((uint64_t)k0 + n > (uint64_t)h->d.kmax + 1)
        return set_error(DC_ERR_INVALID, "rows [%u, %llu) outside 0..kmax=%d", k0, (unsigned long long)k0 + n, h->d.kmax);
    if (!h->d.holds(k0, n))
        return set_error(DC_ERR_STATE, "rows [%u, %llu) not held: the decomposition holds row 0 and rows %d..%d",
                         k0, (unsigned long long)k0 + n, h->d.row_lo, h->d.row_hi);
    const uint64_t V = h->g.V;
    if (n == 0 || V == 0) return DC_OK;
    if (h->d.rows_valid) {
        API_CUDA(cudaMemcpyAsync(out, h->d.rows + (uint64_t)k0 * V, 4ull * n * V, cudaMemcpyDeviceToHost, h->stream));
        API_CUDA(cudaStreamSynchronize(h->stream));
        return DC_OK;
    }
    // expand in chunks of rows through two device staging buffers
    uint64_t chunk_rows = std::max<uint64_t>(1, (256ull << 20) / (4 * V));
    chunk_rows = std::min<uint64_t>(chunk_rows, n);
    int32_t* stage[2] = {nullptr, nullptr};
    for (int i = 0; i < 2; ++i)
        if (cudaMallocAsync(&stage[i], 4 * chunk_rows * V, h->stream) != cudaSuccess) {
            cudaGetLastError();
            if (stage[0]) cudaFreeAsync(stage[0], h->stream);
            return set_error(DC_ERR_NOMEM, "row staging buffer allocation failed");
        }
    int rc = DC_OK;
    int b = 0;
    for (uint64_t r = 0; r < n && rc == DC_OK; r += chunk_rows, b ^= 1) {
        uint64_t m = std::min<uint64_t>(chunk_rows, n - r);
        rc = expand_rows(h, (uint32_t)(k0 + r), (uint32_t)m, stage[b]);
        if (rc == DC_OK && cudaMemcpyAsync(out + r * V, stage[b], 4 * m * V, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
            rc = set_error(DC_ERR_CUDA, "row download failed");
    }
    cudaFreeAsync(stage[0], h->stream);
    cudaFreeAsync(stage[1], h->stream);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (rc == DC_OK && e != cudaSuccess) rc = set_error(DC_ERR_CUDA, "row download: %s", cudaGetErrorString(e));
    return rc;
}

extern "C" int dc_materialize_rows(dc_graph* h) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (!h->d.full())
        return set_error(DC_ERR_STATE, "the decomposition holds row 0 and rows %d..%d only (dc_decompose_rows)",
                         h->d.row_lo, h->d.row_hi);
    if (h->d.rows_valid) return DC_OK;
    uint64_t elems = (uint64_t)(h->d.kmax + 1) * h->g.V;
    if (h->d.rows_cap < elems) {
        if (h->d.rows) cudaFreeAsync(h->d.rows, h->stream);
        h->d.rows = nullptr;
        h->d.rows_cap = 0;
        if (cudaMallocAsync(&h->d.rows, 4 * (elems ? elems : 1), h->stream) != cudaSuccess) {
            cudaGetLastError();
            return set_error(DC_ERR_NOMEM, "dense rows (%llu values) do not fit in device memory",
                             (unsigned long long)elems);
        }
        h->d.rows_cap = elems;
    }
    if (int rc = expand_rows(h, 0, (uint32_t)h->d.kmax + 1, h->d.rows)) return rc;
    API_CUDA(cudaStreamSynchronize(h->stream));
    h->d.rows_valid = true;
    return DC_OK;
}

extern "C" int dc_release_rows(dc_graph* h) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (h->d.rows) cudaFreeAsync(h->d.rows, h->stream);
    cudaStreamSynchronize(h->stream);
    h->d.rows = nullptr;
    h->d.rows_cap = 0;
    h->d.rows_valid = false;
    return DC_OK;
}

extern "C" int dc_get_skyline(dc_graph* h, uint32_t* off, int32_t* ks, int32_t* ls, uint64_t capacity,
                              uint64_t* n_corners) {
    if (!h || !n_corners) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (!h->d.full())
        return set_error(DC_ERR_STATE, "the decomposition holds row 0 and rows %d..%d only (dc_decompose_rows)",
                         h->d.row_lo, h->d.row_hi);
    *n_corners = h->d.n_corners;
    if (!off || !ks || !ls) return DC_OK;
    if (capacity < h->d.n_corners) return set_error(DC_ERR_CAPACITY, "dc_get_skyline: capacity too small");
    const uint64_t V = h->g.V;
    API_CUDA(cudaMemcpyAsync(off, h->d.sky_off, 4 * (V + 1), cudaMemcpyDeviceToHost, h->stream));
    if (h->d.n_corners) {
        API_CUDA(cudaMemcpyAsync(ks, h->d.sky_k, 4 * h->d.n_corners, cudaMemcpyDeviceToHost, h->stream));
        API_CUDA(cudaMemcpyAsync(ls, h->d.sky_l, 4 * h->d.n_corners, cudaMemcpyDeviceToHost, h->stream));
    }
    API_CUDA(cudaStreamSynchronize(h->stream));
    return DC_OK;
}

// writeDecompFile (src/utils.h:98-109).
extern "C" int dc_write_decomp(dc_graph* h, const char* path) {
    if (!h || !path) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (!h->d.full())
        return set_error(DC_ERR_STATE, "the decomposition holds row 0 and rows %d..%d only (dc_decompose_rows)",
                         h->d.row_lo, h->d.row_hi);
    const uint64_t V = h->g.V;
    std::vector<int32_t> km(V ? V : 1), rows((uint64_t)(h->d.kmax + 1) * V + 1);
    if (int rc = dc_get_kmaxes(h, km.data())) return rc;
    if (int rc = dc_get_lmax_rows(h, 0, (uint32_t)h->d.kmax + 1, rows.data())) return rc;
    return dc_decomp_file_write(path, (uint32_t)V, h->d.kmax, h->d.lmax, km.data(), rows.data());
}

// writeDecompFileCPU (src/utils.h:110-124).
extern "C" int dc_write_decomp_cpu(dc_graph* h, const char* path) {
    if (!h || !path) return set_error(DC_ERR_INVALID, "null argument");
    if (!h->d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (!h->d.full())
        return set_error(DC_ERR_STATE, "the decomposition holds row 0 and rows %d..%d only (dc_decompose_rows)",
                         h->d.row_lo, h->d.row_hi);
    const uint64_t V = h->g.V;
    std::vector<int32_t> km(V ? V : 1), rows((uint64_t)(h->d.kmax + 1) * V + 1);
    if (int rc = dc_get_kmaxes(h, km.data())) return rc;
    if (int rc = dc_get_lmax_rows(h, 0, (uint32_t)h->d.kmax + 1, rows.data())) return rc;
    return dc_decomp_cpu_file_write(path, (uint32_t)V, km.data(), rows.data());
}

// Launch-shape knobs of the persistent kernels (tuning).
extern "C" int dc_set_launch(dc_graph* h, int blocks_per_sm) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (blocks_per_sm < 0 || blocks_per_sm > 8) return set_error(DC_ERR_INVALID, "blocks_per_sm must be 0..8");
    h->blocks_per_sm = blocks_per_sm;
    h->peel_bps = 0;
    h->rows_bps = 0;
    return DC_OK;
}

extern "C" int dc_set_wait_limit(dc_graph* h, uint64_t ns) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (ns != 0 && (ns < 1000000ull || ns > 600000000000ull))
        return set_error(DC_ERR_INVALID, "wait limit must be 0 (default) or 1 ms .. 600 s");
    h->wait_ns = ns;
    return DC_OK;
}

extern "C" int dc_test_withhold_barrier(dc_graph* h, int32_t block) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    if (block < -1) return set_error(DC_ERR_INVALID, "block must be -1 (off) or a block index");
    h->barrier_fault_block = block;
    return DC_OK;
}

extern "C" int dc_get_tuning(dc_graph* h, dc_tuning* t) {
    if (!h || !t) return set_error(DC_ERR_INVALID, "null argument");
    const int dflt = h->blocks_per_sm > 0 ? h->blocks_per_sm : 2;
    t->peel_blocks_per_sm = h->peel_bps > 0 ? h->peel_bps : dflt;
    t->rows_blocks_per_sm = h->rows_bps > 0 ? h->rows_bps : dflt;
    t->peel_chunk = (int32_t)h->peel_chunk;
    for (int i = 0; i < kMaxRowSegments - 1; ++i) t->rows_split_permille[i] = h->rows_split[i];
    return DC_OK;
}

extern "C" int dc_set_tuning(dc_graph* h, const dc_tuning* t) {
    if (!h || !t) return set_error(DC_ERR_INVALID, "null argument");
    if (t->peel_blocks_per_sm < 1 || t->peel_blocks_per_sm > 8 || t->rows_blocks_per_sm < 1 ||
        t->rows_blocks_per_sm > 8)
        return set_error(DC_ERR_INVALID, "dc_set_tuning: blocks per SM must be 1..8");
    if (t->peel_chunk < 16 || t->peel_chunk > 4096 || (t->peel_chunk & (t->peel_chunk - 1)))
        return set_error(DC_ERR_INVALID, "dc_set_tuning: peel_chunk must be a power of two in 16..4096");
    constexpr int kCuts = kMaxRowSegments - 1;
    static_assert(sizeof(t->rows_split_permille) == kCuts * sizeof(int32_t), "dc_tuning holds one cut per extra segment");
    for (int i = 0; i < kCuts; ++i) {
        const int32_t c = t->rows_split_permille[i];
        const bool ok = c == 0 ? (i == kCuts - 1 || t->rows_split_permille[i + 1] == 0)
                               : (c <= 999 && (i == 0 || (t->rows_split_permille[i - 1] > 0 &&
                                                          c > t->rows_split_permille[i - 1])));
        if (c < 0 || !ok)
            return set_error(DC_ERR_INVALID,
                             "dc_set_tuning: rows_split_permille must hold ascending values in 1..999, then zeros");
    }
    h->peel_bps = t->peel_blocks_per_sm;
    h->rows_bps = t->rows_blocks_per_sm;
    h->peel_chunk = (unsigned)t->peel_chunk;
    for (int i = 0; i < kCuts; ++i) h->rows_split[i] = t->rows_split_permille[i];
    API_CUDA(cudaSetDevice(h->device));
    return prepare_row_segments(h);
}

// Smallest largest-segment cost over ncut cuts taken from the grid: best[j][i]
// = the best largest cost of rows 1..s_i cut j times with the last cut at i,
// best[j][i] = min over p < i of max(best[j-1][p], cost[i] - cost[p]); the
// last segment adds total - cost[i].  O(ncut n^2); ties keep the lower cut.
extern "C" int dc_plan_row_cuts(const int32_t* grid, const float* cost, int32_t n, float total, int32_t ncut,
                                int32_t* cuts, float* longest) {
    constexpr int kCuts = kMaxRowSegments - 1;
    if (!grid || !cost || !cuts) return set_error(DC_ERR_INVALID, "dc_plan_row_cuts: null argument");
    if (n < 1 || n > 4096 || ncut < 1 || ncut > kCuts || ncut > n)
        return set_error(DC_ERR_INVALID, "dc_plan_row_cuts: need 1 <= n <= 4096 and 1 <= ncut <= min(n, %d)", kCuts);
    for (int i = 0; i < n; ++i)
        if (grid[i] < 1 || grid[i] > 999 || (i && grid[i] <= grid[i - 1]))
            return set_error(DC_ERR_INVALID, "dc_plan_row_cuts: grid must be strictly ascending in 1..999");
    std::vector<float> best((size_t)ncut * n);
    std::vector<int32_t> from((size_t)ncut * n, -1);
    for (int i = 0; i < n; ++i) best[i] = cost[i];
    for (int j = 1; j < ncut; ++j)
        for (int i = 0; i < n; ++i) {
            float b = INFINITY;
            int32_t arg = -1;
            for (int p = j - 1; p < i; ++p) {
                const float v = std::max(best[(size_t)(j - 1) * n + p], cost[i] - cost[p]);
                if (v < b) {
                    b = v;
                    arg = p;
                }
            }
            best[(size_t)j * n + i] = b;
            from[(size_t)j * n + i] = arg;
        }
    float b = INFINITY;
    int32_t last = -1;
    for (int i = ncut - 1; i < n; ++i) {
        const float v = std::max(best[(size_t)(ncut - 1) * n + i], total - cost[i]);
        if (v < b) {
            b = v;
            last = i;
        }
    }
    for (int j = ncut - 1; j >= 0; --j) {
        cuts[j] = grid[last];
        last = from[(size_t)j * n + last];
    }
    if (longest) *longest = b;
    return DC_OK;
}

// Coordinate search: the fused peel's grid and chunk size timed on the peel
// alone, then the row kernel's grid timed on the rows alone (kmax and row 0
// reused); every candidate runs twice and keeps its faster time.  The
// fastest setting stays on the handle, which ends with a full
// decomposition.
extern "C" int dc_autotune(dc_graph* h, dc_tuning* best, float* best_ms) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    API_CUDA(cudaSetDevice(h->device));
    dc_tuning cur;
    dc_get_tuning(h, &cur);
    if (int rc = decompose_range(h, 0, 0)) return rc;  // warm-up
    float peel_best = 1e30f;
    dc_tuning pick = cur;
    for (int bps = 1; bps <= 6; ++bps)
        for (int chunk = 32; chunk <= 256; chunk *= 2) {
            dc_tuning t = pick;
            t.peel_blocks_per_sm = bps;
            t.peel_chunk = chunk;
            dc_set_tuning(h, &t);
            float ms = 1e30f;
            for (int r = 0; r < 2; ++r) {
                if (int rc = decompose_range(h, 0, 0)) return rc;
                ms = std::min(ms, h->times.kmax_ms);
            }
            if (ms < peel_best) {
                peel_best = ms;
                pick.peel_blocks_per_sm = bps;
                pick.peel_chunk = chunk;
            }
        }
    dc_set_tuning(h, &pick);
    if (int rc = decompose_range(h, 0, 0)) return rc;
    float rows_best = 1e30f;
    const int32_t K = h->d.kmax;
    for (int bps = 1; bps <= 8; ++bps) {
        dc_tuning t = pick;
        t.rows_blocks_per_sm = bps;
        dc_set_tuning(h, &t);
        float ms = 1e30f;
        for (int r = 0; r < 2; ++r) {
            if (int rc = decompose_range(h, 1, K)) return rc;
            ms = std::min(ms, h->times.trans_ms);
        }
        if (ms < rows_best) {
            rows_best = ms;
            pick.rows_blocks_per_sm = bps;
        }
    }
    // row segments: a run of rows 1..s costs C(s) and (starting from the
    // vertices of C_{s+1} with the rest already left) rows s+1..kmax cost
    // about C(kmax) - C(s), so segments balance where the cumulative cost
    // splits evenly.  C is measured at cuts of 5..90 % of kmax; for one to
    // three cuts the set with the smallest predicted longest segment is
    // timed for real, and the fastest of those and no split stays.  (More
    // segments share the SMs too thinly: at R-MAT 22 five to eight measured
    // slower than four.)
    constexpr int kGrid = 18;
    int32_t grid[kGrid];
    float cost[kGrid];
    int ng = 0;
    dc_set_tuning(h, &pick);  // C measured at the chosen row grid
    for (int g = 0; g < kGrid && K >= kMinSplitRows; ++g) {  // shorter runs are never split
        const int32_t c = 50 * (g + 1);
        const int32_t srow = (int32_t)((int64_t)K * c / 1000);
        if (srow < 1 || srow >= K || (ng && srow == (int32_t)((int64_t)K * grid[ng - 1] / 1000))) continue;
        if (int rc = decompose_range(h, 1, srow)) return rc;
        grid[ng] = c;
        cost[ng++] = h->times.trans_ms;
    }
    const float total = rows_best;
    constexpr int kCuts = kMaxRowSegments - 1, kTunedCuts = 3;
    for (int ncut = 1; ncut <= kTunedCuts && ncut <= ng; ++ncut) {
        int32_t sel[kCuts] = {};
        if (dc_plan_row_cuts(grid, cost, ng, total, ncut, sel, nullptr) != DC_OK) break;
        dc_tuning t = pick;
        for (int q = 0; q < kCuts; ++q) t.rows_split_permille[q] = q < ncut ? sel[q] : 0;
        if (dc_set_tuning(h, &t) != DC_OK) continue;
        float ms = 1e30f;
        for (int r = 0; r < 3; ++r) {
            if (int rc = decompose_range(h, 1, K)) return rc;
            ms = std::min(ms, h->times.trans_ms);
        }
        if (ms < rows_best) {
            rows_best = ms;
            for (int q = 0; q < kCuts; ++q) pick.rows_split_permille[q] = t.rows_split_permille[q];
        }
    }
    dc_set_tuning(h, &pick);
    if (int rc = decompose(h, 0, 0)) return rc;
    if (best) *best = pick;
    if (best_ms) *best_ms = peel_best + rows_best;
    return DC_OK;
}

extern "C" int dc_host_alloc(uint64_t bytes, void** p) {
    if (!p) return set_error(DC_ERR_INVALID, "null argument");
    *p = nullptr;
    cudaError_t e = cudaHostAlloc(p, bytes ? bytes : 1, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_error(DC_ERR_NOMEM, "pinned host allocation of %llu bytes failed: %s", (unsigned long long)bytes,
                         cudaGetErrorString(e));
    }
    return DC_OK;
}

extern "C" int dc_host_free(void* p) {
    if (p) cudaFreeHost(p);
    return DC_OK;
}

namespace dc {
extern std::atomic<unsigned long long> g_launches;
}

extern "C" int dc_launch_count(unsigned long long* n) {
    if (!n) return set_error(DC_ERR_INVALID, "null argument");
    *n = dc::g_launches.load();
    return DC_OK;
}

extern "C" int dc_synchronize(dc_graph* h) {
    if (!h) return set_error(DC_ERR_INVALID, "null graph");
    API_CUDA(cudaStreamSynchronize(h->stream));
    return DC_OK;
}

extern "C" int dc_graph_stream(dc_graph* h, void** stream) {
    if (!h || !stream) return set_error(DC_ERR_INVALID, "null argument");
    *stream = (void*)h->stream;
    return DC_OK;
}
