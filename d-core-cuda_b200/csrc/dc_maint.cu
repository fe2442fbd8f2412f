// D-core maintenance under batches of edge insertions and deletions.
//
// Reference path (llysdal/d-core-cuda):
//   maintenanceFast (main.cu:1665-1751) and maintenance (main.cu:1536-1663):
//   device-side edge insertion (graphInsertEdges, src/graph_gpu.cu:49-74),
//   kmax maintenance by h-index refinement from +1 upper bounds
//   (kmaxMaintenance, main.cu:668-759, over sub-batches from
//   getKmaxEdgeBatches, main.cu:1441-1525), then a full re-peel of rows
//   k = 0..M+1 where M = max over batch edges of min(kmax[u], kmax[v])
//   (findMValue, main.cu:344-364; main.cu:1735-1743).  Deletion is not
//   implemented there (graph.cpp:73-108, graph_gpu.h:18-19).
//
// This engine keeps the same outcome -- after every batch the result equals
// a full decomposition of the updated graph -- and supports deletions:
//   1. the batch is reduced to its net effect per edge (sequential
//      semantics), deletions are validated, then applied by swap-remove;
//      insertions go into per-list free slots (the store is rebuilt with
//      more slack when a list is full);
//   2. kmax and row 0 are updated either locally (h-index refinement from
//      valid upper bounds on the region that can change) or by the fused
//      full peel;
//   3. rows 1..R are recomputed row to row from the new row 0, where R bounds
//      every row an updated edge or a changed kmax can reach; rows above R
//      keep their skyline corners.
#include <atomic>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dc_engine.cuh"
#include "dc_internal.h"

namespace dc {

extern std::atomic<unsigned long long> g_launches;

#define MT_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess)                                                               \
            return set_error(DC_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), \
                             __FILE__, __LINE__);                                            \
    } while (0)

static constexpr int kMThreads = 256;
static constexpr int kMWarps = kMThreads / 32;

// Stream-ordered pool allocations on the handle's stream (no implicit
// device-wide synchronisation between handles).
template <typename T>
static int mt_malloc(cudaStream_t st, T** p, uint64_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    if (cudaMallocAsync((void**)p, n * sizeof(T), st) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_error(DC_ERR_NOMEM, "device allocation of %llu bytes failed", (unsigned long long)(n * sizeof(T)));
    }
    return DC_OK;
}
template <typename T>
static void mt_free(cudaStream_t st, T*& p) {
    if (p) cudaFreeAsync((void*)p, st);
    p = nullptr;
}

static int mgrid(dc_graph* h, uint64_t n) {
    uint64_t b = (n + kMThreads - 1) / kMThreads;
    uint64_t cap = (uint64_t)h->geom.sms * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// ---------------------------------------------------------------------------
// graph updates
// ---------------------------------------------------------------------------

// Warp per distinct deleted pair: the out-list of u must hold v at least
// `need` times.
__global__ void k_del_validate(uint32_t n, const uint32_t* du, const uint32_t* dv, const int32_t* need,
                               const uint32_t* out_off, const int32_t* out_len, const uint32_t* out_nbr,
                               EngineCtl* c) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = gw; i < n; i += nw) {
        uint32_t u = du[i], v = dv[i];
        const uint32_t* a = out_nbr + out_off[u];
        int len = out_len[u], cnt = 0;
        for (int e = lane; e < len; e += 32) cnt += (a[e] == v);
#pragma unroll
        for (int s = 16; s; s >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, s);
        if (lane == 0 && cnt < need[i]) set_dev_error(c, DC_DEV_ERR_NOTFOUND, 30);
    }
}

// Warp per list: removes the listed neighbours (one occurrence each, in
// order) by swapping with the last live entry.  All deletions of one list
// are in one group, so no two warps touch the same list.
// run: nullptr, or a device flag that must be nonzero for the kernel to act
// (a captured batch skips its updates when the batch failed validation).
__global__ void k_del_apply(uint32_t ngroups, const uint32_t* gvert, const uint32_t* goff, const uint32_t* gnbr,
                            const uint32_t* off, int32_t* len, uint32_t* nbr, EngineCtl* c, const int* run) {
    if (run && !*run) return;
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = gw; g < ngroups; g += nw) {
        uint32_t v = gvert[g];
        uint32_t* a = nbr + off[v];
        int n = len[v];
        for (uint32_t t = goff[g]; t < goff[g + 1]; ++t) {
            uint32_t x = gnbr[t];
            int pos = -1;
            for (int b = 0; b < n && pos < 0; b += 32) {
                int e = b + (int)lane;
                unsigned m = __ballot_sync(0xFFFFFFFFu, e < n && a[e] == x);
                if (m) pos = b + __ffs(m) - 1;
            }
            if (pos < 0) {
                if (lane == 0) set_dev_error(c, DC_DEV_ERR_NOTFOUND, 31);
                break;
            }
            if (lane == 0) {
                a[pos] = a[n - 1];
            }
            --n;
            __syncwarp();
        }
        if (lane == 0) len[v] = n;
    }
}

__global__ void k_ins_need(uint32_t n, const uint32_t* iu, const uint32_t* iv, int32_t* need_out, int32_t* need_in) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        atomicAdd(&need_out[iu[i]], 1);
        atomicAdd(&need_in[iv[i]], 1);
    }
}

__global__ void k_ins_fits(uint32_t V, const uint32_t* out_off, const int32_t* out_len, const int32_t* need_out,
                           const uint32_t* in_off, const int32_t* in_len, const int32_t* need_in, EngineCtl* c) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        if ((uint64_t)out_len[v] + need_out[v] > out_off[v + 1] - out_off[v] ||
            (uint64_t)in_len[v] + need_in[v] > in_off[v + 1] - in_off[v])
            set_dev_error(c, DC_DEV_ERR_CAPACITY, 32);
    }
}

// Appends each edge to the free slots of both lists (capacity checked).
__global__ void k_ins_apply(uint32_t n, const uint32_t* iu, const uint32_t* iv, const uint32_t* out_off,
                            int32_t* out_len, uint32_t* out_nbr, const uint32_t* in_off, int32_t* in_len,
                            uint32_t* in_nbr, const int* run) {
    if (run && !*run) return;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t u = iu[i], v = iv[i];
        int po = atomicAdd(&out_len[u], 1);
        out_nbr[out_off[u] + po] = v;
        int pi = atomicAdd(&in_len[v], 1);
        in_nbr[in_off[v] + pi] = u;
    }
}

// Edge list of the current store (src ascending) into src/dst, using the
// exclusive scan of out_len in eoff.
__global__ void k_store_edges(uint32_t V, const uint32_t* off, const int32_t* len, const unsigned long long* eoff,
                              const uint32_t* nbr, uint32_t* src, uint32_t* dst) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = gw; v < V; v += nw) {
        uint32_t o = off[v];
        int n = len[v];
        uint64_t e0 = eoff[v];
        for (int i = lane; i < n; i += 32) {
            src[e0 + i] = (uint32_t)v;
            dst[e0 + i] = nbr[o + i];
        }
    }
}

__global__ void k_len_to_u64(uint32_t V, const int32_t* len, unsigned long long* out) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        out[v] = (unsigned long long)len[v];
}

// ---------------------------------------------------------------------------
// local maintenance of one core (kmax: in-degree core; row 0: out-degree core)
// ---------------------------------------------------------------------------
// val(v) = max L such that at least L neighbours w in v's count list have
// val(w) >= L (the h-index of the count-list values).  For kmax the count
// list is the in-list (the in-degree core, KList over swapped lists,
// main.cu:218-220); for row 0 it is the out-list.  A vertex's dependents are
// the vertices whose count lists contain it.
struct CoreParams {
    uint32_t V;
    const uint32_t* c_off;
    const int32_t* c_len;
    const uint32_t* c_nbr;
    const uint32_t* d_off;
    const int32_t* d_len;
    const uint32_t* d_nbr;
    int32_t* val;        // exact values before the update on entry, exact after on exit
    const int32_t* old;  // copy of val at entry
    uint32_t* mark;      // queue state per vertex (0 at entry and exit)
    int32_t* stamp;      // region marks
    int32_t stamp_id;
    uint32_t* cand;      // region (insert mode)
    unsigned cand_cap;
    const uint32_t* seeds;
    uint32_t n_seeds;
    int insert_mode;
    int32_t b;  // an insert batch raises no value by more than b
    TicketQueue q;
    EngineCtl* ctl;
    const int* run;  // nullptr, or a device flag that must be nonzero for the kernel to act
};

__device__ __forceinline__ bool core_request(uint32_t* m, EngineCtl* c) {
    unsigned s = ld_vol(m);
    for (int it = 0; it < 1024; ++it) {
        if (s == 0u) {
            unsigned o = atomicCAS(m, 0u, 1u);
            if (o == 0u) return true;
            s = o;
        } else if (s == 2u) {
            unsigned o = atomicCAS(m, 2u, 3u);
            if (o == 2u) return false;
            s = o;
        } else {
            return false;
        }
    }
    set_dev_error(c, DC_DEV_ERR_TIMEOUT, 33);
    return false;
}

struct CoreHook {
    unsigned nworkers;
    __device__ void operator()(EngineCtl* c) const {
        c->t_tail = c->t_head;
        c->outstanding = (int)nworkers;
        c->phase_done = 0;
        c->step++;
        __threadfence();
    }
};

__device__ __forceinline__ void core_block_done(EngineCtl* c, unsigned* s_cnt) {
    __syncwarp();
    if ((threadIdx.x & 31u) == 0) {
        __threadfence();
        unsigned o = atomicAdd(s_cnt, 1u);
        if (o == kMWarps - 1) {
            *s_cnt = 0;
            tq_finish(c, 1);
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kMThreads) k_core_local(CoreParams p) {
    if (p.run && !*(const volatile int*)p.run) return;  // every block returns: no barrier is entered
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const unsigned gwarp = blockIdx.x * kMWarps + wib;
    const unsigned nwarps = gridDim.x * kMWarps;
    EngineCtl* c = p.ctl;
    CoreHook hook{gridDim.x};
    __shared__ unsigned s_prod;
    __shared__ int s_bins[kMWarps][64];
    int* bins = s_bins[wib];
    if (threadIdx.x == 0) s_prod = 0;
    if (!grid_sync_hook(c, hook)) return;
    unsigned ticket = kNoTicket;
    unsigned long long item;

    if (p.insert_mode) {
        // ---- phase A: region that can rise, grown from the roots along
        // dependents whose old value is within b-1 of the current vertex, and
        // kept only where enough count-list neighbours could end at or above
        // the next level
        for (uint32_t base = gwarp * 32; base < p.n_seeds; base += nwarps * 32) {
            uint32_t i = base + lane;
            bool push = false;
            uint32_t r = 0;
            if (i < p.n_seeds) {
                r = p.seeds[i];
                push = atomicExch(&p.stamp[r], p.stamp_id) != p.stamp_id;
            }
            tq_push_warp(c, p.q, push, r);
        }
        core_block_done(c, &s_prod);
        while (tq_take_warp(c, p.q, &ticket, &item)) {
            const uint32_t x = (uint32_t)item;
            const int ox = p.old[x];
            const uint32_t* a = p.c_nbr + p.c_off[x];
            const int n = p.c_len[x];
            int sup = 0;
            for (int e = lane; e < n; e += 32) sup += (p.old[a[e]] >= ox + 1 - p.b);
#pragma unroll
            for (int s = 16; s; s >>= 1) sup += __shfl_xor_sync(0xFFFFFFFFu, sup, s);
            if (sup >= ox + 1) {
                if (lane == 0) {
                    unsigned pos = atomicAdd(&c->log_count, 1u);
                    if (pos < p.cand_cap) p.cand[pos] = x;
                    else set_dev_error(c, DC_DEV_ERR_CAPACITY, 34);
                }
                const uint32_t* dl = p.d_nbr + p.d_off[x];
                const int m = p.d_len[x];
                for (int b0 = 0; b0 < m; b0 += 32) {
                    int e = b0 + (int)lane;
                    bool push = false;
                    uint32_t y = 0;
                    if (e < m) {
                        y = dl[e];
                        int oy = p.old[y];
                        push = oy >= ox - (p.b - 1) && oy <= ox + (p.b - 1) &&
                               atomicExch(&p.stamp[y], p.stamp_id) != p.stamp_id;
                    }
                    tq_push_warp(c, p.q, push, y);
                }
            }
            __syncwarp();
            if (lane == 0) tq_finish(c, 1);
        }
        if (!grid_sync_hook(c, hook)) return;
        // raise the region to its bound
        const unsigned ncand = min(ld_vol(&c->log_count), p.cand_cap);
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ncand; i += gridDim.x * blockDim.x) {
            uint32_t x = p.cand[i];
            p.val[x] = min(p.old[x] + p.b, p.c_len[x]);
        }
        if (!grid_sync_hook(c, hook)) return;
    }

    // ---- phase B: h-index refinement from the upper bounds
    {
        const uint32_t* src = p.insert_mode ? p.cand : p.seeds;
        const uint32_t nsrc = p.insert_mode ? min(ld_vol(&c->log_count), p.cand_cap) : p.n_seeds;
        for (uint32_t base = gwarp * 32; base < nsrc; base += nwarps * 32) {
            uint32_t i = base + lane;
            bool push = false;
            uint32_t x = 0;
            if (i < nsrc) {
                x = src[i];
                push = core_request(&p.mark[x], c);
            }
            tq_push_warp(c, p.q, push, x);
        }
    }
    core_block_done(c, &s_prod);
    unsigned long long drops = 0;
    while (tq_take_warp(c, p.q, &ticket, &item)) {
        const uint32_t x = (uint32_t)item;
        if (lane == 0) {
            atomicExch(&p.mark[x], 2u);
            __threadfence();
        }
        __syncwarp();
        const int cap = ld_vol(&p.val[x]);
        const uint32_t* a = p.c_nbr + p.c_off[x];
        const int n = p.c_len[x];
        int nv = 0;
        if (cap > 0) {
            int carry = 0, hi = cap;
            bool first = true;
            for (;;) {
                int lo = max(0, hi - 63);
                bins[lane] = 0;
                bins[lane + 32] = 0;
                __syncwarp();
                for (int e = lane; e < n; e += 32) {
                    int cw = ld_vol(&p.val[a[e]]);
                    if (cw >= lo) {
                        if (cw >= hi) {
                            if (first || cw == hi) atomicAdd(&bins[hi - lo], 1);
                        } else {
                            atomicAdd(&bins[cw - lo], 1);
                        }
                    }
                }
                __syncwarp();
                int b0 = 2 * lane, b1 = 2 * lane + 1;
                int h0 = bins[b0], h1 = bins[b1];
                int pp = h0 + h1, sc = pp;
#pragma unroll
                for (int s = 1; s < 32; s <<= 1) {
                    int y = __shfl_down_sync(0xFFFFFFFFu, sc, s);
                    if (lane + s < 32) sc += y;
                }
                int cum1 = carry + (sc - pp) + h1, cum0 = cum1 + h0;
                bool ok1 = lo + b1 <= hi && cum1 >= lo + b1;
                bool ok0 = lo + b0 <= hi && cum0 >= lo + b0;
                unsigned m1 = __ballot_sync(0xFFFFFFFFu, ok1), m0 = __ballot_sync(0xFFFFFFFFu, ok0);
                int best = -1;
                if (m1) best = lo + 2 * (31 - __clz(m1)) + 1;
                if (m0) best = max(best, lo + 2 * (31 - __clz(m0)));
                if (best >= 0) {
                    nv = best;
                    break;
                }
                carry += __shfl_sync(0xFFFFFFFFu, sc, 0);
                first = false;
                if (lo == 0) {
                    nv = 0;
                    break;
                }
                hi = lo - 1;
                __syncwarp();
            }
        }
        bool requeue = false;
        if (nv < cap) {
            ++drops;
            if (lane == 0) {
                atomicExch(&p.val[x], nv);
                __threadfence();
            }
            __syncwarp();
            __threadfence();
            const uint32_t* dl = p.d_nbr + p.d_off[x];
            const int m = p.d_len[x];
            for (int b0 = 0; b0 < m; b0 += 32) {
                int e = b0 + (int)lane;
                bool push = false;
                uint32_t y = 0;
                if (e < m) {
                    y = dl[e];
                    int cy = ld_vol(&p.val[y]);
                    push = cy > nv && cy <= cap && core_request(&p.mark[y], c);
                }
                tq_push_warp(c, p.q, push, y);
            }
        }
        if (lane == 0) {
            if (nv < cap && nv > 0) {
                atomicExch(&p.mark[x], 1u);
                requeue = true;
            } else {
                unsigned o = atomicCAS(&p.mark[x], 2u, 0u);
                if (o == 3u) {
                    if (nv > 0) {
                        atomicExch(&p.mark[x], 1u);
                        requeue = true;
                    } else {
                        atomicExch(&p.mark[x], 0u);
                    }
                }
            }
        }
        tq_push_warp(c, p.q, requeue, x);
        if (lane == 0) tq_finish(c, 1);
    }
    if (lane == 0) atomicAdd(&c->drops, drops);
}

// ---------------------------------------------------------------------------
// batch features for the scheduler
// ---------------------------------------------------------------------------
// acc: [0] sum log2(1+deg) over endpoints, [1] sum min-kmax, [2] dense-core
// edges, [3] sum row-0 value over endpoints, [4] sum of degree x kmax over
// endpoints (the list entries a row repair scans at least once; floats);
// iacc: [0] max deg, [1] max min-kmax (ints)
__global__ void k_batch_features(uint32_t n, const uint32_t* u, const uint32_t* v, const int32_t* kmax,
                                 const int32_t* row0, const int32_t* in_len, const int32_t* out_len, int K, float* acc,
                                 int* iacc) {
    float a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0;
    int m0 = 0, m1 = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t x = u[i], y = v[i];
        int dx = in_len[x] + out_len[x], dy = in_len[y] + out_len[y];
        a0 += log2f(1.f + dx) + log2f(1.f + dy);
        int mk = min(kmax[x], kmax[y]);
        a1 += mk;
        a2 += (2 * mk >= K) ? 1.f : 0.f;
        a3 += row0[x] + row0[y];
        a4 += (float)dx * (float)max(kmax[x], 0) + (float)dy * (float)max(kmax[y], 0);
        m0 = max(m0, max(dx, dy));
        m1 = max(m1, mk);
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) {
        a0 += __shfl_xor_sync(0xFFFFFFFFu, a0, s);
        a1 += __shfl_xor_sync(0xFFFFFFFFu, a1, s);
        a2 += __shfl_xor_sync(0xFFFFFFFFu, a2, s);
        a3 += __shfl_xor_sync(0xFFFFFFFFu, a3, s);
        a4 += __shfl_xor_sync(0xFFFFFFFFu, a4, s);
        m0 = max(m0, __shfl_xor_sync(0xFFFFFFFFu, m0, s));
        m1 = max(m1, __shfl_xor_sync(0xFFFFFFFFu, m1, s));
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(&acc[0], a0);
        atomicAdd(&acc[1], a1);
        atomicAdd(&acc[2], a2);
        atomicAdd(&acc[3], a3);
        atomicAdd(&acc[4], a4);
        atomicMax(&iacc[0], m0);
        atomicMax(&iacc[1], m1);
    }
}

// ---------------------------------------------------------------------------
// bound on the rows a batch can change
// ---------------------------------------------------------------------------
__global__ void k_rows_bound_edges(uint32_t n, const uint32_t* u, const uint32_t* v, const int32_t* kold,
                                   const int32_t* knew, int* out) {
    int m = -1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        m = max(m, min(kold[u[i]], kold[v[i]]));
        m = max(m, min(knew[u[i]], knew[v[i]]));
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, s));
    if ((threadIdx.x & 31u) == 0) atomicMax(out, m);
}
__global__ void k_rows_bound_changed(uint32_t V, const int32_t* kold, const int32_t* knew, int* out, int* kmax_new) {
    int m = -1, km = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x) {
        if (kold[i] != knew[i]) m = max(m, max(kold[i], knew[i]));
        km = max(km, knew[i]);
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) {
        m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, s));
        km = max(km, __shfl_xor_sync(0xFFFFFFFFu, km, s));
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicMax(out, m);
        atomicMax(kmax_new, km);
    }
}
__global__ void k_vmax(uint32_t V, const int32_t* a, int* out) {
    int m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, a[i]);
#pragma unroll
    for (int s = 16; s; s >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, s));
    if ((threadIdx.x & 31u) == 0) atomicMax(out, m);
}

// ---------------------------------------------------------------------------
// decisions of a captured batch (BatchStatus, csrc/dc_device.cuh)
// ---------------------------------------------------------------------------
__global__ void k_gb_init(BatchStatus* st, unsigned long long cap, int* dbuf) {
    BatchStatus z = {};
    z.run_apply = 1;
    z.cap = cap;
    *st = z;
    dbuf[0] = -1;  // row bound (max), kmax after the batch (max), lmax (max)
    dbuf[1] = 0;
    dbuf[2] = 0;
}

// After the deletion check or the insertion capacity check: a failed check
// stops the batch before anything is applied.
__global__ void k_gb_gate(const EngineCtl* c, BatchStatus* st) {
    const unsigned e = c->error;
    if (e & DC_DEV_ERR_NOTFOUND) st->notfound = 1;
    if (e & DC_DEV_ERR_CAPACITY) st->need_rebuild = 1;
    if (e) st->run_apply = 0;
}

// After a persistent kernel: its errors stop the batch (reported by the host).
__global__ void k_gb_collect(const EngineCtl* c, BatchStatus* st, int count_region) {
    if (!st->run_apply) return;
    const unsigned e = c->error;
    if (e) {
        st->err |= e;
        st->err_where = c->err_where;
        st->run_apply = 0;
        return;
    }
    if (count_region) st->region += c->log_count;
}

// Expected work of a row repair (row_repair_worthwhile's measure): sum over
// the edges' endpoints of degree x kmax, before the batch.
__global__ void k_gb_work(uint32_t n, const uint32_t* u, const uint32_t* v, const int32_t* kmax,
                          const int32_t* in_len, const int32_t* out_len, BatchStatus* st) {
    unsigned long long w = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = u[i], b = v[i];
        w += (unsigned long long)(in_len[a] + out_len[a]) * (unsigned long long)max(kmax[a], 0);
        w += (unsigned long long)(in_len[b] + out_len[b]) * (unsigned long long)max(kmax[b], 0);
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) w += __shfl_xor_sync(0xFFFFFFFFu, w, s);
    if ((threadIdx.x & 31u) == 0) atomicAdd(&st->work, w);
}

// ---------------------------------------------------------------------------
// skyline merge: rows <= R from the fresh partial skyline, rows > R from the
// previous one
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sky_value_at(const uint32_t* off, const int32_t* ks, const int32_t* ls, uint32_t v,
                                            int k) {
    uint32_t a = off[v], b = off[v + 1];
    int val = 0;
    for (uint32_t i = a; i < b && ks[i] <= k; ++i) val = ls[i];
    return val;
}

__global__ void k_merge_count(uint32_t V, int R, const int32_t* kmax, const uint32_t* noff, const int32_t* nk,
                              const int32_t* nl, const uint32_t* ooff, const int32_t* ok, const int32_t* ol,
                              unsigned long long* cnt) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long c = 0;
        for (uint32_t i = noff[v]; i < noff[v + 1]; ++i) c += nk[i] <= R;
        if (R + 1 <= kmax[v]) {
            int last = sky_value_at(noff, nk, nl, (uint32_t)v, R);
            int at = sky_value_at(ooff, ok, ol, (uint32_t)v, R + 1);
            c += at != last;
            for (uint32_t i = ooff[v]; i < ooff[v + 1]; ++i) c += ok[i] > R + 1;
        }
        cnt[v] = c;
    }
}

__global__ void k_merge_fill(uint32_t V, int R, const int32_t* kmax, const uint32_t* noff, const int32_t* nk,
                             const int32_t* nl, const uint32_t* ooff, const int32_t* ok, const int32_t* ol,
                             const unsigned long long* moff, int32_t* mk, int32_t* ml, uint32_t* moff32) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t o = moff[v];
        for (uint32_t i = noff[v]; i < noff[v + 1]; ++i)
            if (nk[i] <= R) {
                mk[o] = nk[i];
                ml[o] = nl[i];
                ++o;
            }
        if (R + 1 <= kmax[v]) {
            int last = sky_value_at(noff, nk, nl, (uint32_t)v, R);
            int at = sky_value_at(ooff, ok, ol, (uint32_t)v, R + 1);
            if (at != last) {
                mk[o] = R + 1;
                ml[o] = at;
                ++o;
            }
            for (uint32_t i = ooff[v]; i < ooff[v + 1]; ++i)
                if (ok[i] > R + 1) {
                    mk[o] = ok[i];
                    ml[o] = ol[i];
                    ++o;
                }
        }
        moff32[v] = (uint32_t)moff[v];
        if (v == V - 1) moff32[V] = (uint32_t)moff[V];
    }
}

}  // namespace dc

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
namespace dc {

struct NetBatch {
    std::vector<uint32_t> del_u, del_v;  // distinct pairs with a net deletion
    std::vector<int32_t> del_n;          // occurrences to delete
    std::vector<uint32_t> ins_u, ins_v;  // net insertions, one entry per occurrence
    uint64_t n_del = 0, n_ins = 0;
};

// Net effect of a batch under sequential semantics: per distinct (u, v),
// occurrences inserted minus occurrences deleted.
static int net_batch(uint32_t V, const uint32_t* pairs, const uint8_t* is_del, uint64_t b, NetBatch& nb) {
    std::vector<uint64_t> key(b);
    for (uint64_t i = 0; i < b; ++i) {
        uint32_t u = pairs[2 * i], v = pairs[2 * i + 1];
        if (u >= V || v >= V)
            return set_error(DC_ERR_INVALID, "dc_maintain: edge %llu (%u, %u) has a vertex id >= V=%u",
                             (unsigned long long)i, u, v, V);
        key[i] = ((uint64_t)u << 32) | v;
    }
    std::vector<uint64_t> idx(b);
    for (uint64_t i = 0; i < b; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) { return key[x] < key[y] || (key[x] == key[y] && x < y); });
    for (uint64_t i = 0; i < b;) {
        uint64_t j = i;
        int64_t net = 0;
        while (j < b && key[idx[j]] == key[idx[i]]) {
            net += (is_del && is_del[idx[j]]) ? -1 : 1;
            ++j;
        }
        uint32_t u = (uint32_t)(key[idx[i]] >> 32), v = (uint32_t)key[idx[i]];
        if (net < 0) {
            nb.del_u.push_back(u);
            nb.del_v.push_back(v);
            nb.del_n.push_back((int32_t)-net);
            nb.n_del += (uint64_t)-net;
        } else {
            for (int64_t r = 0; r < net; ++r) {
                nb.ins_u.push_back(u);
                nb.ins_v.push_back(v);
            }
            nb.n_ins += (uint64_t)net;
        }
        i = j;
    }
    return DC_OK;
}

template <typename T>
static int upload(dc_graph* h, T** d, const std::vector<T>& hv) {
    if (mt_malloc(h->stream, d, hv.size())) return DC_ERR_NOMEM;
    if (!hv.empty()) MT_CUDA(cudaMemcpyAsync(*d, hv.data(), sizeof(T) * hv.size(), cudaMemcpyHostToDevice, h->stream));
    return DC_OK;
}

int sched_choose(dc_sched* s, const float* feat);

// Rule of thumb (the scheduler's fallback): the local update of kmax and
// row 0 grows with the batch (its bound on how far a value can rise is the
// number of inserted edges), the fused peel is a fixed pass over the graph.
static constexpr uint64_t kSchedLocalMax = 1ull << 16;
// Row mode 1 repairs rows in place for batches of at most this many net
// updates (the rule of thumb's local-method limit too).
static constexpr uint64_t kRuleRepairMax = 64;

int choose_method(dc_graph* h, uint64_t n_ins, uint64_t n_del) {
    (void)h;
    return (n_ins + n_del <= kRuleRepairMax) ? DC_MAINT_LOCAL : DC_MAINT_REPEEL;
}

// The 16 scheduler features of a net batch against the current graph and
// decomposition (before the batch is applied).
static int batch_features(dc_graph* h, const NetBatch& nb, float* f) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    std::vector<uint32_t> u(nb.del_u), v(nb.del_v);
    u.insert(u.end(), nb.ins_u.begin(), nb.ins_u.end());
    v.insert(v.end(), nb.ins_v.begin(), nb.ins_v.end());
    const uint64_t n = u.size();
    float acc[5] = {0, 0, 0, 0, 0};
    int iacc[2] = {0, 0};
    if (n) {
        uint32_t *du = nullptr, *dv = nullptr;
        if (upload(h, &du, u) || upload(h, &dv, v)) {
            mt_free(h->stream, du);
            mt_free(h->stream, dv);
            return DC_ERR_NOMEM;
        }
        float* dacc = (float*)h->scratch->tmp64;
        int* diacc = (int*)(dacc + 6);
        MT_CUDA(cudaMemsetAsync(dacc, 0, 32, h->stream));
        ++g_launches;
        k_batch_features<<<mgrid(h, n), kMThreads, 0, h->stream>>>((uint32_t)n, du, dv, d.kmax_v, d.row0, g.in_len,
                                                                   g.out_len, d.kmax, dacc, diacc);
        MT_CUDA(cudaMemcpyAsync(acc, dacc, 20, cudaMemcpyDeviceToHost, h->stream));
        MT_CUDA(cudaMemcpyAsync(iacc, diacc, 8, cudaMemcpyDeviceToHost, h->stream));
        MT_CUDA(cudaStreamSynchronize(h->stream));
        mt_free(h->stream, du);
        mt_free(h->stream, dv);
    }
    const double nn = n ? (double)n : 1.0, K1 = d.kmax + 1.0, L1 = d.lmax + 1.0;
    f[0] = (float)std::log2(1.0 + nb.n_ins);
    f[1] = (float)std::log2(1.0 + nb.n_del);
    f[2] = (float)std::log2(1.0 + g.V);
    f[3] = (float)std::log2(1.0 + g.E);
    f[4] = (float)std::log2(K1);
    f[5] = (float)std::log2(L1);
    f[6] = (float)(acc[0] / (2.0 * nn));
    f[7] = (float)std::log2(1.0 + iacc[0]);
    f[8] = (float)(acc[1] / nn / K1);
    f[9] = (float)(iacc[1] / K1);
    f[10] = (float)(acc[2] / nn);
    f[11] = (float)(acc[3] / (2.0 * nn) / L1);
    f[12] = (float)std::log2(1.0 + (double)d.n_corners / (g.V ? g.V : 1));
    f[13] = (float)((double)nb.n_ins / (double)std::max<uint64_t>(1, nb.n_ins + nb.n_del));
    f[14] = (float)std::log2(1.0 + n);
    // expected work of an in-place row repair against a recomputation
    // (the rule of thumb repairs below 1/160 of the graph's degree x kmax)
    f[15] = (float)std::log2(1.0 + 160.0 * acc[4] / (double)std::max<uint64_t>(1, h->full_work));
    return DC_OK;
}

// Groups (vertex, neighbour) deletions by vertex: one group per list.
static void group_by(const std::vector<uint32_t>& key, const std::vector<uint32_t>& other,
                     const std::vector<int32_t>& count, std::vector<uint32_t>& gvert, std::vector<uint32_t>& goff,
                     std::vector<uint32_t>& gnbr) {
    std::vector<uint64_t> idx(key.size());
    for (uint64_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return key[a] < key[b]; });
    gvert.clear();
    goff.clear();
    gnbr.clear();
    for (uint64_t i = 0; i < idx.size(); ++i) {
        if (i == 0 || key[idx[i]] != key[idx[i - 1]]) {
            gvert.push_back(key[idx[i]]);
            goff.push_back((uint32_t)gnbr.size());
        }
        for (int32_t r = 0; r < count[idx[i]]; ++r) gnbr.push_back(other[idx[i]]);
    }
    goff.push_back((uint32_t)gnbr.size());
}

// Applies the validated deletions to both adjacency sides.
static int apply_deletions(dc_graph* h, const NetBatch& nb) {
    DevGraph& g = h->g;
    if (nb.del_u.empty()) return DC_OK;
    int rc = DC_OK;
    uint32_t *du = nullptr, *dv = nullptr;
    int32_t* dn = nullptr;
    if ((rc = upload(h, &du, nb.del_u)) || (rc = upload(h, &dv, nb.del_v)) || (rc = upload(h, &dn, nb.del_n))) {
        mt_free(h->stream, du); mt_free(h->stream, dv); mt_free(h->stream, dn);
        return rc;
    }
    MT_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
    if (h->wait_ns)
        MT_CUDA(cudaMemcpyAsync(&h->ctl->wait_ns, &h->wait_ns, sizeof(h->wait_ns), cudaMemcpyHostToDevice, h->stream));
    ++g_launches;
    k_del_validate<<<mgrid(h, nb.del_u.size() * 32), kMThreads, 0, h->stream>>>(
        (uint32_t)nb.del_u.size(), du, dv, dn, g.out_off, g.out_len, g.out_nbr, h->ctl);
    EngineCtl hc;
    rc = check_ctl(h, &hc, "dc_maintain: deletion check");
    mt_free(h->stream, du);
    mt_free(h->stream, dv);
    mt_free(h->stream, dn);
    if (rc != DC_OK) {
        if (hc.error & DC_DEV_ERR_NOTFOUND)
            return set_error(DC_ERR_NOT_FOUND, "dc_maintain: a deleted edge is not in the graph (batch not applied)");
        return rc;
    }
    for (int side = 0; side < 2; ++side) {
        std::vector<uint32_t> gvert, goff, gnbr;
        if (side == 0) group_by(nb.del_u, nb.del_v, nb.del_n, gvert, goff, gnbr);
        else group_by(nb.del_v, nb.del_u, nb.del_n, gvert, goff, gnbr);
        uint32_t *d_gv = nullptr, *d_go = nullptr, *d_gn = nullptr;
        if ((rc = upload(h, &d_gv, gvert)) || (rc = upload(h, &d_go, goff)) || (rc = upload(h, &d_gn, gnbr))) {
            mt_free(h->stream, d_gv); mt_free(h->stream, d_go); mt_free(h->stream, d_gn);
            return rc;
        }
        ++g_launches;
        k_del_apply<<<mgrid(h, gvert.size() * 32), kMThreads, 0, h->stream>>>(
            (uint32_t)gvert.size(), d_gv, d_go, d_gn, side == 0 ? g.out_off : g.in_off,
            side == 0 ? g.out_len : g.in_len, side == 0 ? g.out_nbr : g.in_nbr, h->ctl, nullptr);
        cudaError_t e = cudaStreamSynchronize(h->stream);
        mt_free(h->stream, d_gv);
        mt_free(h->stream, d_go);
        mt_free(h->stream, d_gn);
        if (e != cudaSuccess) return set_error(DC_ERR_CUDA, "deletion apply: %s", cudaGetErrorString(e));
    }
    rc = check_ctl(h, &hc, "dc_maintain: deletion apply");
    if (rc != DC_OK) return rc;
    g.E -= nb.n_del;
    g.sorted_kmax = false;
    return DC_OK;
}

// Rebuilds the adjacency store with more free slots (keeps the decomposition).
static int rebuild_store(dc_graph* h, const uint32_t* d_iu, const uint32_t* d_iv, uint64_t n_ins) {
    DevGraph& g = h->g;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    uint64_t E = g.E + n_ins;
    uint32_t *src = nullptr, *dst = nullptr;
    if (mt_malloc(h->stream, &src, E) || mt_malloc(h->stream, &dst, E)) {
        mt_free(h->stream, src);
        return DC_ERR_NOMEM;
    }
    ++g_launches;
    k_len_to_u64<<<mgrid(h, V), kMThreads, 0, h->stream>>>(V, g.out_len, (unsigned long long*)s->tmp64);
    if (int rc = scan_tmp64(h, V)) {
        mt_free(h->stream, src); mt_free(h->stream, dst);
        return rc;
    }
    ++g_launches;
    k_store_edges<<<mgrid(h, (uint64_t)V * 32), kMThreads, 0, h->stream>>>(
        V, g.out_off, g.out_len, (const unsigned long long*)s->tmp64, g.out_nbr, src, dst);
    MT_CUDA(cudaMemcpyAsync(src + g.E, d_iu, 4 * n_ins, cudaMemcpyDeviceToDevice, h->stream));
    MT_CUDA(cudaMemcpyAsync(dst + g.E, d_iv, 4 * n_ins, cudaMemcpyDeviceToDevice, h->stream));
    MT_CUDA(cudaStreamSynchronize(h->stream));
    Decomp keep = h->d;
    h->d = Decomp();
    uint32_t gm = h->gap_min, gd = h->gap_div;
    h->gap_min = std::max<uint32_t>(gm, 2);
    h->gap_div = gd ? std::min<uint32_t>(gd, 8) : 8;
    int rc = build_from_device_edges(h, V, E, src, dst);
    cudaStreamSynchronize(h->stream);
    free_decomp(h->d, h->stream);
    h->d = keep;
    mt_free(h->stream, src);
    mt_free(h->stream, dst);
    return rc;
}

// Inserts the net insertions; returns 1 in *rebuilt when the store grew.
static int apply_insertions(dc_graph* h, const NetBatch& nb, uint32_t** d_iu_out, uint32_t** d_iv_out, int* rebuilt) {
    DevGraph& g = h->g;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    *rebuilt = 0;
    *d_iu_out = *d_iv_out = nullptr;
    if (nb.ins_u.empty()) return DC_OK;
    uint32_t *iu = nullptr, *iv = nullptr;
    int rc = DC_OK;
    if ((rc = upload(h, &iu, nb.ins_u)) || (rc = upload(h, &iv, nb.ins_v))) {
        mt_free(h->stream, iu); mt_free(h->stream, iv);
        return rc;
    }
    const uint32_t n = (uint32_t)nb.ins_u.size();
    MT_CUDA(cudaMemsetAsync(s->key2, 0, 4ull * V, h->stream));
    MT_CUDA(cudaMemsetAsync(s->cdeg2, 0, 4ull * V, h->stream));
    MT_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
    if (h->wait_ns)
        MT_CUDA(cudaMemcpyAsync(&h->ctl->wait_ns, &h->wait_ns, sizeof(h->wait_ns), cudaMemcpyHostToDevice, h->stream));
    ++g_launches;
    k_ins_need<<<mgrid(h, n), kMThreads, 0, h->stream>>>(n, iu, iv, s->key2, s->cdeg2);
    ++g_launches;
    k_ins_fits<<<mgrid(h, V), kMThreads, 0, h->stream>>>(V, g.out_off, g.out_len, s->key2, g.in_off, g.in_len,
                                                         s->cdeg2, h->ctl);
    EngineCtl hc;
    rc = check_ctl(h, &hc, "dc_maintain: capacity check");
    if (rc != DC_OK && (hc.error & DC_DEV_ERR_CAPACITY)) {
        set_error(DC_OK, "%s", "");
        rc = rebuild_store(h, iu, iv, n);
        *rebuilt = 1;
    } else if (rc == DC_OK) {
        ++g_launches;
        k_ins_apply<<<mgrid(h, n), kMThreads, 0, h->stream>>>(n, iu, iv, g.out_off, g.out_len, g.out_nbr, g.in_off,
                                                              g.in_len, g.in_nbr, nullptr);
        g.E += n;
    }
    if (rc != DC_OK) {
        mt_free(h->stream, iu); mt_free(h->stream, iv);
        return rc;
    }
    g.sorted_kmax = false;
    *d_iu_out = iu;
    *d_iv_out = iv;
    return DC_OK;
}

// Parameters of one local core update.  which: 0 = kmax (count list =
// in-list), 1 = row 0 (count list = out-list).  insert_mode: roots + bound b.
static int core_params(dc_graph* h, int which, int32_t* val, const int32_t* old, const uint32_t* d_seeds,
                       uint32_t n_seeds, int insert_mode, int32_t b, CoreParams* out) {
    DevGraph& g = h->g;
    Scratch* s = h->scratch;
    CoreParams& p = *out;
    p.V = g.V;
    if (which == 0) {
        p.c_off = g.in_off; p.c_len = g.in_len; p.c_nbr = g.in_nbr;
        p.d_off = g.out_off; p.d_len = g.out_len; p.d_nbr = g.out_nbr;
    } else {
        p.c_off = g.out_off; p.c_len = g.out_len; p.c_nbr = g.out_nbr;
        p.d_off = g.in_off; p.d_len = g.in_len; p.d_nbr = g.in_nbr;
    }
    p.val = val;
    p.old = old;
    p.mark = s->mark;
    p.stamp = s->stamp;
    p.stamp_id = 1;
    p.cand = s->rem0;
    p.cand_cap = g.V + 1;
    p.seeds = d_seeds;
    p.n_seeds = n_seeds;
    p.insert_mode = insert_mode;
    p.b = b;
    p.run = nullptr;
    if (int rc = ensure_tring(h, 2ull * g.V + (uint64_t)h->geom.sms * 64 + 4096)) return rc;
    p.q.slots = s->tring;
    p.q.mask = (unsigned)(s->tring_cap - 1);
    p.ctl = h->ctl;
    return DC_OK;
}

// One local core update, waited for.
static int core_local(dc_graph* h, int which, int32_t* val, const int32_t* old, const uint32_t* d_seeds,
                      uint32_t n_seeds, int insert_mode, int32_t b, uint64_t* region) {
    if (n_seeds == 0) return DC_OK;
    CoreParams p;
    if (int rc = core_params(h, which, val, old, d_seeds, n_seeds, insert_mode, b, &p)) return rc;
    if (insert_mode) MT_CUDA(cudaMemsetAsync(h->scratch->stamp, 0xFF, 4ull * h->g.V, h->stream));
    void* args[] = {&p};
    EngineCtl hc;
    if (int rc = run_persistent(h, (const void*)k_core_local, args, "core update", &hc)) return rc;
    if (region) *region += insert_mode ? hc.log_count : n_seeds;
    return DC_OK;
}

// Appends one record of the maintenance log (scheduler training data).
static void log_batch(dc_graph* h, const float* feat, const dc_maint_stats* st) {
    MaintLogRec r;
    memcpy(r.feat, feat, sizeof(r.feat));
    r.method = st->method;
    r.total_ms = st->total_ms;
    r.core_ms = st->core_ms;
    r.rows_ms = st->rows_ms;
    h->maint_log.push_back(r);
}

// Time limit of an in-place row repair of rows 1..R: what recomputing them
// is expected to cost (the rows phase of the last full decomposition, scaled
// by R / kmax, plus the recomputation's fixed passes over C_1), so that a
// repair that turns out larger than expected gives up in time.  Row mode 2
// (repair whenever the batch fits) sets no limit.
static unsigned long long repair_deadline_ns(const dc_graph* h, int32_t R, int rmode) {
    if (rmode == 2) return 0;
    const double K = std::max<int32_t>(1, h->d.kmax);
    const double ms = 2.0 + h->full_rows_ms * std::min(1.0, (double)R / K) + 0.1 * h->full_rows_ms;
    return (unsigned long long)(ms * 1e6);
}

// Rows 1..R recomputed from the new row 0 (kmax and row 0 already updated)
// and merged with the old skyline above R; then the decomposition is current
// with kmax Knew and lmax.  On failure the decomposition is marked invalid.
static int recompute_rows(dc_graph* h, int32_t R, int32_t Knew, int32_t lmax) {
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = h->g.V;
    MT_CUDA(cudaMemcpyAsync(s->row0, d.row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
    uint64_t nlog = 0;
    int rc = rows_from_row0(h, Knew, R, R > 48, &nlog, 1, false);
    if (rc != DC_OK) return rc;
    // the old skyline stays readable while rows 0..R are assembled in
    // spare slot 0 and merged into spare slot 1; then the merged one is
    // current and the other two go back to the slots (no allocation
    // once the slots have grown to the graph's size)
    uint32_t* o_off = d.sky_off;
    int32_t* o_k = d.sky_k;
    int32_t* o_l = d.sky_l;
    const uint64_t o_cap = d.corner_cap;
    if ((rc = sky_take_spare(h, 0, 0, &d.sky_off, &d.sky_k, &d.sky_l, &d.corner_cap)) == DC_OK)
        rc = build_skyline_from_log(h, nlog);
    if (rc == DC_OK) {
        unsigned long long* cnt = (unsigned long long*)s->tmp64;
        ++g_launches;
        k_merge_count<<<mgrid(h, V), kMThreads, 0, h->stream>>>(V, R, d.kmax_v, d.sky_off, d.sky_k, d.sky_l, o_off,
                                                                o_k, o_l, cnt);
        rc = scan_tmp64(h, V);
        unsigned long long total = 0;
        if (rc == DC_OK) {
            cudaMemcpyAsync(&total, s->tmp64 + V, sizeof(total), cudaMemcpyDeviceToHost, h->stream);
            cudaStreamSynchronize(h->stream);
        }
        uint32_t* m_off = nullptr;
        int32_t *m_k = nullptr, *m_l = nullptr;
        uint64_t m_cap = 0;
        if (rc == DC_OK) rc = sky_take_spare(h, 1, total, &m_off, &m_k, &m_l, &m_cap);
        if (rc == DC_OK) {
            ++g_launches;
            k_merge_fill<<<mgrid(h, V), kMThreads, 0, h->stream>>>(V, R, d.kmax_v, d.sky_off, d.sky_k, d.sky_l,
                                                                   o_off, o_k, o_l, cnt, m_k, m_l, m_off);
            cudaStreamSynchronize(h->stream);
            sky_put_spare(h, 0, d.sky_off, d.sky_k, d.sky_l, d.corner_cap);
            d.sky_off = m_off;
            d.sky_k = m_k;
            d.sky_l = m_l;
            d.corner_cap = m_cap;
            d.n_corners = total;
        }
    }
    sky_put_spare(h, 1, o_off, o_k, o_l, o_cap);
    if (rc != DC_OK) {
        d.valid = false;
        return rc;
    }
    d.kmax = Knew;
    d.lmax = lmax;
    d.rows_valid = false;
    d.valid = true;
    return DC_OK;
}

// ---------------------------------------------------------------------------
// a maintenance batch as one captured CUDA graph
// ---------------------------------------------------------------------------
// A batch of one kind of update (deletions or insertions) on the local
// method with rows repaired in place is enqueued once on the handle's
// stream under stream capture and run as ONE graph launch: the batch
// arrays' upload, the deletion check or the insertion capacity check, the
// list updates, the kmax and row-0 updates, the row bound, the repair of
// rows 1..R, the skyline merge and the read-back of the batch's status.
// Every branch the host-driven batch takes between kernels is taken on the
// device (BatchStatus): kernels behind a branch act only while its run flag
// is set.  What the graph cannot finish -- a list without free slots (the
// store is rebuilt), a repair that is not expected to pay or gives up, a
// merged skyline larger than its buffer -- the host finishes after the
// launch from the state the graph left (the graph never half-applies a
// batch: nothing is written before both checks pass).  The graph is
// re-captured per batch (its grids and buffers change) and applied to the
// handle's executable graph by cudaGraphExecUpdate, so it is instantiated
// once per kind.  Its timing events are event-record nodes (recorded with
// cudaEventRecordExternal; a plain record inside a capture only orders
// streams).
static constexpr uint32_t kCapturedMax = 1536;

void free_captured_batches(dc_graph* h) {
    for (auto& e : h->cb_exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
    if (h->cb_host) cudaFreeHost(h->cb_host);
    if (h->cb_dev) cudaFreeAsync(h->cb_dev, h->stream);
    h->cb_host = nullptr;
    h->cb_dev = nullptr;
    h->cb_status = nullptr;
    h->cb_words = 0;
}

// Staging for `words` words of batch arrays plus the status block.
static int captured_buffers(dc_graph* h, uint64_t words) {
    if (words <= h->cb_words && h->cb_host) return DC_OK;
    const uint64_t want = (std::max<uint64_t>(4096, 2 * words) + 63) & ~63ull;
    const uint64_t status_words = (sizeof(BatchStatus) + 255) / 4;
    if (h->cb_host) cudaFreeHost(h->cb_host);
    if (h->cb_dev) cudaFreeAsync(h->cb_dev, h->stream);
    h->cb_host = nullptr;
    h->cb_dev = nullptr;
    h->cb_words = 0;
    if (cudaHostAlloc((void**)&h->cb_host, 4 * (want + status_words), cudaHostAllocDefault) != cudaSuccess ||
        cudaMallocAsync((void**)&h->cb_dev, 4 * (want + status_words), h->stream) != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "captured batch: staging allocation failed");
    }
    h->cb_status = reinterpret_cast<BatchStatus*>(h->cb_dev + want);
    h->cb_words = want;
    return DC_OK;
}

// Enqueues the whole batch (no host waits).  Arrays: u/v of the batch's
// edges (deletions: distinct pairs with their counts in cnt; insertions:
// one entry per occurrence), deletions grouped per list side in g*.
struct CapturedArgs {
    bool ins;
    uint32_t n;
    const uint32_t *u, *v, *cnt;
    uint32_t ng[2];
    const uint32_t *gv[2], *go[2], *gn[2];
    int rmode;
    uint64_t log_cap;
    uint64_t cap1;  // corners the merged skyline's buffer holds
    uint32_t *coff, *noff;
    int32_t *ck, *cl, *nk, *nl;
    CoreParams cp[2];
};

static int captured_enqueue(dc_graph* h, CapturedArgs& a, uint64_t words) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    cudaStream_t st = h->stream;
    BatchStatus* bs = h->cb_status;
    int* dbuf = (int*)s->cursor;
    cudaEvent_t* ev = h->ev;
    MT_CUDA(cudaEventRecordWithFlags(ev[0], st, cudaEventRecordExternal));
    MT_CUDA(cudaMemcpyAsync(h->cb_dev, h->cb_host, 4 * words, cudaMemcpyHostToDevice, st));
    ++g_launches;
    k_gb_init<<<1, 1, 0, st>>>(bs, a.cap1, dbuf);
    MT_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), st));
    // ---- checks before anything is written
    if (!a.ins) {
        ++g_launches;
        k_del_validate<<<mgrid(h, (uint64_t)a.n * 32), kMThreads, 0, st>>>(a.n, a.u, a.v, (const int32_t*)a.cnt,
                                                                          g.out_off, g.out_len, g.out_nbr, h->ctl);
    } else {
        MT_CUDA(cudaMemsetAsync(s->key2, 0, 4ull * V, st));
        MT_CUDA(cudaMemsetAsync(s->cdeg2, 0, 4ull * V, st));
        g_launches += 2;
        k_ins_need<<<mgrid(h, a.n), kMThreads, 0, st>>>(a.n, a.u, a.v, s->key2, s->cdeg2);
        k_ins_fits<<<mgrid(h, V), kMThreads, 0, st>>>(V, g.out_off, g.out_len, s->key2, g.in_off, g.in_len, s->cdeg2,
                                                      h->ctl);
    }
    ++g_launches;
    k_gb_gate<<<1, 1, 0, st>>>(h->ctl, bs);
    if (a.rmode == 1) {
        ++g_launches;
        k_gb_work<<<mgrid(h, a.n), kMThreads, 0, st>>>(a.n, a.u, a.v, d.kmax_v, g.in_len, g.out_len, bs);
    }
    MT_CUDA(cudaMemcpyAsync(s->kmax_old, d.kmax_v, 4ull * V, cudaMemcpyDeviceToDevice, st));
    // ---- list updates
    if (!a.ins) {
        for (int side = 0; side < 2; ++side) {
            if (!a.ng[side]) continue;
            ++g_launches;
            k_del_apply<<<mgrid(h, (uint64_t)a.ng[side] * 32), kMThreads, 0, st>>>(
                a.ng[side], a.gv[side], a.go[side], a.gn[side], side == 0 ? g.out_off : g.in_off,
                side == 0 ? g.out_len : g.in_len, side == 0 ? g.out_nbr : g.in_nbr, h->ctl, &bs->run_apply);
        }
    } else {
        ++g_launches;
        k_ins_apply<<<mgrid(h, a.n), kMThreads, 0, st>>>(a.n, a.u, a.v, g.out_off, g.out_len, g.out_nbr, g.in_off,
                                                         g.in_len, g.in_nbr, &bs->run_apply);
    }
    // ---- kmax and row 0, locally
    if (!a.ins) {
        MT_CUDA(cudaMemcpyAsync(s->row0_old, d.row0, 4ull * V, cudaMemcpyDeviceToDevice, st));
    } else {
        MT_CUDA(cudaMemcpyAsync(s->cdeg2, d.kmax_v, 4ull * V, cudaMemcpyDeviceToDevice, st));
        MT_CUDA(cudaMemcpyAsync(s->key2, d.row0, 4ull * V, cudaMemcpyDeviceToDevice, st));
    }
    for (int which = 0; which < 2; ++which) {
        if (a.ins) MT_CUDA(cudaMemsetAsync(s->stamp, 0xFF, 4ull * V, st));
        void* args[] = {&a.cp[which]};
        if (int rc = persistent_enqueue(h, (const void*)k_core_local, args, "core update", h->ctl, st)) return rc;
        ++g_launches;
        k_gb_collect<<<1, 1, 0, st>>>(h->ctl, bs, a.ins ? 1 : 0);
    }
    MT_CUDA(cudaEventRecordWithFlags(ev[1], st, cudaEventRecordExternal));
    MT_CUDA(cudaEventRecordWithFlags(ev[2], st, cudaEventRecordExternal));
    // ---- the rows a batch can change, and what to do with them
    g_launches += 3;
    k_rows_bound_edges<<<mgrid(h, a.n), kMThreads, 0, st>>>(a.n, a.u, a.v, s->kmax_old, d.kmax_v, dbuf);
    k_rows_bound_changed<<<mgrid(h, V), kMThreads, 0, st>>>(V, s->kmax_old, d.kmax_v, dbuf, dbuf + 1);
    k_vmax<<<mgrid(h, V), kMThreads, 0, st>>>(V, d.row0, dbuf + 2);
    if (int rc = decide_enqueue(h, bs, dbuf, a.rmode, a.n, a.ins)) return rc;
    MT_CUDA(cudaEventRecordWithFlags(ev[4], st, cudaEventRecordExternal));
    if (int rc = repair_enqueue(h, a.ins, a.u, a.v, a.n, a.log_cap, bs)) return rc;
    MT_CUDA(cudaEventRecordWithFlags(ev[5], st, cudaEventRecordExternal));
    if (int rc = merge_enqueue(h, bs, a.coff, a.ck, a.cl, a.noff, a.nk, a.nl)) return rc;
    MT_CUDA(cudaEventRecordWithFlags(ev[3], st, cudaEventRecordExternal));
    MT_CUDA(cudaMemcpyAsync(h->cb_host + h->cb_words, bs, sizeof(BatchStatus), cudaMemcpyDeviceToHost, st));
    return DC_OK;
}

// Runs a one-kind batch as one captured graph.  *handled = false (and
// nothing changed) when the batch needs the host path: a list without free
// slots, or a graph the driver does not accept (the handle then stops
// capturing).
static int maintain_captured(dc_graph* h, const NetBatch& nb, int rmode, dc_maint_stats* st, bool* handled) {
    *handled = false;
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    CapturedArgs a;
    memset(&a, 0, sizeof(a));
    a.ins = nb.del_u.empty();
    a.rmode = rmode;
    // ---- batch arrays packed into one upload
    std::vector<uint32_t> w;
    size_t o_u = 0, o_v = 0, o_c = 0, o_g[2][3] = {};
    if (a.ins) {
        a.n = (uint32_t)nb.ins_u.size();
        w.insert(w.end(), nb.ins_u.begin(), nb.ins_u.end());
        o_v = w.size();
        w.insert(w.end(), nb.ins_v.begin(), nb.ins_v.end());
    } else {
        a.n = (uint32_t)nb.del_u.size();
        w.insert(w.end(), nb.del_u.begin(), nb.del_u.end());
        o_v = w.size();
        w.insert(w.end(), nb.del_v.begin(), nb.del_v.end());
        o_c = w.size();
        for (int32_t c : nb.del_n) w.push_back((uint32_t)c);
        for (int side = 0; side < 2; ++side) {
            std::vector<uint32_t> gv, go, gn;
            if (side == 0) group_by(nb.del_u, nb.del_v, nb.del_n, gv, go, gn);
            else group_by(nb.del_v, nb.del_u, nb.del_n, gv, go, gn);
            a.ng[side] = (uint32_t)gv.size();
            o_g[side][0] = w.size();
            w.insert(w.end(), gv.begin(), gv.end());
            o_g[side][1] = w.size();
            w.insert(w.end(), go.begin(), go.end());
            o_g[side][2] = w.size();
            w.insert(w.end(), gn.begin(), gn.end());
        }
    }
    if (int rc = captured_buffers(h, w.size())) return rc;
    memcpy(h->cb_host, w.data(), 4 * w.size());
    a.u = h->cb_dev + o_u;
    a.v = h->cb_dev + o_v;
    a.cnt = h->cb_dev + o_c;
    for (int side = 0; side < 2; ++side) {
        a.gv[side] = h->cb_dev + o_g[side][0];
        a.go[side] = h->cb_dev + o_g[side][1];
        a.gn[side] = h->cb_dev + o_g[side][2];
    }
    // ---- everything the graph uses, allocated before the capture
    if (!s->kmax_old && (mt_malloc(h->stream, &s->kmax_old, (uint64_t)V + 1) ||
                         mt_malloc(h->stream, &s->row0_old, (uint64_t)V + 1)))
        return DC_ERR_NOMEM;
    uint64_t log_cap = 0;
    if (int rc = ensure_change_log(h, &log_cap)) return rc;
    a.log_cap = std::min<uint64_t>(log_cap, 1ull << 22);
    if (int rc = repair_prepare(h)) return rc;
    const int32_t bb = (int32_t)std::min<uint64_t>(nb.n_ins, 0x3FFFFFFF);
    if (!a.ins) {
        if (int rc = core_params(h, 0, d.kmax_v, s->kmax_old, a.v, a.n, 0, 0, &a.cp[0])) return rc;
        if (int rc = core_params(h, 1, d.row0, s->row0_old, a.u, a.n, 0, 0, &a.cp[1])) return rc;
    } else {
        if (int rc = core_params(h, 0, d.kmax_v, s->cdeg2, a.v, a.n, 1, bb, &a.cp[0])) return rc;
        if (int rc = core_params(h, 1, d.row0, s->key2, a.u, a.n, 1, bb, &a.cp[1])) return rc;
    }
    a.cp[0].run = a.cp[1].run = &h->cb_status->run_apply;
    uint64_t cap0 = 0;
    if (int rc = sky_take_spare(h, 0, a.log_cap, &a.coff, &a.ck, &a.cl, &cap0)) return rc;
    int rc = sky_take_spare(h, 1, d.n_corners + d.n_corners / 8 + V / 4 + 4096, &a.noff, &a.nk, &a.nl, &a.cap1);
    if (rc != DC_OK) {
        sky_put_spare(h, 0, a.coff, a.ck, a.cl, cap0);
        return rc;
    }
    auto put_back = [&](bool slot1) {
        sky_put_spare(h, 0, a.coff, a.ck, a.cl, cap0);
        if (slot1) sky_put_spare(h, 1, a.noff, a.nk, a.nl, a.cap1);
    };
    MT_CUDA(cudaStreamSynchronize(h->stream));  // allocations done before the capture
    // ---- capture, update the executable graph, launch
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGetLastError();
        put_back(true);
        h->captured_batches = false;
        return DC_OK;
    }
    const unsigned long long launches0 = g_launches.load();
    rc = captured_enqueue(h, a, w.size());
    cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
    cudaGraphExec_t& ex = h->cb_exec[a.ins ? 1 : 0];
    if (rc == DC_OK && ec == cudaSuccess && ex) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(ex, graph, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(ex);
            ex = nullptr;
        }
    }
    if (rc == DC_OK && ec == cudaSuccess && !ex && cudaGraphInstantiate(&ex, graph, 0) != cudaSuccess) ec = cudaErrorUnknown;
    if (graph) cudaGraphDestroy(graph);
    if (rc != DC_OK || ec != cudaSuccess) {
        // the graph was not built: nothing ran; the host path takes the batch
        // and the handle's later batches (reported once per handle)
        fprintf(stderr, "dcore_b200: maintenance batches run host-driven on this graph: capture failed (%s; %s)\n",
                rc != DC_OK ? dc_last_error() : "", cudaGetErrorString(ec));
        cudaGetLastError();
        g_launches = launches0;
        put_back(true);
        h->captured_batches = false;
        set_error(DC_OK, "%s", "");
        return DC_OK;
    }
    MT_CUDA(cudaGraphLaunch(ex, h->stream));
    MT_CUDA(cudaStreamSynchronize(h->stream));
    const BatchStatus r = *reinterpret_cast<const BatchStatus*>(h->cb_host + h->cb_words);
    // ---- what the graph decided
    if (r.notfound) {
        put_back(true);
        return set_error(DC_ERR_NOT_FOUND, "dc_maintain: a deleted edge is not in the graph (batch not applied)");
    }
    if (r.need_rebuild) {  // nothing applied: the host path rebuilds the store
        put_back(true);
        return DC_OK;
    }
    *handled = true;
    if (r.err) {
        put_back(true);
        d.valid = false;
        d.peel_valid = false;
        if (r.err & DC_DEV_ERR_TIMEOUT)
            return set_error(DC_ERR_TIMEOUT, "captured batch: bounded device wait expired (site %u)", r.err_where);
        return set_error(DC_ERR_CUDA, "captured batch: device error 0x%x (site %u)", r.err, r.err_where);
    }
    if (a.ins) g.E += nb.n_ins;
    else g.E -= nb.n_del;
    g.sorted_kmax = false;
    st->method = DC_MAINT_LOCAL;
    st->region = r.region + (a.ins ? 0 : 2ull * a.n);
    st->rows_recomputed = r.R + 1;
    st->ins_scanned = a.ins ? r.scanned : 0;
    st->captured = 1;
    cudaEvent_t* ev = h->ev;
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    st->apply_ms = ms;
    cudaEventElapsedTime(&ms, ev[1], ev[2]);
    st->core_ms = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    st->rows_ms = ms;
    cudaEventElapsedTime(&ms, ev[0], ev[3]);
    st->total_ms = ms;
    if (r.R > 0) {
        cudaEventElapsedTime(&ms, ev[4], ev[5]);
        if (a.ins) st->ins_repair_ms = ms;
        else st->del_repair_ms = ms;
    }
    cudaGetLastError();  // a timing query that failed leaves no error behind
    if (r.R >= 0 && r.run_merge) {
        // the merged skyline is current; the old one becomes a spare
        sky_put_spare(h, 0, a.coff, a.ck, a.cl, cap0);
        sky_put_spare(h, 1, d.sky_off, d.sky_k, d.sky_l, d.corner_cap);
        d.sky_off = a.noff;
        d.sky_k = a.nk;
        d.sky_l = a.nl;
        d.corner_cap = a.cap1;
        d.n_corners = r.total;
        if (r.R > 0) st->rows_local = a.ins ? 2 : 1;
    } else {
        put_back(true);
        if (r.R >= 0 && (r.merge_overflow || r.fallback)) {
            // the host finishes the rows (timed apart, added to the batch)
            cudaEventRecord(ev[6], h->stream);
            bool applied = false;
            if (r.merge_overflow) {
                if ((rc = apply_change_log(h, r.nlog, &applied)) != DC_OK) {
                    d.valid = false;
                    return rc;
                }
                if (applied && r.R > 0) st->rows_local = a.ins ? 2 : 1;
            }
            if (!applied && (rc = recompute_rows(h, r.R, r.Knew, r.lmax)) != DC_OK) return rc;
            cudaEventRecord(ev[7], h->stream);
            MT_CUDA(cudaStreamSynchronize(h->stream));
            cudaEventElapsedTime(&ms, ev[6], ev[7]);
            st->rows_ms += ms;
            st->total_ms += ms;
        }
    }
    d.kmax = r.Knew;
    d.lmax = r.lmax;
    d.rows_valid = false;
    d.valid = true;
    d.row_lo = 1;
    d.row_hi = d.kmax;
    st->kmax = d.kmax;
    st->lmax = d.lmax;
    return DC_OK;
}

// repair_mode: the row maintenance mode of this batch (-1: the handle's);
// nested: a part of a split batch (no features, no log record).
static int maintain_impl(dc_graph* h, const uint32_t* pairs, const uint8_t* is_del, uint64_t b, int method,
                         int repair_mode, bool nested, dc_maint_stats* st) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    const uint32_t V = g.V;
    dc_maint_stats local_st;
    if (!st) st = &local_st;
    memset(st, 0, sizeof(*st));
    if (b && !pairs) return set_error(DC_ERR_INVALID, "dc_maintain: null edge array");
    if (method < DC_MAINT_AUTO || method > DC_MAINT_REPEEL) return set_error(DC_ERR_INVALID, "dc_maintain: bad method %d", method);
    if (int rc = ensure_scratch(h, V)) return rc;
    Scratch* s = h->scratch;
    if (!d.full())
        if (int rc = decompose(h, 0, 0)) return rc;
    NetBatch nb;
    if (int rc = net_batch(V, pairs, is_del, b, nb)) return rc;
    // features of the batch against the decomposition before it
    float feat[16];
    const bool want_feat = !nested && (h->log_maint || (method == DC_MAINT_AUTO && h->sched));
    if (want_feat)
        if (int rc = batch_features(h, nb, feat)) return rc;
    int rmode = repair_mode >= 0 ? repair_mode : h->row_repair;
    bool by_rule = false;  // method picked by the rule of thumb (halves of a split batch pick their own)
    if (method == DC_MAINT_AUTO) {
        // the network picks the incremental path (local kmax / row-0 update,
        // rows repaired in place wherever the batch fits, within the time
        // limit: row mode 3) or the full one
        // (fused re-peel, rows recomputed) where both are practical; past
        // kSchedLocalMax net updates the local update's region covers most
        // of the graph and the full path is taken without asking.  Without
        // a network the rule of thumb picks the method and the handle's mode
        // the rows.
        int m = !nested && h->sched && nb.n_ins + nb.n_del <= kSchedLocalMax ? sched_choose(h->sched, feat) : -1;
        if (m == DC_MAINT_LOCAL) {
            method = DC_MAINT_LOCAL;
            rmode = 3;
        } else if (m == DC_MAINT_REPEEL) {
            method = DC_MAINT_REPEEL;
            rmode = 0;
        } else {
            method = choose_method(h, nb.n_ins, nb.n_del);
            by_rule = true;
        }
    }
    // the rule's row mode repairs small batches only: past kRuleRepairMax net
    // updates the expected-work estimate misses the cascades that deletions
    // near the dense core start, and a recomputation is the safer bet
    if (rmode == 1 && nb.n_ins + nb.n_del > kRuleRepairMax) rmode = 0;
    // ---- one kind of update, local method, rows in place: one graph launch
    const uint64_t n_one = nb.del_u.empty() ? nb.ins_u.size() : nb.del_u.size();
    if (h->captured_batches && method == DC_MAINT_LOCAL && rmode != 0 && nb.del_u.empty() != nb.ins_u.empty() &&
        n_one <= kCapturedMax && !h->trace_dev && h->barrier_fault_block < 0 && d.kmax_v && d.sky_off) {
        bool handled = false;
        st->deleted = nb.n_del;
        st->inserted = nb.n_ins;
        int rc = maintain_captured(h, nb, rmode, st, &handled);
        if (rc != DC_OK) {
            if (handled) {
                d.valid = false;
                d.peel_valid = false;
            }
            return rc;
        }
        if (handled) {
            h->mtimes.total_ms = st->total_ms;
            if (h->log_maint && want_feat) log_batch(h, feat, st);
            return DC_OK;
        }
        memset(st, 0, sizeof(*st));
    }
    bool repair_del = false;  // rows of the deletions repaired in place
    if (rmode && !nb.del_u.empty() && nb.del_u.size() <= row_repair_max_deletions() && d.kmax_v) {
        uint32_t *eu = nullptr, *ev = nullptr;
        if (upload(h, &eu, nb.del_u) == DC_OK && upload(h, &ev, nb.del_v) == DC_OK)
            repair_del = rmode >= 2 || row_repair_worthwhile(h, eu, ev, (uint32_t)nb.del_u.size());
        mt_free(h->stream, eu);
        mt_free(h->stream, ev);
    }
    bool repair_ins = false;  // rows of the insertions repaired in place
    if (rmode && !nb.ins_u.empty() && nb.ins_u.size() <= row_repair_max_insertions() && d.kmax_v) {
        uint32_t *eu = nullptr, *ev = nullptr;
        if (upload(h, &eu, nb.ins_u) == DC_OK && upload(h, &ev, nb.ins_v) == DC_OK)
            repair_ins = rmode >= 2 || row_repair_worthwhile(h, eu, ev, (uint32_t)nb.ins_u.size());
        mt_free(h->stream, eu);
        mt_free(h->stream, ev);
    }
    if (repair_del && !nb.ins_u.empty()) {
        // deletions first (their rows repaired in place), then the
        // insertions with their own row maintenance: the net effect per edge
        // makes the two commute.  (Insertions repaired in place after
        // deletions that recompute rows 1..R would only add to that
        // recomputation, so they split the batch only with the deletions.)
        std::vector<uint32_t> pd(2 * nb.del_u.size()), pi(2 * nb.ins_u.size());
        for (size_t i = 0; i < nb.del_u.size(); ++i) {
            pd[2 * i] = nb.del_u[i];
            pd[2 * i + 1] = nb.del_v[i];
        }
        for (size_t i = 0; i < nb.ins_u.size(); ++i) {
            pi[2 * i] = nb.ins_u[i];
            pi[2 * i + 1] = nb.ins_v[i];
        }
        std::vector<uint8_t> ones(nb.del_u.size(), 1);
        dc_maint_stats a, c;
        const int half = by_rule ? DC_MAINT_AUTO : method;
        if (int rc = maintain_impl(h, pd.data(), ones.data(), nb.del_u.size(), half, rmode, true, &a)) return rc;
        if (int rc = maintain_impl(h, pi.data(), nullptr, nb.ins_u.size(), half, rmode, true, &c)) return rc;
        *st = c;
        st->deleted = a.deleted;
        st->rows_recomputed = std::max(a.rows_recomputed, c.rows_recomputed);
        st->rebuilt = a.rebuilt | c.rebuilt;
        st->rows_local = a.rows_local | c.rows_local;
        st->del_repair_ms = a.del_repair_ms;
        st->ins_repair_ms = c.ins_repair_ms;
        st->ins_scanned = c.ins_scanned;
        st->region = a.region + c.region;
        st->apply_ms = a.apply_ms + c.apply_ms;
        st->core_ms = a.core_ms + c.core_ms;
        st->rows_ms = a.rows_ms + c.rows_ms;
        st->total_ms = a.total_ms + c.total_ms;
        st->method = method;
        h->mtimes.total_ms = st->total_ms;
        if (h->log_maint && want_feat) log_batch(h, feat, st);
        return DC_OK;
    }
    st->deleted = nb.n_del;
    st->inserted = nb.n_ins;
    st->method = method;
    cudaEvent_t* ev = h->ev;
    cudaEventRecord(ev[0], h->stream);
    if (!s->kmax_old && (mt_malloc(h->stream, &s->kmax_old, (uint64_t)V + 1) || mt_malloc(h->stream, &s->row0_old, (uint64_t)V + 1)))
        return DC_ERR_NOMEM;
    // values before the batch (for the row bound) and row 0 in scratch
    MT_CUDA(cudaMemcpyAsync(s->kmax_old, d.kmax_v, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
    uint32_t *d_du = nullptr, *d_dv = nullptr, *d_iu = nullptr, *d_iv = nullptr;
    int rc = DC_OK;
    int rebuilt = 0;
    uint64_t region = 0;
    // ---- deletions
    if (!nb.del_u.empty()) {
        if ((rc = apply_deletions(h, nb))) return rc;
        std::vector<uint32_t> heads(nb.del_v), tails(nb.del_u);
        if ((rc = upload(h, &d_dv, heads)) || (rc = upload(h, &d_du, tails))) goto out;
        if (method == DC_MAINT_LOCAL) {
            MT_CUDA(cudaMemcpyAsync(s->row0_old, d.row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
            if ((rc = core_local(h, 0, d.kmax_v, s->kmax_old, d_dv, (uint32_t)heads.size(), 0, 0, &region))) goto out;
            if ((rc = core_local(h, 1, d.row0, s->row0_old, d_du, (uint32_t)tails.size(), 0, 0, &region))) goto out;
        }
    }
    // ---- insertions
    if (!nb.ins_u.empty()) {
        if ((rc = apply_insertions(h, nb, &d_iu, &d_iv, &rebuilt))) goto out;
        if (method == DC_MAINT_LOCAL) {
            int32_t bb = (int32_t)std::min<uint64_t>(nb.n_ins, 0x3FFFFFFF);
            int32_t* old_k = s->cdeg2;  // values before the insertions
            int32_t* old_r = s->key2;
            MT_CUDA(cudaMemcpyAsync(old_k, d.kmax_v, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
            MT_CUDA(cudaMemcpyAsync(old_r, d.row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
            if ((rc = core_local(h, 0, d.kmax_v, old_k, d_iv, (uint32_t)nb.ins_u.size(), 1, bb, &region))) goto out;
            if ((rc = core_local(h, 1, d.row0, old_r, d_iu, (uint32_t)nb.ins_u.size(), 1, bb, &region))) goto out;
        }
    }
    cudaEventRecord(ev[1], h->stream);
    if (method == DC_MAINT_REPEEL) {
        int32_t km = 0, lm = 0;
        if ((rc = peel_kmax_row0(h, &km, &lm))) goto out;
        MT_CUDA(cudaMemcpyAsync(d.row0, s->row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
    }
    cudaEventRecord(ev[2], h->stream);
    st->region = region;
    st->rebuilt = (uint32_t)rebuilt;
    {
        // ---- rows that can change: rows up to R
        int* dbuf = (int*)s->cursor;  // [0] = R, [1] = new kmax, [2] = new lmax
        int init[3] = {-1, 0, 0};
        MT_CUDA(cudaMemcpyAsync(dbuf, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
        if (!nb.del_u.empty()) {
            ++g_launches;
            k_rows_bound_edges<<<mgrid(h, nb.del_u.size()), kMThreads, 0, h->stream>>>(
                (uint32_t)nb.del_u.size(), d_du, d_dv, s->kmax_old, d.kmax_v, dbuf);
        }
        if (!nb.ins_u.empty()) {
            ++g_launches;
            k_rows_bound_edges<<<mgrid(h, nb.ins_u.size()), kMThreads, 0, h->stream>>>(
                (uint32_t)nb.ins_u.size(), d_iu, d_iv, s->kmax_old, d.kmax_v, dbuf);
        }
        ++g_launches;
        k_rows_bound_changed<<<mgrid(h, V), kMThreads, 0, h->stream>>>(V, s->kmax_old, d.kmax_v, dbuf, dbuf + 1);
        ++g_launches;
        k_vmax<<<mgrid(h, V), kMThreads, 0, h->stream>>>(V, d.row0, dbuf + 2);
        int res[3];
        MT_CUDA(cudaMemcpyAsync(res, dbuf, sizeof(res), cudaMemcpyDeviceToHost, h->stream));
        MT_CUDA(cudaStreamSynchronize(h->stream));
        const int32_t Knew = res[1];
        const int32_t R = std::min(res[0], Knew);
        st->rows_recomputed = R + 1;
        if (R < 0) {
            // nothing changed
            d.kmax = Knew;
            d.lmax = res[2];
            d.rows_valid = false;
            st->kmax = d.kmax;
            st->lmax = d.lmax;
            goto timing;
        }
        // ---- no row above 0 can change: only row 0's corners are new
        if (R == 0) {
            bool applied = false;
            if ((rc = apply_change_log(h, 0, &applied))) goto out;
            if (applied) {
                d.kmax = Knew;
                d.lmax = res[2];
                d.rows_valid = false;
                d.valid = true;
                st->kmax = d.kmax;
                st->lmax = d.lmax;
                goto timing;
            }
        }
        // ---- deletions only: repair rows 1..R in place
        if (repair_del && nb.ins_u.empty()) {
            bool applied = false;
            cudaEventRecord(ev[4], h->stream);
            if ((rc = rows_repair(h, R, d_du, d_dv, (uint32_t)nb.del_u.size(), repair_deadline_ns(h, R, rmode),
                                  &applied)))
                goto out;
            cudaEventRecord(ev[5], h->stream);
            cudaEventSynchronize(ev[5]);
            cudaEventElapsedTime(&st->del_repair_ms, ev[4], ev[5]);
            if (applied) {
                st->rows_local = 1;
                d.kmax = Knew;
                d.lmax = res[2];
                d.rows_valid = false;
                d.valid = true;
                st->kmax = d.kmax;
                st->lmax = d.lmax;
                goto timing;
            }
        }
        // ---- insertions only: repair rows 1..R in place
        if (repair_ins && nb.del_u.empty()) {
            bool applied = false;
            unsigned long long scanned = 0;
            cudaEventRecord(ev[4], h->stream);
            if ((rc = rows_repair_ins(h, R, d_iu, d_iv, (uint32_t)nb.ins_u.size(), repair_deadline_ns(h, R, rmode), &applied,
                                      &scanned)))
                goto out;
            cudaEventRecord(ev[5], h->stream);
            cudaEventSynchronize(ev[5]);
            cudaEventElapsedTime(&st->ins_repair_ms, ev[4], ev[5]);
            st->ins_scanned = scanned;
            if (applied) {
                st->rows_local = 2;
                d.kmax = Knew;
                d.lmax = res[2];
                d.rows_valid = false;
                d.valid = true;
                st->kmax = d.kmax;
                st->lmax = d.lmax;
                goto timing;
            }
        }
        // ---- rows 0..R from the new row 0, rows above R from the old skyline
        if ((rc = recompute_rows(h, R, Knew, res[2]))) goto out;
        st->kmax = d.kmax;
        st->lmax = d.lmax;
    }
timing:
    cudaEventRecord(ev[3], h->stream);
    MT_CUDA(cudaStreamSynchronize(h->stream));
    {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        st->apply_ms = ms;
        cudaEventElapsedTime(&ms, ev[1], ev[2]);
        st->core_ms = ms;
        cudaEventElapsedTime(&ms, ev[2], ev[3]);
        st->rows_ms = ms;
        cudaEventElapsedTime(&ms, ev[0], ev[3]);
        st->total_ms = ms;
        h->mtimes.total_ms = ms;
    }
    st->kmax = d.kmax;
    st->lmax = d.lmax;
    if (h->log_maint && want_feat) log_batch(h, feat, st);
out:
    mt_free(h->stream, d_du);
    mt_free(h->stream, d_dv);
    mt_free(h->stream, d_iu);
    mt_free(h->stream, d_iv);
    if (rc != DC_OK) {
        d.valid = false;
        d.peel_valid = false;
    } else {
        d.row_lo = 1;
        d.row_hi = d.kmax;
    }
    return rc;
}

int maintain(dc_graph* h, const uint32_t* pairs, const uint8_t* is_del, uint64_t b, int method, dc_maint_stats* st) {
    return maintain_impl(h, pairs, is_del, b, method, -1, false, st);
}

}  // namespace dc
