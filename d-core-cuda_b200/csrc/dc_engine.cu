// Device engine: slack CSR/CSC build, persistent peel, incremental row
// transitions, skyline assembly and dense row expansion.
//
// Reference path (llysdal/d-core-cuda):
//   graph upload      moveGraphToDevice, src/cuda_memory.h:32-41
//   peel pass         scan + process kernels driven by KListInplace,
//                     main.cu:27-141, 171-195
//   decomposition     dcore, main.cu:197-262 (kmax via swapInOut, then one
//                     pass per k = 0..kmax)
// The engine computes the same numbers with a different schedule: one
// persistent cooperative kernel per pass (software grid barrier per level, a
// device work queue for cascades, no host round trip per level), and rows
// k >= 1 derived from row k-1 by h-index refinement instead of one fresh
// peel per row (see k_transitions).
#include <atomic>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dc_engine.cuh"
#include "dc_internal.h"

namespace dc {

// Kernel launches issued by the engine since load (host counter).
std::atomic<unsigned long long> g_launches{0};

#define DC_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess)                                                               \
            return set_error(DC_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), \
                             __FILE__, __LINE__);                                            \
    } while (0)

static constexpr int kThreads = 256;
static constexpr int kWarpsPerBlock = kThreads / 32;

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------

// Device buffers of a handle come from the device's stream-ordered pool on
// the handle's stream: no implicit device-wide synchronisation, so handles on
// different streams (the serving loop runs many) keep their kernels
// overlapping while they allocate and free.
template <typename T>
static int dmalloc(cudaStream_t st, T** p, uint64_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMallocAsync((void**)p, n * sizeof(T), st);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "device allocation of %llu bytes failed: %s",
                         (unsigned long long)(n * sizeof(T)), cudaGetErrorString(e));
    }
    return DC_OK;
}
template <typename T>
static void dfree(cudaStream_t st, T*& p) {
    if (p) cudaFreeAsync((void*)p, st);
    p = nullptr;
}

__device__ __forceinline__ unsigned warp_incl_scan(unsigned x) {
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    return x;
}

__device__ __forceinline__ unsigned long long warp_incl_scan64(unsigned long long x) {
    const unsigned lane = threadIdx.x & 31u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    return x;
}

// Block-wide exclusive scan of one 64-bit value per thread; returns the block
// total through *total.
__device__ unsigned long long block_excl_scan64(unsigned long long x, unsigned long long* total) {
    __shared__ unsigned long long s_w[32];
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    unsigned long long inc = warp_incl_scan64(x);
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (w == 0) {
        unsigned nw = blockDim.x >> 5;
        unsigned long long v = lane < nw ? s_w[lane] : 0ull;
        unsigned long long vi = warp_incl_scan64(v);
        if (lane < nw) s_w[lane] = vi - v;
        if (lane == nw - 1) s_w[31] = vi;
    }
    __syncthreads();
    unsigned long long res = inc - x + s_w[w];
    *total = s_w[31];
    __syncthreads();
    return res;
}

// Block-wide reservation for the peel's scans: every thread of the block
// contributes nk entries to append to a list (counter *list_ctr) and ni queue
// items; thread 0 reserves both ranges with one atomic each (the items'
// outstanding count is raised before their slots can be filled) and every
// thread gets its own offsets.  All threads of the block must call it.
__device__ __forceinline__ void block_reserve(EngineCtl* c, unsigned* list_ctr, unsigned nk, unsigned ni,
                                              unsigned* keep_off, unsigned* item_off) {
    __shared__ unsigned s_kb, s_ib;
    unsigned long long tot;
    const unsigned long long ex = block_excl_scan64(((unsigned long long)nk << 32) | ni, &tot);
    if (threadIdx.x == 0) {
        const unsigned tk = (unsigned)(tot >> 32), ti = (unsigned)tot;
        s_kb = tk ? atomicAdd(list_ctr, tk) : 0u;
        s_ib = 0;
        if (ti) {
            atomicAdd(&c->outstanding, (int)ti);
            s_ib = atomicAdd(&c->t_tail, ti);
        }
    }
    __syncthreads();
    *keep_off = s_kb + (unsigned)(ex >> 32);
    *item_off = s_ib + (unsigned)ex;
    __syncthreads();
}

// Block-wide minimum, one global atomicMin per block (all threads call it).
__device__ __forceinline__ void block_atomic_min(int* dst, int x) {
    __shared__ int s_m;
    if (threadIdx.x == 0) s_m = 0x7FFFFFFF;
    __syncthreads();
#pragma unroll
    for (int o = 16; o; o >>= 1) x = min(x, __shfl_xor_sync(0xFFFFFFFFu, x, o));
    if ((threadIdx.x & 31u) == 0 && x != 0x7FFFFFFF) atomicMin(&s_m, x);
    __syncthreads();
    if (threadIdx.x == 0 && s_m != 0x7FFFFFFF) atomicMin(dst, s_m);
    __syncthreads();
}

// ---------------------------------------------------------------------------
// cooperative exclusive scan (u64), n elements in place; out[n] = total
// ---------------------------------------------------------------------------
__global__ void k_scan_coop(unsigned long long* data, uint64_t n, unsigned long long* partial, EngineCtl* c) {
    const uint64_t nb = gridDim.x;
    const uint64_t per = (n + nb - 1) / nb;
    const uint64_t lo = min(n, per * blockIdx.x), hi = min(n, lo + per);
    // phase 1: block sums
    unsigned long long s = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += data[i];
    unsigned long long tot;
    block_excl_scan64(s, &tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
    if (!grid_sync(c)) return;
    // phase 2: block 0 scans the partials
    if (blockIdx.x == 0) {
        unsigned long long carry = 0;
        for (uint64_t b0 = 0; b0 < nb; b0 += blockDim.x) {
            uint64_t b = b0 + threadIdx.x;
            unsigned long long v = b < nb ? partial[b] : 0ull;
            unsigned long long t2;
            unsigned long long ex = block_excl_scan64(v, &t2);
            if (b < nb) partial[b] = ex + carry;
            carry += t2;
            __syncthreads();
        }
        if (threadIdx.x == 0) data[n] = carry;
    }
    if (!grid_sync(c)) return;
    // phase 3: scan own range
    unsigned long long carry = partial[blockIdx.x];
    for (uint64_t b0 = lo; b0 < hi; b0 += blockDim.x) {
        uint64_t i = b0 + threadIdx.x;
        unsigned long long v = i < hi ? data[i] : 0ull;
        unsigned long long t2;
        unsigned long long ex = block_excl_scan64(v, &t2);
        if (i < hi) data[i] = ex + carry;
        carry += t2;
    }
}

// ---------------------------------------------------------------------------
// graph build
// ---------------------------------------------------------------------------
__global__ void k_count_degrees(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, int32_t* out_len,
                                int32_t* in_len, EngineCtl* c) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s = src[e], d = dst[e];
        if (s >= V || d >= V) {
            set_dev_error(c, DC_DEV_ERR_BADID, 10);
            continue;
        }
        atomicAdd(&out_len[s], 1);
        atomicAdd(&in_len[d], 1);
    }
}

// capacity of v's list = len + max(gap_min, len / gap_div)
__global__ void k_capacity(uint32_t V, const int32_t* len, uint32_t gap_min, uint32_t gap_div, unsigned long long* cap) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t l = (uint32_t)len[v];
        uint32_t g = gap_min;
        if (gap_div) g = max(g, l / gap_div);
        cap[v] = (unsigned long long)l + g;
    }
}

__global__ void k_off_to_u32(uint32_t V, const unsigned long long* in, uint32_t* out) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= V; v += (uint64_t)gridDim.x * blockDim.x)
        out[v] = (uint32_t)in[v];
}

__global__ void k_scatter_edges(uint64_t E, const uint32_t* src, const uint32_t* dst, const uint32_t* out_off,
                                int32_t* out_fill, uint32_t* out_nbr, const uint32_t* in_off, int32_t* in_fill,
                                uint32_t* in_nbr) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s = src[e], d = dst[e];
        int po = atomicAdd(&out_fill[s], 1);
        out_nbr[out_off[s] + po] = d;
        int pi = atomicAdd(&in_fill[d], 1);
        in_nbr[in_off[d] + pi] = s;
    }
}

// ---------------------------------------------------------------------------
// incremental rows: shared helpers
// ---------------------------------------------------------------------------
static constexpr int kWin = 64;

// The last warp of a block to finish its seeding share reports the block as
// one producer (outstanding counts blocks, not warps: far fewer atomics on
// the shared counter per step).
__device__ __forceinline__ void block_producer_done(EngineCtl* c, unsigned* s_cnt) {
    __syncwarp();
    if ((threadIdx.x & 31u) == 0) {
        __threadfence();
        unsigned o = atomicAdd(s_cnt, 1u);
        if (o == (blockDim.x >> 5) - 1) {
            *s_cnt = 0;
            if (c->trace) {
                int st = ld_vol(&c->step);
                if (st >= 0 && (unsigned)st < c->trace_cap) atomicMax(&c->trace[8 * st + 5], gtimer());
            }
            tq_finish(c, 1);
        }
    }
    __syncwarp();
}

// Per-vertex queue state for the transition drain:
//   0 idle, 1 queued, 2 being evaluated, 3 being evaluated and re-run
//   requested.  A vertex is never evaluated by two warps at once, and a
//   request that lands during an evaluation re-queues the vertex when that
//   evaluation ends.  Returns true when the caller must push the vertex.
__device__ __forceinline__ bool mark_request(uint32_t* m, EngineCtl* c) {
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
    set_dev_error(c, DC_DEV_ERR_TIMEOUT, 21);
    return false;
}

// ---------------------------------------------------------------------------
// fused peel, ticket queue, chunked items
// ---------------------------------------------------------------------------
struct PeelInst {
    const uint32_t* a_off;
    const int32_t* a_len;
    const uint32_t* a_nbr;
    const uint32_t* b_off;
    const int32_t* b_len;
    const uint32_t* b_nbr;
    const int32_t* member;  // nullptr: all vertices
    int32_t k;              // constraint threshold (0: none)
    int32_t* key;
    int32_t* cdeg;
    int32_t* val;
    uint32_t* rem0;
    uint32_t* rem1;
};

struct Peel2Params {
    uint32_t V;
    int ninst;
    unsigned chunk;  // adjacency entries per queue item
    PeelInst in[2];
    TicketQueue q;
    EngineCtl* ctl;
};

__device__ __forceinline__ unsigned long long peel_item(uint32_t v, unsigned ch, int inst) {
    return (unsigned long long)v | ((unsigned long long)ch << 32) | ((unsigned long long)inst << 63);
}

__device__ __forceinline__ unsigned peel_nitems(const PeelInst& I, uint32_t x, unsigned CH) {
    unsigned len = (unsigned)(I.k > 0 ? I.a_len[x] : 0) + (unsigned)I.b_len[x];
    return (len + CH - 1) / CH;
}

struct PeelHook {
    int ninst;
    unsigned nworkers;
    __device__ void operator()(EngineCtl* c) const {
        // next level: a level whose scan found nothing to remove changed no
        // degree, so the following levels up to the least degree kept are
        // empty too and are skipped
        if (c->step < 0) {
            c->level = 0;
        } else if (c->t_tail == c->trace_tail0) {
            int m = 0x7FFFFFFF;
            for (int i = 0; i < ninst; ++i)
                if (c->rc_next[i].v) m = min(m, c->minkey[i].v);
            c->level = max(c->level + 1, m == 0x7FFFFFFF ? c->level + 1 : m);
        } else {
            c->level = c->level + 1;
        }
        for (int i = 0; i < ninst; ++i) {
            c->rc_cur[i] = c->rc_next[i].v;
            c->rc_next[i].v = 0;
            c->minkey[i].v = 0x7FFFFFFF;
        }
        trace_step_end(c);
        c->t_tail = c->t_head;
        c->trace_tail0 = c->t_tail;
        c->outstanding = (int)nworkers;
        c->phase_done = 0;
        __threadfence();
    }
};

// Converged warp: when the warp holds no item of its own (*keep empty), it
// keeps the first of the items the lowest lane with *cnt > 0 is about to push
// (*first, then *first + chunk step for the rest) to process next itself; the
// kept item counts as outstanding like a queued one.
__device__ __forceinline__ void keep_first_item(EngineCtl* c, unsigned long long* keep, unsigned* cnt,
                                                unsigned long long* first) {
    if (*keep != kEmptyItem) return;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, *cnt > 0);
    if (!m) return;
    const unsigned src = __ffs(m) - 1;
    const unsigned long long it = __shfl_sync(0xFFFFFFFFu, *first, src);
    if (lane == src) {
        *first += 1ull << 32;  // next chunk of the same vertex
        --*cnt;
    }
    if (lane == 0) atomicAdd(&c->outstanding, 1);
    *keep = it;
}

// Up to two independent peels advance level by level in one grid: the kmax
// pass (peeling in-degree, swapInOut + KListInplace(k = 0), main.cu:218-220)
// and row 0 (peeling out-degree), or two rows of the per-row method.  Level
// L of each peel removes every remaining vertex whose peeling degree is at
// most L (scan, main.cu:37-56) and the cascade that follows (process,
// main.cu:100-135) with value L.  Work items are (vertex, chunk of its
// adjacency), so hub lists spread over many warps.
#ifndef DC_PEEL_MIN_BLOCKS
#define DC_PEEL_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kThreads, DC_PEEL_MIN_BLOCKS) k_peel2(Peel2Params p) {
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const unsigned gwarp = blockIdx.x * kWarpsPerBlock + wib;
    const unsigned nwarps = gridDim.x * kWarpsPerBlock;
    EngineCtl* c = p.ctl;
    const unsigned CH = p.chunk;
    PeelHook hook{p.ninst, gridDim.x};
    __shared__ unsigned s_prod;
    if (threadIdx.x == 0) s_prod = 0;
    __syncthreads();

    // ---- init (remaining lists appended block by block: one atomic per block chunk)
    for (int i = 0; i < p.ninst; ++i) {
        const PeelInst& I = p.in[i];
        for (uint64_t base = (uint64_t)blockIdx.x * kThreads; base < p.V; base += (uint64_t)gridDim.x * kThreads) {
            uint64_t vi = base + threadIdx.x;
            bool ok = vi < p.V, in = false;
            uint32_t v = (uint32_t)vi;
            if (ok) {
                in = !I.member || I.member[v] >= I.k;
                if (!in) {
                    I.val[v] = 0;
                } else {
                    I.val[v] = -1;
                    int kd = 0, cd = 0;
                    if (!I.member) {
                        kd = I.a_len[v];
                    } else {
                        uint32_t o = I.a_off[v], e = o + (uint32_t)I.a_len[v];
                        for (; o < e; ++o) kd += (I.member[I.a_nbr[o]] >= I.k);
                        o = I.b_off[v];
                        e = o + (uint32_t)I.b_len[v];
                        for (; o < e; ++o) cd += (I.member[I.b_nbr[o]] >= I.k);
                    }
                    I.key[v] = kd;
                    I.cdeg[v] = cd;
                }
            }
            unsigned pos, unused;
            block_reserve(c, &c->rc_next[i].v, (ok && in) ? 1u : 0u, 0u, &pos, &unused);
            if (ok && in) I.rem0[pos] = v;
        }
    }
    if (!grid_sync_hook(c, hook)) return;

    unsigned ticket = kNoTicket;
    for (int it = 0;; ++it) {
        const int L = ld_vol(&c->level);
        bool any_left = false;
        for (int i = 0; i < p.ninst; ++i) any_left |= ld_vol(&c->rc_cur[i]) != 0u;
        if (!any_left) break;
        unsigned pushed_mask = 0;
        // ---- scan remaining lists
        for (int i = 0; i < p.ninst; ++i) {
            const PeelInst& I = p.in[i];
            const unsigned n_rem = ld_vol(&c->rc_cur[i]);
            const uint32_t* rc = (it & 1) ? I.rem1 : I.rem0;
            uint32_t* rn = (it & 1) ? I.rem0 : I.rem1;
            // block-cooperative: the kept vertices and the pushed items of a
            // chunk of blockDim vertices take one reservation per block
            // (kSeedPer vertices per thread and step)
            constexpr int kSeedPer = 1;  // measured: four per thread was slower (18.3 -> 19.2 ms)
            int kmin = 0x7FFFFFFF;
            for (unsigned base = blockIdx.x * kThreads * kSeedPer; base < n_rem;
                 base += gridDim.x * kThreads * kSeedPer) {
                uint32_t vv[kSeedPer];
                unsigned cnt[kSeedPer];
                unsigned keepm = 0, nk = 0, ni = 0;
                bool pushed = false;
#pragma unroll
                for (int r = 0; r < kSeedPer; ++r) {
                    const unsigned idx = base + r * kThreads + threadIdx.x;
                    const bool ok = idx < n_rem;
                    const uint32_t v = ok ? rc[idx] : 0;
                    bool keep = false, push = false;
                    if (ok && ld_vol(&I.val[v]) == -1) {
                        int kv = ld_vol(&I.key[v]);
                        if (kv <= L) {
                            push = atomicCAS(&I.val[v], -1, L) == -1;
                        } else {
                            keep = true;
                            kmin = min(kmin, kv);
                        }
                    }
                    vv[r] = v;
                    cnt[r] = push ? peel_nitems(I, v, CH) : 0u;
                    keepm |= keep ? 1u << r : 0u;
                    nk += keep ? 1u : 0u;
                    ni += cnt[r];
                    pushed |= push;
                }
                unsigned kpos, ipos;
                block_reserve(c, &c->rc_next[i].v, nk, ni, &kpos, &ipos);
                if (ni) __threadfence();
#pragma unroll
                for (int r = 0; r < kSeedPer; ++r) {
                    if (keepm & (1u << r)) rn[kpos++] = vv[r];
                    for (unsigned j = 0; j < cnt[r]; ++j) {
                        volatile unsigned long long* sl = &p.q.slots[(ipos++) & p.q.mask];
                        *sl = peel_item(vv[r], j, i);
                    }
                }
                if (__any_sync(0xFFFFFFFFu, pushed)) pushed_mask |= 1u << i;
            }
            block_atomic_min(&c->minkey[i].v, kmin);
        }
        block_producer_done(c, &s_prod);
        // ---- drain the cascade: the warp's kept item first, else the queue;
        // finished items are counted off in batches (before the warp waits)
        unsigned long long item;
        unsigned long long pkeep = kEmptyItem;
        unsigned done_pending = 0;
        for (;;) {
            if (pkeep != kEmptyItem) {
                item = pkeep;
                pkeep = kEmptyItem;
            } else if (!tq_take_warp_lazy(c, p.q, &ticket, &item, &done_pending)) {
                break;
            }
            const int i = (int)(item >> 63);
            const uint32_t x = (uint32_t)item;
            const unsigned ch = (unsigned)((item >> 32) & 0x7FFFFFFFull);
            const PeelInst& I = p.in[i];
            const unsigned la = (unsigned)(I.k > 0 ? I.a_len[x] : 0);
            const unsigned len = la + (unsigned)I.b_len[x];
            const unsigned e0 = ch * CH, e1 = min(len, e0 + CH);
            const uint32_t ao = I.a_off[x], bo = I.b_off[x];
            bool pushed = false;
            for (unsigned base = e0; base < e1; base += 64) {
                // two entries per lane, both atomics issued before either result is used
                unsigned ea = base + lane, eb = base + 32 + lane;
                int olda = 0, oldb = 0;
                uint32_t ua = 0, ub = 0;
                bool isa_a = false, isa_b = false;
                if (ea < e1) {
                    isa_a = ea < la;
                    ua = isa_a ? I.a_nbr[ao + ea] : I.b_nbr[bo + (ea - la)];
                }
                if (eb < e1) {
                    isa_b = eb < la;
                    ub = isa_b ? I.a_nbr[ao + eb] : I.b_nbr[bo + (eb - la)];
                }
                if (ea < e1) olda = atomicSub(isa_a ? &I.cdeg[ua] : &I.key[ua], 1);
                if (eb < e1) oldb = atomicSub(isa_b ? &I.cdeg[ub] : &I.key[ub], 1);
                bool pa = ea < e1 && (isa_a ? olda == I.k : olda == L + 1) && ld_vol(&I.val[ua]) == -1 &&
                          atomicCAS(&I.val[ua], -1, L) == -1;
                bool pb = eb < e1 && (isa_b ? oldb == I.k : oldb == L + 1) && ld_vol(&I.val[ub]) == -1 &&
                          atomicCAS(&I.val[ub], -1, L) == -1;
                unsigned cnta = pa ? peel_nitems(I, ua, CH) : 0u;
                unsigned long long fa = peel_item(ua, 0, i);
                keep_first_item(c, &pkeep, &cnta, &fa);
                tq_push_warp_multi(c, p.q, cnta, fa, 1ull << 32);
                unsigned cntb = pb ? peel_nitems(I, ub, CH) : 0u;
                unsigned long long fb = peel_item(ub, 0, i);
                keep_first_item(c, &pkeep, &cntb, &fb);
                tq_push_warp_multi(c, p.q, cntb, fb, 1ull << 32);
                pushed |= __any_sync(0xFFFFFFFFu, pa || pb);
            }
            if (pushed) pushed_mask |= 1u << i;
            __syncwarp();
            if (lane == 0) ++done_pending;
        }
        if (lane == 0) {
            for (int i = 0; i < p.ninst; ++i)
                if (pushed_mask & (1u << i)) atomicMax(&c->maxv[i], L);
        }
        if (!grid_sync_hook(c, hook)) return;
    }
}

// ---------------------------------------------------------------------------
// incremental rows with exact support counters
// ---------------------------------------------------------------------------
struct Trans2Params {
    uint32_t V;
    const uint32_t* out_off;
    int32_t* out_len;
    uint32_t* out_nbr;
    const uint32_t* in_off;
    int32_t* in_len;
    uint32_t* in_nbr;
    const int32_t* kmax;
    int32_t K;
    int32_t K0;     // first row to compute; cur holds row 0 (K0 > 1 jumps straight to row K0)
    // preleft: cur already holds -1 for the vertices outside C_K0 and the
    // counters ignore them, so the first row has no leaving set and seeds
    // every member whose out-count is below its value as well (the host
    // always starts runs this way; 0 = the leaving pass removes them)
    int preleft;
    int32_t Kstop;  // last row to compute (rows above stay untouched)
    int sorted;     // lists ordered by neighbour kmax, descending
    const uint32_t* order;  // C_k = order[0 .. ck[k]); nullptr: the graph is relabeled, C_k = ids 0 .. ck[k]-1
    const uint32_t* ck;
    int32_t* cur;
    int32_t* cnt_out;  // #{u in N_out(v) : cur[u] >= cur[v]}  (never above the truth)
    int32_t* cnt_in;   // #{w in N_in(v)  : cur[w] >= cur[v]}
    uint32_t* mark;
    int32_t* stamp;
    uint32_t* logidx;
    uint32_t* log_v;
    int32_t* log_k;
    int32_t* log_l;
    unsigned long long log_cap;
    TicketQueue q;
    EngineCtl* ctl;
};

struct TransHook {
    unsigned nworkers;
    int K;
    int K0;
    __device__ void operator()(EngineCtl* c) const {
        // next row: after a row that needed no work, jump to the first row
        // whose leaving set or seed set can be non-empty (next_min)
        if (c->step < 0) c->level = K0;
        else if (c->t_tail == c->trace_tail0) c->level = max(c->level + 1, c->next_min);
        else c->level = c->level + 1;
        c->next_min = K + 1;
        trace_step_end(c);
        c->t_tail = c->t_head;
        c->trace_tail0 = c->t_tail;
        c->outstanding = (int)nworkers;
        c->phase_done = 0;
        __threadfence();
    }
};

// Starting values of a run of rows that starts at row a: row 0 inside C_a,
// -1 (left) outside.
__global__ void k_preleft_cur(uint32_t V, const int32_t* kmax, const int32_t* row0, int32_t a, int32_t* cur) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        cur[v] = kmax[v] >= a ? row0[v] : -1;
}

// This lane's share of #{entries u of list a[0..n) : cur[u] >= cv}, 128
// entries per warp step; on kmax-sorted lists (sorted != 0) the count stops
// after the step whose last entry has cur == -1 (outside C_a: so is every
// later entry).
__device__ __forceinline__ int count_at_least(const int32_t* cur, const uint32_t* a, int n, int cv, int sorted) {
    const unsigned lane = threadIdx.x & 31u;
    int c = 0;
    for (int b = 0; b < n; b += 128) {
        int x[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = b + 32 * r + (int)lane;
            x[r] = e < n ? cur[a[e]] : -1;
            c += (x[r] >= cv);
        }
        if (sorted && b + 128 < n && __shfl_sync(0xFFFFFFFFu, x[3], 31) == -1) break;
    }
    return c;
}

// Counters of v against every neighbour, at v's starting value (vertices
// with a value below 1 get zero counts: they are never evaluated and no
// counter includes them).  On kmax-sorted lists (sorted != 0) a list ends at
// its first neighbour outside C_a: cur holds -1 there and for every later
// entry, which counts nothing.
__global__ void k_counters_init(uint32_t V, const uint32_t* out_off, const int32_t* out_len, const uint32_t* out_nbr,
                                const uint32_t* in_off, const int32_t* in_len, const uint32_t* in_nbr,
                                const int32_t* cur, int32_t* cnt_out, int32_t* cnt_in, int sorted) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = gw; v < V; v += nw) {
        int cv = cur[v];
        int co = 0, ci = 0;
        if (cv < 1) {  // never evaluated, never counted: no support needed
            if (lane == 0) {
                cnt_out[v] = 0;
                cnt_in[v] = 0;
            }
            continue;
        }
        co = count_at_least(cur, out_nbr + out_off[v], out_len[v], cv, sorted);
        ci = count_at_least(cur, in_nbr + in_off[v], in_len[v], cv, sorted);
#pragma unroll
        for (int s = 16; s; s >>= 1) {
            co += __shfl_xor_sync(0xFFFFFFFFu, co, s);
            ci += __shfl_xor_sync(0xFFFFFFFFu, ci, s);
        }
        if (lane == 0) {
            cnt_out[v] = co;
            cnt_in[v] = ci;
        }
    }
}

// Converged warp: when the warp holds no item of its own yet (*keep ==
// kNoKeep), it keeps the first request of the lowest requesting lane to
// evaluate next itself instead of queueing it: the link from a drop to the
// neighbour's evaluation skips the queue's publish and take.  The kept item
// counts as outstanding like a queued one.
constexpr uint32_t kNoKeep = 0xFFFFFFFFu;
// Requests of a lane: bit r of *req set = u[r] is requested (r < 4); the
// items stay in registers (no dynamically indexed array).
__device__ __forceinline__ uint32_t first_requested(unsigned req, const uint32_t u[4]) {
    return (req & 1u) ? u[0] : (req & 2u) ? u[1] : (req & 4u) ? u[2] : u[3];
}
__device__ __forceinline__ void keep_one(EngineCtl* c, uint32_t* keep, unsigned* req, const uint32_t u[4]) {
    if (*keep != kNoKeep) return;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, *req != 0u);
    if (!m) return;
    const unsigned src = __ffs(m) - 1;
    const uint32_t item = __shfl_sync(0xFFFFFFFFu, first_requested(*req, u), src);
    if (lane == src) *req &= *req - 1u;  // drop the kept request
    if (lane == 0) atomicAdd(&c->outstanding, 1);
    *keep = item;
}

// ---- vectorised list passes of the row kernel ----------------------------
// A list is read with 16-byte id loads: the list at element offset o of its
// array, length n, is covered by the virtual indices t in [o & 3, (o & 3) + n)
// of the 16-byte aligned window starting at o - (o & 3); lane l takes the
// four ids at t = b + 4 l .. b + 4 l + 3 of the step starting at b (128
// entries per list and step), so eight neighbour values per lane (both
// lists) are gathered in flight at once.  The adjacency arrays are 16-byte
// aligned and padded so that the last window of the last list stays inside.
__device__ __forceinline__ void load_ids4(const uint32_t* nbr, uint32_t o, int end, int b, bool active, uint32_t u[4]) {
    const int t0 = b + 4 * (int)(threadIdx.x & 31u);
    uint4 w = make_uint4(0u, 0u, 0u, 0u);
    if (active && t0 < end) w = *reinterpret_cast<const uint4*>(nbr + (o - (o & 3u)) + t0);
    u[0] = w.x;
    u[1] = w.y;
    u[2] = w.z;
    u[3] = w.w;
}

__device__ __forceinline__ int sel4(const int x[4], int q) { return q == 0 ? x[0] : q == 1 ? x[1] : q == 2 ? x[2] : x[3]; }

// Value of the step's last entry (virtual index last >= b) for the early stop
// on kmax-sorted lists.
__device__ __forceinline__ int last_value(const int x[4], int b, int last) {
    const int r = last - b;
    return __shfl_sync(0xFFFFFFFFu, sel4(x, r & 3), r >> 2);
}

// hist_pass2 with 16-byte id loads (same bins, counts and stopping rule).
__device__ __forceinline__ int hist_pass2v(const int32_t* cur, const uint32_t* onbr, uint32_t oo, int no,
                                           const uint32_t* inbr, uint32_t io, int ni, int lo, int hi, bool first,
                                           bool sorted, int* bo, int* bi) {
    const unsigned lane = threadIdx.x & 31u;
    const int so = (int)(oo & 3u), si = (int)(io & 3u), endo = so + no, endi = si + ni;
    int to = 0, ti = 0, entries = 0;
    bool doneo = no <= 0, donei = ni <= 0;
    for (int b = 0; !(doneo && donei); b += 128) {
        uint32_t uo[4], ui[4];
        load_ids4(onbr, oo, endo, b, !doneo, uo);
        load_ids4(inbr, io, endi, b, !donei, ui);
        const int t0 = b + 4 * (int)lane;
        int co[4], ci[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int t = t0 + q;
            co[q] = (!doneo && t >= so && t < endo) ? ld_vol(&cur[uo[q]]) : -1;
            ci[q] = (!donei && t >= si && t < endi) ? ld_vol(&cur[ui[q]]) : -1;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int x = co[q];
            to += first ? (x >= hi) : (x == hi);
            if (x >= lo && x < hi) atomicAdd(&bo[x - lo], 1);
            x = ci[q];
            ti += first ? (x >= hi) : (x == hi);
            if (x >= lo && x < hi) atomicAdd(&bi[x - lo], 1);
        }
        if (!doneo) {
            const int last = min(b + 127, endo - 1);
            entries += last + 1 - max(b, so);
            const int lv = last_value(co, b, last);
            if (b + 128 >= endo || (sorted && lv == -1)) doneo = true;
        }
        if (!donei) {
            const int last = min(b + 127, endi - 1);
            entries += last + 1 - max(b, si);
            const int lv = last_value(ci, b, last);
            if (b + 128 >= endi || (sorted && lv == -1)) donei = true;
        }
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) {
        to += __shfl_xor_sync(0xFFFFFFFFu, to, s);
        ti += __shfl_xor_sync(0xFFFFFFFFu, ti, s);
    }
    if (lane == 0) {
        if (to) atomicAdd(&bo[hi - lo], to);
        if (ti) atomicAdd(&bi[hi - lo], ti);
    }
    return entries;
}

// Converged warp: each lane pushes items_a[r] for bits r of ma and items_b[r]
// for bits r of mb (r < 4), one reservation for the warp.
__device__ __forceinline__ void tq_push_warp_mask8(EngineCtl* c, TicketQueue q, unsigned ma, const uint32_t items_a[4],
                                                   unsigned mb, const uint32_t items_b[4]) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned cnt = __popc(ma) + __popc(mb);
    unsigned x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    const unsigned total = __shfl_sync(0xFFFFFFFFu, x, 31);
    if (total == 0) return;
    unsigned base = 0;
    if (lane == 0) {
        atomicAdd(&c->outstanding, (int)total);
        base = atomicAdd(&c->t_tail, total);
    }
    base = __shfl_sync(0xFFFFFFFFu, base, 0) + (x - cnt);
    if (cnt) __threadfence();
#pragma unroll
    for (unsigned r = 0; r < 4; ++r)
        if (ma & (1u << r)) *(volatile unsigned long long*)&q.slots[(base + __popc(ma & ((1u << r) - 1u))) & q.mask] =
            (unsigned long long)items_a[r];
    base += __popc(ma);
#pragma unroll
    for (unsigned r = 0; r < 4; ++r)
        if (mb & (1u << r)) *(volatile unsigned long long*)&q.slots[(base + __popc(mb & ((1u << r) - 1u))) & q.mask] =
            (unsigned long long)items_b[r];
}

// recount_pass over both lists at once with 16-byte id loads: counts the
// neighbours with value >= nv into *cnt_o / *cnt_i (this lane's share) and
// takes x's support away from the neighbours whose level lies in (nv, cap]
// (out-neighbours lose a unit of cnt_in, in-neighbours one of cnt_out); a
// step's counter decrements are all issued before any result is used.
// Stops like hist_pass2v.  Returns the entries read.
__device__ __forceinline__ int recount_pass2v(const Trans2Params& p, EngineCtl* c, uint32_t oo, int no, uint32_t io,
                                              int ni, int nv, int cap, int j, int* cnt_o, int* cnt_i,
                                              uint32_t* keep) {
    const unsigned lane = threadIdx.x & 31u;
    const int so = (int)(oo & 3u), si = (int)(io & 3u), endo = so + no, endi = si + ni;
    int entries = 0;
    bool doneo = no <= 0, donei = ni <= 0;
    for (int b = 0; !(doneo && donei); b += 128) {
        uint32_t uo[4], ui[4];
        load_ids4(p.out_nbr, oo, endo, b, !doneo, uo);
        load_ids4(p.in_nbr, io, endi, b, !donei, ui);
        const int t0 = b + 4 * (int)lane;
        int co[4], ci[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int t = t0 + q;
            co[q] = (!doneo && t >= so && t < endo) ? ld_vol(&p.cur[uo[q]]) : -1;
            ci[q] = (!donei && t >= si && t < endi) ? ld_vol(&p.cur[ui[q]]) : -1;
        }
        int oldo[4], oldi[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            *cnt_o += (co[q] >= nv);
            *cnt_i += (ci[q] >= nv);
            oldo[q] = (co[q] > nv && co[q] <= cap) ? atomicSub(&p.cnt_in[uo[q]], 1) : 0x7FFFFFFF;
            oldi[q] = (ci[q] > nv && ci[q] <= cap) ? atomicSub(&p.cnt_out[ui[q]], 1) : 0x7FFFFFFF;
        }
        unsigned ro = 0, ri = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (oldo[q] != 0x7FFFFFFF && oldo[q] - 1 < j && mark_request(&p.mark[uo[q]], c)) ro |= 1u << q;
            if (oldi[q] != 0x7FFFFFFF && oldi[q] - 1 < ci[q] && mark_request(&p.mark[ui[q]], c)) ri |= 1u << q;
        }
        keep_one(c, keep, &ro, uo);
        keep_one(c, keep, &ri, ui);
        tq_push_warp_mask8(c, p.q, ro, uo, ri, ui);
        if (!doneo) {
            const int last = min(b + 127, endo - 1);
            entries += last + 1 - max(b, so);
            const int lv = last_value(co, b, last);
            if (b + 128 >= endo || (p.sorted && lv == -1)) doneo = true;
        }
        if (!donei) {
            const int last = min(b + 127, endi - 1);
            entries += last + 1 - max(b, si);
            const int lv = last_value(ci, b, last);
            if (b + 128 >= endi || (p.sorted && lv == -1)) donei = true;
        }
    }
    return entries;
}

#ifndef DC_TRANS2_MIN_BLOCKS
#define DC_TRANS2_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kThreads, DC_TRANS2_MIN_BLOCKS) k_trans2(Trans2Params p) {
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const unsigned gwarp = blockIdx.x * kWarpsPerBlock + wib;
    const unsigned nwarps = gridDim.x * kWarpsPerBlock;
    EngineCtl* c = p.ctl;
    __shared__ int s_ho[kWarpsPerBlock][kWin];
    __shared__ int s_hi[kWarpsPerBlock][kWin];
    int* ho = s_ho[wib];
    int* hi_ = s_hi[wib];
    TransHook hook{gridDim.x, p.Kstop, p.K0};
    unsigned long long my_evals = 0, my_drops = 0, my_entries = 0;
    unsigned ticket = kNoTicket;
    __shared__ unsigned s_prod;
    if (threadIdx.x == 0) s_prod = 0;
    if (!grid_sync_hook(c, hook)) return;

    int jprev = p.preleft ? p.K0 : 0;  // row currently held in cur
    bool seed_out = p.preleft != 0;
    for (;;) {
        const int j = ld_vol(&c->level);
        if (j > p.Kstop) break;
        // rows jprev+1 .. j-1 equal row jprev; vertices with kmax in
        // [jprev, j-1] leave now (all but those with kmax == j-1 have value 0)
        const uint32_t vj = p.ck[j], vprev = p.ck[jprev];
        // ---- vertices leaving C_j: value -1; neighbours they supported lose one count
        int lmin = 0x7FFFFFFF;  // bound on the next row that can need work (see hook)
        for (uint32_t i = vj + gwarp; i < vprev; i += nwarps) {
            uint32_t x = p.order ? p.order[i] : i;
            int a = ld_vol(&p.cur[x]);
            __syncwarp();
            if (lane == 0) {
                atomicExch(&p.cur[x], -1);
                __threadfence();
            }
            __syncwarp();
            if (a < 1) continue;
            __threadfence();
            uint32_t o = p.out_off[x];
            int n = p.out_len[x];
            for (int b = 0; b < n; b += 32) {
                bool req = false;
                uint32_t z = 0;
                int cz = -1;
                if (b + (int)lane < n) {
                    z = p.out_nbr[o + b + lane];
                    cz = ld_vol(&p.cur[z]);
                    if (cz >= 1 && cz <= a) {
                        int old = atomicSub(&p.cnt_in[z], 1);
                        if (old - 1 < j) req = mark_request(&p.mark[z], c);
                        else lmin = min(lmin, min(old - 1, p.kmax[z]) + 1);
                    }
                }
                tq_push_warp(c, p.q, req, z);
                int last = min(31, n - 1 - b);
                if (p.sorted && __shfl_sync(0xFFFFFFFFu, cz, last) == -1) break;
            }
            o = p.in_off[x];
            n = p.in_len[x];
            for (int b = 0; b < n; b += 32) {
                bool req = false;
                uint32_t y = 0;
                int cy = -1;
                if (b + (int)lane < n) {
                    y = p.in_nbr[o + b + lane];
                    cy = ld_vol(&p.cur[y]);
                    if (cy >= 1 && cy <= a) {
                        int old = atomicSub(&p.cnt_out[y], 1);
                        req = (old - 1 < cy) && mark_request(&p.mark[y], c);
                    }
                }
                tq_push_warp(c, p.q, req, y);
                int last = min(31, n - 1 - b);
                if (p.sorted && __shfl_sync(0xFFFFFFFFu, cy, last) == -1) break;
            }
        }
#pragma unroll
        for (int s = 16; s; s >>= 1) lmin = min(lmin, __shfl_xor_sync(0xFFFFFFFFu, lmin, s));
        if (lane == 0 && lmin != 0x7FFFFFFF) atomicMin(&c->next_min, lmin);
        // ---- seeds: members whose in-count at their own level is below j;
        // the least min(cnt_in, kmax) + 1 of the others bounds the next row
        // that can need work
        int jmin = 0x7FFFFFFF;
        for (uint32_t base = gwarp * 32; base < vj; base += nwarps * 32) {
            uint32_t i = base + lane;
            bool req = false;
            uint32_t v = 0;
            if (i < vj) {
                v = p.order ? p.order[i] : i;
                const int cv = ld_vol(&p.cur[v]);
                if (cv >= 1) {
                    int ci = ld_vol(&p.cnt_in[v]);
                    if (ci < j || (seed_out && ld_vol(&p.cnt_out[v]) < cv)) req = mark_request(&p.mark[v], c);
                    else jmin = min(jmin, min(ci, p.kmax[v]) + 1);
                }
            }
            tq_push_warp(c, p.q, req, v);
        }
#pragma unroll
        for (int s = 16; s; s >>= 1) jmin = min(jmin, __shfl_xor_sync(0xFFFFFFFFu, jmin, s));
        if (lane == 0 && jmin != 0x7FFFFFFF) atomicMin(&c->next_min, jmin);
        block_producer_done(c, &s_prod);

        // ---- drain: the warp's kept item first, else the queue; finished
        // items are counted off in batches (before the warp waits)
        unsigned long long item;
        uint32_t keep = kNoKeep;
        unsigned done_pending = 0;
        for (;;) {
            if (keep != kNoKeep) {
                item = keep;
                keep = kNoKeep;
            } else if (!tq_take_warp_lazy(c, p.q, &ticket, &item, &done_pending)) {
                break;
            }
            const uint32_t x = (uint32_t)item;
            if (lane == 0) {
                atomicExch(&p.mark[x], 2u);
                __threadfence();
            }
            __syncwarp();
            const int cap = ld_vol(&p.cur[x]);
            if (p.kmax[x] < j || cap < 1) {
                if (lane == 0) {
                    atomicExch(&p.mark[x], 0u);
                    ++done_pending;
                }
                continue;
            }
            int s0o = 0, s0i = 0;
            if (lane == 0) {
                s0o = ld_vol(&p.cnt_out[x]);
                s0i = ld_vol(&p.cnt_in[x]);
            }
            __threadfence();
            const uint32_t oo = p.out_off[x], io = p.in_off[x];
            const unsigned long long ev_entries0 = my_entries;
            // ---- new value from windowed histograms
            int carry_o = 0, carry_i = 0, hi = cap, nv = -1, c_o = 0, c_i = 0;
            bool first = true;
            for (;;) {
                int lo = max(0, hi - (kWin - 1));
                ho[lane] = 0;
                ho[lane + 32] = 0;
                hi_[lane] = 0;
                hi_[lane + 32] = 0;
                __syncwarp();
                my_entries += hist_pass2v(p.cur, p.out_nbr, oo, p.out_len[x], p.in_nbr, io, p.in_len[x], lo, hi, first,
                                          p.sorted != 0, ho, hi_);
                __syncwarp();
                int b0 = 2 * lane, b1 = 2 * lane + 1;
                int o0 = ho[b0], o1 = ho[b1], i0 = hi_[b0], i1 = hi_[b1];
                int po = o0 + o1, pi = i0 + i1;
                int so = po, si = pi;
#pragma unroll
                for (int s = 1; s < 32; s <<= 1) {
                    int yo = __shfl_down_sync(0xFFFFFFFFu, so, s);
                    int yi = __shfl_down_sync(0xFFFFFFFFu, si, s);
                    if (lane + s < 32) {
                        so += yo;
                        si += yi;
                    }
                }
                int cum_o1 = carry_o + (so - po) + o1, cum_i1 = carry_i + (si - pi) + i1;
                int cum_o0 = cum_o1 + o0, cum_i0 = cum_i1 + i0;
                int L0 = lo + b0, L1 = lo + b1;
                bool ok1 = (L1 <= hi) && cum_o1 >= L1 && cum_i1 >= j;
                bool ok0 = (L0 <= hi) && cum_o0 >= L0 && cum_i0 >= j;
                unsigned m1 = __ballot_sync(0xFFFFFFFFu, ok1), m0 = __ballot_sync(0xFFFFFFFFu, ok0);
                int t1 = m1 ? 31 - __clz(m1) : -1, t0 = m0 ? 31 - __clz(m0) : -1;
                int best = -1, bt = 0, bodd = 0;
                if (t1 >= 0) {
                    best = lo + 2 * t1 + 1;
                    bt = t1;
                    bodd = 1;
                }
                if (t0 >= 0 && lo + 2 * t0 > best) {
                    best = lo + 2 * t0;
                    bt = t0;
                    bodd = 0;
                }
                if (best >= 0) {
                    int xo = bodd ? cum_o1 : cum_o0, xi = bodd ? cum_i1 : cum_i0;
                    c_o = __shfl_sync(0xFFFFFFFFu, xo, bt);
                    c_i = __shfl_sync(0xFFFFFFFFu, xi, bt);
                    nv = best;
                    break;
                }
                carry_o += __shfl_sync(0xFFFFFFFFu, so, 0);
                carry_i += __shfl_sync(0xFFFFFFFFu, si, 0);
                first = false;
                if (lo == 0) {  // unreachable for members of C_j
                    nv = 0;
                    c_o = carry_o;
                    c_i = carry_i;
                    break;
                }
                hi = lo - 1;
                __syncwarp();
            }
            ++my_evals;
            if (c->trace && lane == 0) {
                int st = ld_vol(&c->step);
                if (st >= 0 && (unsigned)st < c->trace_cap)
                    atomicMax(&c->trace[8 * st + 7], (unsigned long long)(my_entries - ev_entries0));
            }
            if (nv < cap) {
                ++my_drops;
                if (lane == 0) {
                    atomicExch(&p.cur[x], nv);
                    __threadfence();
                    if (p.stamp[x] != j) {
                        unsigned long long li = atomicAdd(&c->log_count, 1u);
                        if (li < p.log_cap) {
                            p.stamp[x] = j;
                            p.logidx[x] = (uint32_t)li;
                            p.log_v[li] = x;
                            p.log_k[li] = j;
                            p.log_l[li] = nv;
                        } else {
                            set_dev_error(c, DC_DEV_ERR_CAPACITY, 20);
                        }
                    } else {
                        p.log_l[p.logidx[x]] = nv;
                    }
                }
                __syncwarp();
                __threadfence();
                // recount at nv after the write, and take x's support away
                // from neighbours whose level lies in (nv, cap]
                c_o = 0;
                c_i = 0;
                // out-neighbours z hold x in cnt_in; in-neighbours y hold x in cnt_out
                my_entries += recount_pass2v(p, c, oo, p.out_len[x], io, p.in_len[x], nv, cap, j, &c_o, &c_i, &keep);
#pragma unroll
                for (int s = 16; s; s >>= 1) {
                    c_o += __shfl_xor_sync(0xFFFFFFFFu, c_o, s);
                    c_i += __shfl_xor_sync(0xFFFFFFFFu, c_i, s);
                }
            }
            bool requeue = false;
            if (lane == 0) {
                int no = atomicAdd(&p.cnt_out[x], c_o - s0o) + (c_o - s0o);
                int ni = atomicAdd(&p.cnt_in[x], c_i - s0i) + (c_i - s0i);
                bool stable = nv < 1 || (no >= nv && ni >= j);
                __threadfence();
                if (!stable) {
                    atomicExch(&p.mark[x], 1u);
                    requeue = true;
                } else {
                    unsigned o = atomicCAS(&p.mark[x], 2u, 0u);
                    if (o == 3u) {
                        atomicExch(&p.mark[x], 1u);
                        requeue = true;
                    }
                }
            }
            tq_push_warp(c, p.q, requeue, x);
            if (lane == 0) ++done_pending;
        }
        jprev = j;
        seed_out = false;
        if (!grid_sync_hook(c, hook)) break;
    }
    if (lane == 0) {
        atomicAdd(&c->evals, my_evals);
        atomicAdd(&c->drops, my_drops);
        atomicAdd(&c->edges_scanned, my_entries);
    }
}

// ---------------------------------------------------------------------------
// adjacency lists ordered by neighbour kmax, descending
// ---------------------------------------------------------------------------
// With every list in this order, the neighbours inside C_j = {kmax >= j}
// form a prefix of the list, so row-to-row evaluations read only that
// prefix.  Short lists: one thread, insertion sort.  Medium lists: one block,
// bitonic sort of (kmax, id) pairs in shared memory.  Long lists: one block,
// counting sort by kmax through a scratch copy of the list.
static constexpr int kSortShort = 32;
static constexpr int kSortWarp = 256;
static constexpr int kSortMid = 4096;

// Where the entries of list i come from: the list itself (sorted in place),
// or, when the relabeled graph is built, list order[i] of the handle's graph
// with every entry renamed by pos (copy, rename and sort in one pass).
struct ListSrc {
    const uint32_t* off;
    const uint32_t* nbr;
    const uint32_t* order;  // nullptr: in place
    const uint32_t* pos;
};
__device__ __forceinline__ const uint32_t* src_list(const ListSrc& s, uint32_t i, const uint32_t* own) {
    return s.order ? s.nbr + s.off[s.order[i]] : own;
}
__device__ __forceinline__ uint32_t src_id(const ListSrc& s, uint32_t u) { return s.order ? s.pos[u] : u; }

// Lists of at most kSortShort entries are sorted here, one thread each;
// longer ones are listed for the warp sort (up to kSortWarp), the block
// sort (up to kSortMid) or the counting sort.
__global__ void k_sort_short(uint32_t V, const uint32_t* off, const int32_t* len, uint32_t* nbr, const int32_t* kmax,
                             uint32_t* warp_list, uint32_t* mid_list, uint32_t* big_list, unsigned* cnt, ListSrc src) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        int n = len[v];
        if (n > kSortMid) {
            big_list[atomicAdd(&cnt[2], 1u)] = (uint32_t)v;
            continue;
        }
        if (n > kSortWarp) {
            mid_list[atomicAdd(&cnt[1], 1u)] = (uint32_t)v;
            continue;
        }
        if (n > kSortShort) {
            warp_list[atomicAdd(&cnt[0], 1u)] = (uint32_t)v;
            continue;
        }
        uint32_t* a = nbr + off[v];
        const uint32_t* in = src_list(src, (uint32_t)v, a);
        if (n < 2) {
            if (n == 1 && src.order) a[0] = src_id(src, in[0]);
            continue;
        }
        uint32_t ids[kSortShort];
        int ks[kSortShort];
        for (int i = 0; i < n; ++i) {
            ids[i] = src_id(src, in[i]);
            ks[i] = kmax[ids[i]];
        }
        for (int i = 1; i < n; ++i) {
            uint32_t x = ids[i];
            int kx = ks[i];
            int jj = i - 1;
            while (jj >= 0 && ks[jj] < kx) {
                ids[jj + 1] = ids[jj];
                ks[jj + 1] = ks[jj];
                --jj;
            }
            ids[jj + 1] = x;
            ks[jj + 1] = kx;
        }
        for (int i = 0; i < n; ++i) a[i] = ids[i];
    }
}

// One warp per list of kSortShort+1 .. kSortWarp entries: the list and its
// neighbours' kmax go to the warp's shared buffer, every entry's place is its
// rank (entries with a larger kmax, or an equal kmax and a smaller index, go
// before it), and the entries are written back at their places.  The list
// count is read on the device (no host round trip).
constexpr int kSortWarpThreads = 256;
// Lane-strided entries i = lane + 32 t, t < T: rank among the n staged
// entries, written to a[rank].  Staged keys are (kmax << 8) | (255 - index),
// all distinct, so the rank (kmax descending, index ascending on ties) is the
// number of larger keys.
template <int T>
__device__ __forceinline__ void warp_rank_place(const uint32_t* ids, const uint32_t* ks, int n, uint32_t* a) {
    const unsigned lane = threadIdx.x & 31u;
    uint32_t mk[T];
    int rank[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const int i = (int)lane + 32 * t;
        mk[t] = i < n ? ks[i] : 0xFFFFFFFFu;
        rank[t] = 0;
    }
    for (int j = 0; j < n; ++j) {
        const uint32_t kj = ks[j];
#pragma unroll
        for (int t = 0; t < T; ++t) rank[t] += kj > mk[t];
    }
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const int i = (int)lane + 32 * t;
        if (i < n) a[rank[t]] = ids[i];
    }
}
__global__ void __launch_bounds__(kSortWarpThreads) k_sort_warp(const uint32_t* off, const int32_t* len,
                                                                 uint32_t* nbr, const int32_t* kmax,
                                                                 const uint32_t* list, const unsigned* n_list,
                                                                 ListSrc src) {
    constexpr int kW = kSortWarpThreads / 32;
    static_assert(kSortWarp <= 256, "index part of the staged keys is 8 bits");
    __shared__ uint32_t s_id[kW][kSortWarp];
    __shared__ uint32_t s_k[kW][kSortWarp];
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    const unsigned nl = *n_list;
    for (unsigned li = blockIdx.x * kW + w; li < nl; li += gridDim.x * kW) {
        const uint32_t v = list[li];
        const int n = len[v];
        uint32_t* a = nbr + off[v];
        const uint32_t* in = src_list(src, v, a);
        for (int i = lane; i < n; i += 32) {
            const uint32_t u = src_id(src, in[i]);
            s_id[w][i] = u;
            s_k[w][i] = ((uint32_t)kmax[u] << 8) | (uint32_t)(255 - i);
        }
        __syncwarp();
        switch ((n + 31) >> 5) {  // chunks of 32 entries (uniform over the warp)
            case 1: warp_rank_place<1>(s_id[w], s_k[w], n, a); break;
            case 2: warp_rank_place<2>(s_id[w], s_k[w], n, a); break;
            case 3: warp_rank_place<3>(s_id[w], s_k[w], n, a); break;
            case 4: warp_rank_place<4>(s_id[w], s_k[w], n, a); break;
            case 5: warp_rank_place<5>(s_id[w], s_k[w], n, a); break;
            case 6: warp_rank_place<6>(s_id[w], s_k[w], n, a); break;
            case 7: warp_rank_place<7>(s_id[w], s_k[w], n, a); break;
            default: warp_rank_place<8>(s_id[w], s_k[w], n, a); break;
        }
        __syncwarp();
    }
}

// One block per list of kSortWarp+1 .. kSortMid entries: a counting sort by
// neighbour kmax in shared memory (K + 1 bins, the list staged in shared
// memory), written back in place.  Entries of equal kmax keep no particular
// order; only the kmax order matters to the readers.  Dynamic shared memory:
// 4 (K + 1) + 8 kSortMid bytes.
__global__ void k_sort_mid(const uint32_t* off, const int32_t* len, uint32_t* nbr, const int32_t* kmax, int K,
                           const uint32_t* list, unsigned n_list, ListSrc src) {
    extern __shared__ unsigned s_mid[];
    unsigned* bins = s_mid;                   // K + 1
    uint32_t* ids = s_mid + (K + 1);          // kSortMid
    int* ks = (int*)(ids + kSortMid);         // kSortMid
    for (unsigned li = blockIdx.x; li < n_list; li += gridDim.x) {
        const uint32_t v = list[li];
        const int n = len[v];
        uint32_t* a = nbr + off[v];
        const uint32_t* in = src_list(src, v, a);
        for (int i = threadIdx.x; i <= K; i += blockDim.x) bins[i] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t u = src_id(src, in[i]);
            const int k = kmax[u];
            ids[i] = u;
            ks[i] = k;
            atomicAdd(&bins[K - k], 1u);
        }
        __syncthreads();
        unsigned long long carry = 0;
        for (int b0 = 0; b0 <= K; b0 += blockDim.x) {
            const int b = b0 + threadIdx.x;
            const unsigned long long x = b <= K ? bins[b] : 0ull;
            unsigned long long tot;
            const unsigned long long ex = block_excl_scan64(x, &tot);
            if (b <= K) bins[b] = (unsigned)(ex + carry);
            carry += tot;
            __syncthreads();
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) a[atomicAdd(&bins[K - ks[i]], 1u)] = ids[i];
        __syncthreads();
    }
}

// bins = K + 1 counters in shared memory (K < kSortBigBins)
static constexpr int kSortBigBins = 11264;
__global__ void k_sort_big(const uint32_t* off, const int32_t* len, uint32_t* nbr, uint32_t* tmp, const int32_t* kmax,
                           int K, const uint32_t* list, unsigned n_list, ListSrc src) {
    __shared__ unsigned bins[kSortBigBins];
    for (unsigned li = blockIdx.x; li < n_list; li += gridDim.x) {
        uint32_t v = list[li];
        const int n = len[v];
        uint32_t* a = nbr + off[v];
        // in place: staged through tmp; from a source list: straight into a
        uint32_t* t = src.order ? a : tmp + off[v];
        const uint32_t* in = src_list(src, v, a);
        for (int i = threadIdx.x; i <= K; i += blockDim.x) bins[i] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&bins[K - kmax[src_id(src, in[i])]], 1u);
        __syncthreads();
        // exclusive scan of bins (K+1 values), chunked by blockDim
        unsigned long long carry = 0;
        for (int b0 = 0; b0 <= K; b0 += blockDim.x) {
            int b = b0 + threadIdx.x;
            unsigned long long x = b <= K ? bins[b] : 0ull;
            unsigned long long tot;
            unsigned long long ex = block_excl_scan64(x, &tot);
            if (b <= K) bins[b] = (unsigned)(ex + carry);
            carry += tot;
            __syncthreads();
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            uint32_t u = src_id(src, in[i]);
            unsigned pos = atomicAdd(&bins[K - kmax[u]], 1u);
            t[pos] = u;
        }
        __syncthreads();
        if (!src.order)
            for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = t[i];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// order by kmax, skyline assembly, expansion
// ---------------------------------------------------------------------------
// Counts per kmax value.  Most vertices share a few small values, so the
// counts go to per-block shared bins first (when kmax + 1 <= kHistShared).
constexpr int kHistShared = 8192;
__global__ void k_kmax_hist(uint32_t V, const int32_t* kmax, uint32_t* hist, int32_t K) {
    extern __shared__ uint32_t sh[];
    const bool shared = K + 1 <= kHistShared;
    if (shared)
        for (int i = threadIdx.x; i <= K; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(shared ? &sh[kmax[v]] : &hist[kmax[v]], 1u);
    __syncthreads();
    if (shared)
        for (int i = threadIdx.x; i <= K; i += blockDim.x)
            if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// w[k] += in + out degree of every vertex with kmax == k (shared-memory
// bins when the range fits, else global atomics)
__global__ void k_kmax_degree_hist(uint32_t V, const int32_t* kmax, const int32_t* in_len, const int32_t* out_len,
                                   int32_t K, unsigned long long* w) {
    extern __shared__ unsigned long long sw[];
    const bool shared = K + 1 <= 4096;
    if (shared)
        for (int i = threadIdx.x; i <= K; i += blockDim.x) sw[i] = 0;
    __syncthreads();
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long dgr = (unsigned long long)(in_len[v] + out_len[v]);
        if (shared) atomicAdd(&sw[kmax[v]], dgr);
        else atomicAdd(&w[kmax[v]], dgr);
    }
    __syncthreads();
    if (shared)
        for (int i = threadIdx.x; i <= K; i += blockDim.x)
            if (sw[i]) atomicAdd(&w[i], sw[i]);
}

// cursor[k] = first position of bucket k in descending-kmax order
// Warp-aggregated: lanes holding the same kmax take their positions with one
// atomic (the leader's) instead of one each.
__global__ void k_order_scatter(uint32_t V, const int32_t* kmax, uint32_t* cursor, uint32_t* order) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x) & ~31ull; base < V; base += stride) {
        const uint64_t v = base + (threadIdx.x & ~31u) % blockDim.x + lane;
        const bool ok = v < V;
        const int key = ok ? kmax[v] : -1;
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
        const unsigned leader = __ffs(peers) - 1;
        unsigned p0 = 0;
        if (ok && lane == leader) p0 = atomicAdd(&cursor[key], (unsigned)__popc(peers));
        p0 = __shfl_sync(0xFFFFFFFFu, p0, leader);
        if (ok) order[p0 + __popc(peers & ((1u << lane) - 1u))] = (uint32_t)v;
    }
}

// corner bound per vertex: min(kmax, row0) + 1
__global__ void k_corner_bound(uint32_t V, const int32_t* kmax, const int32_t* row0, unsigned long long* acc) {
    unsigned long long s = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        s += (unsigned long long)min(kmax[v], row0[v]);
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if ((threadIdx.x & 31u) == 0) atomicAdd(acc, s);
}

// Row ranges of the segments of a split run of rows.
struct SegBounds {
    int32_t lo[kMaxRowSegments], hi[kMaxRowSegments];
    int n;
};
// Corner bounds per segment: acc[i] = corners of rows lo[i]..hi[i] (a
// vertex's value drops at least one per corner, so it has at most
// min(rows it belongs to, row 0 value) of them; the first corner of a
// segment that starts from row 0 is one of them).
__global__ void k_corner_bounds(uint32_t V, const int32_t* kmax, const int32_t* row0, SegBounds b,
                                unsigned long long* acc) {
    unsigned long long t[kMaxRowSegments] = {};
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t km = kmax[v], r0 = row0[v];
#pragma unroll
        for (int i = 0; i < kMaxRowSegments; ++i)
            if (i < b.n) t[i] += (unsigned long long)max(0, min(min(km, b.hi[i]) - b.lo[i] + 1, r0));
    }
#pragma unroll
    for (int i = 0; i < kMaxRowSegments; ++i) {
#pragma unroll
        for (int o = 16; o; o >>= 1) t[i] += __shfl_xor_sync(0xFFFFFFFFu, t[i], o);
        if ((threadIdx.x & 31u) == 0 && i < b.n && t[i]) atomicAdd(&acc[i], t[i]);
    }
}

// log entries with a negative row are void (dropped corners)
__global__ void k_sky_count(uint32_t V, uint64_t nlog, const uint32_t* log_v, const int32_t* log_k,
                            unsigned long long* cnt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlog; i += (uint64_t)gridDim.x * blockDim.x)
        if (log_k[i] >= 0) atomicAdd(&cnt[log_v[i]], 1ull);
}
// A row segment that jumped from row 0 to row k logs vertex v at row k
// whenever its value differs from row 0; the corner is void when the value
// equals row k-1's (cur after the previous segment).  Counts the void entries.
__global__ void k_seg_void(uint64_t n, const uint32_t* log_v, int32_t* log_k, const int32_t* log_l, int32_t k,
                           const int32_t* cur, unsigned long long* dropped) {
    unsigned long long t = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (log_k[i] == k && log_l[i] == cur[log_v[i]]) {
            log_k[i] = -1;
            ++t;
        }
#pragma unroll
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
    if ((threadIdx.x & 31u) == 0 && t) atomicAdd(dropped, t);
}
__global__ void k_set_one(uint32_t V, unsigned long long* cnt) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        cnt[v] = 1ull;
}
__global__ void k_sky_fill_row0(uint32_t V, const unsigned long long* off, const int32_t* row0, int32_t* sky_k,
                                int32_t* sky_l, uint32_t* fill) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t o = off[v];
        sky_k[o] = 0;
        sky_l[o] = row0[v];
        fill[v] = 1;
    }
}
__global__ void k_sky_fill_log(uint64_t nlog, const uint32_t* log_v, const int32_t* log_k, const int32_t* log_l,
                               const unsigned long long* off, int32_t* sky_k, int32_t* sky_l, uint32_t* fill) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlog; i += (uint64_t)gridDim.x * blockDim.x) {
        if (log_k[i] < 0) continue;
        uint32_t v = log_v[i];
        uint32_t pos = atomicAdd(&fill[v], 1u);
        sky_k[off[v] + pos] = log_k[i];
        sky_l[off[v] + pos] = log_l[i];
    }
}
// sort each vertex's corners by k (insertion sort; lists are short)
__global__ void k_sky_sort(uint32_t V, const unsigned long long* off, int32_t* sky_k, int32_t* sky_l, uint32_t* off32) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t a = off[v], b = off[v + 1];
        for (uint64_t i = a + 1; i < b; ++i) {
            int kk = sky_k[i], ll = sky_l[i];
            uint64_t jj = i;
            while (jj > a && sky_k[jj - 1] > kk) {
                sky_k[jj] = sky_k[jj - 1];
                sky_l[jj] = sky_l[jj - 1];
                --jj;
            }
            sky_k[jj] = kk;
            sky_l[jj] = ll;
        }
        off32[v] = (uint32_t)a;
        if (v == V - 1) off32[V] = (uint32_t)b;
    }
}

// Dense rows [k0, k0+n): rows[(k-k0)*V + v]
// Four consecutive vertices per thread and one 16-byte streaming store per
// row (V a multiple of 4, so every row starts 16-byte aligned); the output is
// far larger than L2, hence the streaming (evict-first) stores.
__global__ void k_expand4(uint32_t V, uint32_t k0, uint32_t n, const int32_t* kmax, const uint32_t* sky_off,
                          const int32_t* sky_k, const int32_t* sky_l, int32_t* rows) {
    const uint32_t V4 = V / 4;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < V4; t += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t ci[4], b[4];
        int val[4], nextk[4], km[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t v = 4 * (uint32_t)t + q;
            const uint32_t a = sky_off[v];
            b[q] = sky_off[v + 1];
            km[q] = kmax[v];
            uint32_t c = a;
            while (c + 1 < b[q] && (uint32_t)sky_k[c + 1] <= k0) ++c;
            ci[q] = c;
            val[q] = sky_l[c];
            nextk[q] = (c + 1 < b[q]) ? sky_k[c + 1] : 0x7FFFFFFF;
        }
        int4* out = reinterpret_cast<int4*>(rows) + t;
        for (uint32_t r = 0; r < n; ++r) {
            const int k = (int)(k0 + r);
            int o[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                while (k >= nextk[q]) {
                    ++ci[q];
                    val[q] = sky_l[ci[q]];
                    nextk[q] = (ci[q] + 1 < b[q]) ? sky_k[ci[q] + 1] : 0x7FFFFFFF;
                }
                o[q] = (k <= km[q]) ? val[q] : 0;
            }
            __stcs(out + (uint64_t)r * V4, make_int4(o[0], o[1], o[2], o[3]));
        }
    }
}

__global__ void k_expand(uint32_t V, uint32_t k0, uint32_t n, const int32_t* kmax, const uint32_t* sky_off,
                         const int32_t* sky_k, const int32_t* sky_l, int32_t* rows) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t a = sky_off[v], b = sky_off[v + 1];
        int km = kmax[v];
        uint32_t ci = a;
        while (ci + 1 < b && (uint32_t)sky_k[ci + 1] <= k0) ++ci;
        int val = sky_l[ci];
        int nextk = (ci + 1 < b) ? sky_k[ci + 1] : 0x7FFFFFFF;
        for (uint32_t r = 0; r < n; ++r) {
            int k = (int)(k0 + r);
            while (k >= nextk) {
                ++ci;
                val = sky_l[ci];
                nextk = (ci + 1 < b) ? sky_k[ci + 1] : 0x7FFFFFFF;
            }
            rows[(uint64_t)r * V + v] = (k <= km) ? val : 0;
        }
    }
}

// skyline from dense rows (per-row peel method)
__global__ void k_rows_corner_count(uint32_t V, uint32_t K, const int32_t* kmax, const int32_t* rows,
                                    unsigned long long* cnt) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        int km = kmax[v];
        unsigned long long c = 1;
        for (int k = 1; k <= km; ++k) c += rows[(uint64_t)k * V + v] != rows[(uint64_t)(k - 1) * V + v];
        cnt[v] = c;
    }
}
__global__ void k_rows_corner_fill(uint32_t V, const int32_t* kmax, const int32_t* rows, const unsigned long long* off,
                                   int32_t* sky_k, int32_t* sky_l, uint32_t* off32) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        int km = kmax[v];
        uint64_t o = off[v];
        sky_k[o] = 0;
        sky_l[o] = rows[v];
        ++o;
        for (int k = 1; k <= km; ++k) {
            int x = rows[(uint64_t)k * V + v];
            if (x != rows[(uint64_t)(k - 1) * V + v]) {
                sky_k[o] = k;
                sky_l[o] = x;
                ++o;
            }
        }
        off32[v] = (uint32_t)off[v];
        if (v == V - 1) off32[V] = (uint32_t)off[V];
    }
}

__global__ void k_max_reduce(uint64_t n, const int32_t* a, int* out) {
    int m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, a[i]);
#pragma unroll
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31u) == 0) atomicMax(out, m);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int grid_for(dc_graph* h, uint64_t n) {
    uint64_t b = (n + kThreads - 1) / kThreads;
    uint64_t cap = (uint64_t)h->geom.sms * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

int coop_launch(dc_graph* h, const void* fn, void** args, int threads, const char* name) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0);
    if (e != cudaSuccess || per_sm < 1)
        return set_error(DC_ERR_CUDA, "%s: occupancy query failed (%s)", name, cudaGetErrorString(e));
    per_sm = std::min(per_sm, 1024 / threads);
    dim3 grid((unsigned)(per_sm * h->geom.sms)), block((unsigned)threads);
    DC_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
    e = cudaLaunchCooperativeKernel(fn, grid, block, args, 0, h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "%s: cooperative launch failed (%s)", name, cudaGetErrorString(e));
    }
    return DC_OK;
}

int check_ctl(dc_graph* h, EngineCtl* hc, const char* what) { return check_ctl_on(h->ctl, h->stream, hc, what); }

int check_ctl_on(EngineCtl* ctl, cudaStream_t st, EngineCtl* hc, const char* what) {
    DC_CUDA(cudaMemcpyAsync(hc, ctl, sizeof(EngineCtl), cudaMemcpyDeviceToHost, st));
    DC_CUDA(cudaStreamSynchronize(st));
    if (hc->error) {
        if (hc->error & DC_DEV_ERR_TIMEOUT)
            return set_error(DC_ERR_TIMEOUT, "%s: bounded device wait expired (site %u)", what, hc->err_where);
        if (hc->error & DC_DEV_ERR_BADID) return set_error(DC_ERR_INVALID, "%s: vertex id out of range", what);
        if (hc->error & DC_DEV_ERR_CAPACITY) return set_error(DC_ERR_CAPACITY, "%s: device buffer capacity exceeded", what);
        return set_error(DC_ERR_CUDA, "%s: device error 0x%x (site %u)", what, hc->error, hc->err_where);
    }
    return DC_OK;
}

int init_handle(dc_graph* h) {
    DC_CUDA(cudaGetDevice(&h->device));
    // two attributes, not the whole property set (cudaGetDeviceProperties is
    // slow, and every handle pays this)
    int coop = 0, sms = 0;
    DC_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device));
    DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    if (!coop) return set_error(DC_ERR_NO_DEVICE, "device lacks cooperative launch");
    h->geom.sms = sms;
    h->geom.threads = kThreads;
    DC_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    // Freed blocks stay in the device's default pool for reuse instead of
    // going back to the driver at every synchronisation.
    cudaMemPool_t pool;
    DC_CUDA(cudaDeviceGetDefaultMemPool(&pool, h->device));
    uint64_t keep = ~0ull;
    DC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    if (dmalloc(h->stream, &h->ctl, 1)) return DC_ERR_NOMEM;
    for (auto& e : h->ev) DC_CUDA(cudaEventCreate(&e));
    return DC_OK;
}

void free_graph_arrays(DevGraph& g, cudaStream_t st) {
    dfree(st, g.out_off);
    dfree(st, g.out_len);
    dfree(st, g.out_nbr_alloc);
    g.out_nbr = nullptr;
    dfree(st, g.in_off);
    dfree(st, g.in_len);
    dfree(st, g.in_nbr_alloc);
    g.in_nbr = nullptr;
    g.out_cap = g.in_cap = 0;
}

int sky_take_spare(dc_graph* h, int slot, uint64_t n, uint32_t** off, int32_t** k, int32_t** l, uint64_t* cap) {
    Decomp& d = h->d;
    if (d.spare_cap[slot] < n || !d.spare_k[slot]) {
        dfree(h->stream, d.spare_k[slot]);
        dfree(h->stream, d.spare_l[slot]);
        d.spare_cap[slot] = 0;
        const uint64_t want = n + n / 4 + 1;
        if (dmalloc(h->stream, &d.spare_k[slot], want) || dmalloc(h->stream, &d.spare_l[slot], want))
            return DC_ERR_NOMEM;
        d.spare_cap[slot] = want;
    }
    if (!d.spare_off[slot] && dmalloc(h->stream, &d.spare_off[slot], (uint64_t)h->g.V + 1)) return DC_ERR_NOMEM;
    *off = d.spare_off[slot];
    *k = d.spare_k[slot];
    *l = d.spare_l[slot];
    *cap = d.spare_cap[slot];
    d.spare_off[slot] = nullptr;
    d.spare_k[slot] = nullptr;
    d.spare_l[slot] = nullptr;
    d.spare_cap[slot] = 0;
    return DC_OK;
}

void sky_put_spare(dc_graph* h, int slot, uint32_t* off, int32_t* k, int32_t* l, uint64_t cap) {
    Decomp& d = h->d;
    dfree(h->stream, d.spare_off[slot]);
    dfree(h->stream, d.spare_k[slot]);
    dfree(h->stream, d.spare_l[slot]);
    d.spare_off[slot] = off;
    d.spare_k[slot] = k;
    d.spare_l[slot] = l;
    d.spare_cap[slot] = (k && l) ? cap : 0;
}

void free_decomp(Decomp& d, cudaStream_t st) {
    dfree(st, d.kmax_v);
    dfree(st, d.row0);
    dfree(st, d.sky_off);
    dfree(st, d.sky_k);
    dfree(st, d.sky_l);
    dfree(st, d.rows);
    for (int i = 0; i < 2; ++i) {
        dfree(st, d.spare_off[i]);
        dfree(st, d.spare_k[i]);
        dfree(st, d.spare_l[i]);
        d.spare_cap[i] = 0;
    }
    d.rows_cap = 0;
    d.corner_cap = 0;
    d.valid = false;
    d.rows_valid = false;
}

void free_scratch(dc_graph* h) {
    Scratch* s = h->scratch;
    if (!s) return;
    for (RowSegment& g : s->seg) {
        if (g.stream) cudaStreamSynchronize(g.stream);
        dfree(h->stream, g.cur);
        dfree(h->stream, g.cnt_out);
        dfree(h->stream, g.cnt_in);
        dfree(h->stream, g.mark);
        dfree(h->stream, g.stamp);
        dfree(h->stream, g.logidx);
        dfree(h->stream, g.tring);
        dfree(h->stream, g.ctl);
        if (g.stream) cudaStreamDestroy(g.stream);
        for (auto& e : g.ev)
            if (e) cudaEventDestroy(e);
    }
    dfree(h->stream, s->key);
    dfree(h->stream, s->cdeg);
    dfree(h->stream, s->cur);
    dfree(h->stream, s->row0);
    dfree(h->stream, s->mark);
    dfree(h->stream, s->stamp);
    dfree(h->stream, s->logidx);
    dfree(h->stream, s->rem0);
    dfree(h->stream, s->rem1);
    dfree(h->stream, s->order);
    dfree(h->stream, s->ck);
    dfree(h->stream, s->ring);
    dfree(h->stream, s->log_v);
    dfree(h->stream, s->log_k);
    dfree(h->stream, s->log_l);
    dfree(h->stream, s->tmp64);
    dfree(h->stream, s->partial);
    dfree(h->stream, s->cursor);
    dfree(h->stream, s->key2);
    dfree(h->stream, s->cdeg2);
    dfree(h->stream, s->rem2);
    dfree(h->stream, s->rem3);
    dfree(h->stream, s->cnt_out);
    dfree(h->stream, s->tring);
    dfree(h->stream, s->w_out_len);
    dfree(h->stream, s->w_in_len);
    dfree(h->stream, s->w_out_nbr);
    dfree(h->stream, s->w_in_nbr);
    dfree(h->stream, s->kmax_old);
    dfree(h->stream, s->row0_old);
    dfree(h->stream, s->pos);
    dfree(h->stream, s->kmax_r);
    dfree(h->stream, s->row0_r);
    for (int i = 0; i < 2; ++i) {
        dfree(h->stream, s->r_off[i]);
        dfree(h->stream, s->r_len[i]);
        dfree(h->stream, s->r_nbr_alloc[i]);
    }
    delete s;
    h->scratch = nullptr;
}

int ensure_scratch(dc_graph* h, uint32_t V) {
    if (!h->scratch) h->scratch = new Scratch();
    Scratch* s = h->scratch;
    if (s->cap_V >= V && s->key) return DC_OK;
    // release V-sized buffers and reallocate
    dfree(h->stream, s->key); dfree(h->stream, s->cdeg); dfree(h->stream, s->cur); dfree(h->stream, s->row0); dfree(h->stream, s->mark); dfree(h->stream, s->stamp);
    dfree(h->stream, s->logidx); dfree(h->stream, s->rem0); dfree(h->stream, s->rem1); dfree(h->stream, s->order); dfree(h->stream, s->ring); dfree(h->stream, s->tmp64);
    dfree(h->stream, s->partial); dfree(h->stream, s->cursor);
    dfree(h->stream, s->key2); dfree(h->stream, s->cdeg2); dfree(h->stream, s->rem2); dfree(h->stream, s->rem3); dfree(h->stream, s->cnt_out);
    uint64_t n = (uint64_t)V + 1;
    if (dmalloc(h->stream, &s->key, n) || dmalloc(h->stream, &s->cdeg, n) || dmalloc(h->stream, &s->cur, n) || dmalloc(h->stream, &s->row0, n) ||
        dmalloc(h->stream, &s->mark, n) || dmalloc(h->stream, &s->stamp, n) || dmalloc(h->stream, &s->logidx, n) || dmalloc(h->stream, &s->rem0, n) ||
        dmalloc(h->stream, &s->rem1, n) || dmalloc(h->stream, &s->order, n) || dmalloc(h->stream, &s->tmp64, n + 1) ||
        dmalloc(h->stream, &s->partial, (uint64_t)h->geom.sms * 64 + 64) || dmalloc(h->stream, &s->cursor, n + 1) ||
        dmalloc(h->stream, &s->key2, n) || dmalloc(h->stream, &s->cdeg2, n) || dmalloc(h->stream, &s->rem2, n) || dmalloc(h->stream, &s->rem3, n) ||
        dmalloc(h->stream, &s->cnt_out, n))
        return DC_ERR_NOMEM;
    uint64_t need = (uint64_t)V + (uint64_t)h->geom.sms * 64 * 32 + 64;
    uint64_t rc = 1024;
    while (rc < need) rc <<= 1;
    if (dmalloc(h->stream, &s->ring, rc)) return DC_ERR_NOMEM;
    s->ring_mask = (uint32_t)(rc - 1);
    s->cap_V = V;
    return DC_OK;
}

uint64_t device_footprint(const dc_graph* h) {
    const DevGraph& g = h->g;
    const Decomp& d = h->d;
    uint64_t V1 = (uint64_t)g.V + 1;
    uint64_t b = sizeof(EngineCtl);
    if (g.out_off) b += 2 * 4 * (2 * V1) + 4 * (g.out_cap + g.in_cap);
    if (d.kmax_v) b += 4 * (3 * V1) + 8 * d.corner_cap;
    for (int i = 0; i < 2; ++i) b += 8 * d.spare_cap[i] + (d.spare_off[i] ? 4 * V1 : 0);
    b += 4 * d.rows_cap;
    if (const Scratch* s = h->scratch) {
        uint64_t n = (uint64_t)s->cap_V + 1;
        if (s->key) b += 4 * (16 * n + 1) + 8 * (n + 1) + 8 * ((uint64_t)h->geom.sms * 64 + 64) + 4ull * (s->ring_mask + 1ull);
        b += 4ull * s->ck_cap + 12 * s->log_cap + 8 * s->tring_cap;
        b += 4 * (s->w_out_cap + s->w_in_cap);
        if (s->kmax_old) b += 8 * n;
        if (s->pos) b += 4 * 7 * ((uint64_t)s->r_cap_V + 1);     // relabeled graph: ids, kmax, row 0, offsets, lengths
        if (s->r_nbr_alloc[0]) b += 2 * 4 * (s->r_cap + 7);     // its lists
    }
    return b;
}

// Exclusive scan of n u64 values in s->tmp64 (tmp64[n] receives the total).
int scan_tmp64(dc_graph* h, uint64_t n) {
    Scratch* s = h->scratch;
    unsigned long long* data = (unsigned long long*)s->tmp64;
    unsigned long long* part = (unsigned long long*)s->partial;
    void* args[] = {&data, &n, &part, &h->ctl};
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_scan_coop, 256, 0);
    per_sm = std::max(1, std::min(per_sm, 8));
    DC_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
    ++g_launches;
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_scan_coop, dim3(per_sm * h->geom.sms), dim3(256), args,
                                                0, h->stream);
    if (e != cudaSuccess) return set_error(DC_ERR_CUDA, "scan launch failed: %s", cudaGetErrorString(e));
    return DC_OK;
}

static int finish_build(dc_graph* h, uint32_t V, uint64_t E, const uint32_t* d_src, const uint32_t* d_dst) {
    DevGraph& g = h->g;
    Scratch* s = h->scratch;
    // capacities -> offsets (out)
    for (int side = 0; side < 2; ++side) {
        int32_t* len = side == 0 ? g.out_len : g.in_len;
        ++g_launches;
        k_capacity<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, len, h->gap_min, h->gap_div,
                                                               (unsigned long long*)s->tmp64);
        if (int rc = scan_tmp64(h, V)) return rc;
        unsigned long long total = 0;
        DC_CUDA(cudaMemcpyAsync(&total, s->tmp64 + V, sizeof(total), cudaMemcpyDeviceToHost, h->stream));
        DC_CUDA(cudaStreamSynchronize(h->stream));
        if (total >= 0xFFFFFFFFull)
            return set_error(DC_ERR_CAPACITY, "adjacency with slack exceeds 2^32 entries (u32 offsets)");
        uint32_t** off = side == 0 ? &g.out_off : &g.in_off;
        uint32_t** nbr = side == 0 ? &g.out_nbr : &g.in_nbr;
        uint32_t** alloc = side == 0 ? &g.out_nbr_alloc : &g.in_nbr_alloc;
        // the row kernel reads ids in aligned 16-byte groups: the lists
        // start at a 16-byte boundary (three spare entries in front cover
        // any alignment of the allocation) and four spare entries at the end
        // cover the last group of the last list
        if (dmalloc(h->stream, off, (uint64_t)V + 1) || dmalloc(h->stream, alloc, total + 7)) return DC_ERR_NOMEM;
        *nbr = (uint32_t*)(((uintptr_t)*alloc + 15u) & ~(uintptr_t)15u);
        ++g_launches;
        k_off_to_u32<<<grid_for(h, (uint64_t)V + 1), kThreads, 0, h->stream>>>(V, (unsigned long long*)s->tmp64, *off);
        if (side == 0) g.out_cap = total;
        else g.in_cap = total;
    }
    DC_CUDA(cudaMemsetAsync(g.out_len, 0, sizeof(int32_t) * V, h->stream));
    DC_CUDA(cudaMemsetAsync(g.in_len, 0, sizeof(int32_t) * V, h->stream));
    if (E)
        ++g_launches;
        k_scatter_edges<<<grid_for(h, E), kThreads, 0, h->stream>>>(E, d_src, d_dst, g.out_off, g.out_len, g.out_nbr,
                                                                     g.in_off, g.in_len, g.in_nbr);
    DC_CUDA(cudaGetLastError());
    g.V = V;
    g.E = E;
    g.sorted_kmax = false;
    return DC_OK;
}

int build_from_device_edges(dc_graph* h, uint32_t V, uint64_t E, const uint32_t* d_src, const uint32_t* d_dst) {
    free_graph_arrays(h->g, h->stream);
    free_decomp(h->d, h->stream);
    if (int rc = ensure_scratch(h, V)) return rc;
    DevGraph& g = h->g;
    if (dmalloc(h->stream, &g.out_len, (uint64_t)V + 1) || dmalloc(h->stream, &g.in_len, (uint64_t)V + 1)) return DC_ERR_NOMEM;
    DC_CUDA(cudaMemsetAsync(g.out_len, 0, sizeof(int32_t) * ((uint64_t)V + 1), h->stream));
    DC_CUDA(cudaMemsetAsync(g.in_len, 0, sizeof(int32_t) * ((uint64_t)V + 1), h->stream));
    DC_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
    if (E) k_count_degrees<<<grid_for(h, E), kThreads, 0, h->stream>>>(V, E, d_src, d_dst, g.out_len, g.in_len, h->ctl);
    EngineCtl hc;
    if (int rc = check_ctl(h, &hc, "graph build")) return rc;
    return finish_build(h, V, E, d_src, d_dst);
}

__global__ void k_host_csr_len(uint32_t V, const int32_t* deg, int32_t* len) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        len[v] = deg[v];
}

// Expands a CSR with arbitrary per-list slots into an edge list on device.
__global__ void k_csr_to_edges(uint32_t V, const uint32_t* off, const int32_t* len, const unsigned long long* eoff,
                               const uint32_t* nbr, uint32_t* src, uint32_t* dst, int swap) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = gw; v < V; v += nw) {
        uint32_t o = off[v];
        int n = len[v];
        uint64_t e0 = eoff[v];
        for (int i = lane; i < n; i += 32) {
            uint32_t u = nbr[o + i];
            if (!swap) {
                src[e0 + i] = (uint32_t)v;
                dst[e0 + i] = u;
            } else {
                src[e0 + i] = u;
                dst[e0 + i] = (uint32_t)v;
            }
        }
    }
}

int build_from_host_csr(dc_graph* h, uint32_t V, uint64_t E, const int32_t* in_deg, const int32_t* out_deg,
                        const uint32_t* in_off, const uint32_t* out_off, const uint32_t* in_nbr,
                        const uint32_t* out_nbr, uint64_t nbr_len) {
    (void)in_deg;
    (void)in_off;
    (void)in_nbr;
    // The reference binary stores both directions; the out-lists define the
    // edge multiset, so the device rebuilds both sides from them.
    free_graph_arrays(h->g, h->stream);
    free_decomp(h->d, h->stream);
    if (int rc = ensure_scratch(h, V)) return rc;
    uint32_t *d_off = nullptr, *d_nbr = nullptr, *d_src = nullptr, *d_dst = nullptr;
    int32_t* d_deg = nullptr;
    int rc = DC_OK;
    if ((rc = dmalloc(h->stream, &d_off, (uint64_t)V + 1)) || (rc = dmalloc(h->stream, &d_nbr, nbr_len)) || (rc = dmalloc(h->stream, &d_deg, V)) ||
        (rc = dmalloc(h->stream, &d_src, E)) || (rc = dmalloc(h->stream, &d_dst, E))) {
        dfree(h->stream, d_off); dfree(h->stream, d_nbr); dfree(h->stream, d_deg); dfree(h->stream, d_src); dfree(h->stream, d_dst);
        return rc;
    }
    Scratch* s = h->scratch;
    cudaMemcpyAsync(d_off, out_off, sizeof(uint32_t) * ((uint64_t)V + 1), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(d_nbr, out_nbr, sizeof(uint32_t) * nbr_len, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(d_deg, out_deg, sizeof(int32_t) * V, cudaMemcpyHostToDevice, h->stream);
    // edge offsets = exclusive scan of degrees
    std::vector<unsigned long long> eo((size_t)V + 1);
    unsigned long long acc = 0;
    for (uint32_t v = 0; v < V; ++v) {
        eo[v] = acc;
        acc += (unsigned long long)out_deg[v];
    }
    eo[V] = acc;
    if (acc != E) {
        dfree(h->stream, d_off); dfree(h->stream, d_nbr); dfree(h->stream, d_deg); dfree(h->stream, d_src); dfree(h->stream, d_dst);
        return set_error(DC_ERR_INVALID, "binary graph: out-degrees sum to %llu, header says %llu", acc,
                         (unsigned long long)E);
    }
    cudaMemcpyAsync(s->tmp64, eo.data(), sizeof(unsigned long long) * ((size_t)V + 1), cudaMemcpyHostToDevice,
                    h->stream);
    ++g_launches;
    k_csr_to_edges<<<grid_for(h, (uint64_t)V * 32), kThreads, 0, h->stream>>>(
        V, d_off, d_deg, (const unsigned long long*)s->tmp64, d_nbr, d_src, d_dst, 0);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    dfree(h->stream, d_off);
    dfree(h->stream, d_nbr);
    dfree(h->stream, d_deg);
    if (e != cudaSuccess) {
        dfree(h->stream, d_src); dfree(h->stream, d_dst);
        return set_error(DC_ERR_CUDA, "binary graph upload failed: %s", cudaGetErrorString(e));
    }
    rc = build_from_device_edges(h, V, E, d_src, d_dst);
    cudaStreamSynchronize(h->stream);
    dfree(h->stream, d_src);
    dfree(h->stream, d_dst);
    return rc;
}

int ensure_tring(dc_graph* h, uint64_t need) {
    Scratch* s = h->scratch;
    uint64_t cap = 1024;
    while (cap < need) cap <<= 1;
    if (s->tring_cap >= cap && s->tring) return DC_OK;
    dfree(h->stream, s->tring);
    s->tring_cap = 0;
    if (dmalloc(h->stream, &s->tring, cap)) return DC_ERR_NOMEM;
    s->tring_cap = cap;
    DC_CUDA(cudaMemsetAsync(s->tring, 0xFF, sizeof(unsigned long long) * cap, h->stream));
    return DC_OK;
}

// Two 256-thread blocks per SM: measured best or near it from R-MAT 19 to 22
// once the queue counters sit on separate lines (the autotuner refines it).
static constexpr int kDefaultBlocksPerSm = 2;

static int persistent_grid(dc_graph* h, const void* fn, int bps, int* blocks) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0);
    if (e != cudaSuccess || per_sm < 1)
        return set_error(DC_ERR_CUDA, "occupancy query failed (%s)", cudaGetErrorString(e));
    if (bps <= 0) bps = h->blocks_per_sm > 0 ? h->blocks_per_sm : kDefaultBlocksPerSm;
    per_sm = std::min(per_sm, bps);
    *blocks = per_sm * h->geom.sms;
    return DC_OK;
}

// A control block as persistent_launch prepares it (no trace, no test
// hook), written by the device: usable inside a captured CUDA graph.
__global__ void k_ctl_init(EngineCtl* c, unsigned long long wait_ns) {
    uint32_t* w = reinterpret_cast<uint32_t*>(c);
    for (uint32_t i = threadIdx.x; i < sizeof(EngineCtl) / 4; i += blockDim.x) w[i] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        c->step = -1;
        c->wait_ns = wait_ns;
    }
}

int ctl_init_enqueue(dc_graph* h, EngineCtl* ctl, cudaStream_t st) {
    ++g_launches;
    k_ctl_init<<<1, 256, 0, st>>>(ctl, h->wait_ns);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DC_OK : set_error(DC_ERR_CUDA, "control block init: %s", cudaGetErrorString(e));
}

// Capture-safe persistent launch: the control block is initialised by a
// kernel and nothing is waited for (the caller reads the block's status
// later).
int persistent_enqueue(dc_graph* h, const void* fn, void** args, const char* name, EngineCtl* ctl, cudaStream_t st,
                       int bps) {
    int blocks = 0;
    if (int rc = persistent_grid(h, fn, bps, &blocks)) return rc;
    if (int rc = ctl_init_enqueue(h, ctl, st)) return rc;
    ++g_launches;
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kThreads), args, 0, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "%s: cooperative launch failed (%s)", name, cudaGetErrorString(e));
    }
    return DC_OK;
}

// Initialises a control block (on stream st) and launches a persistent
// kernel there without waiting.  The handle's own block carries the trace.
static int persistent_launch(dc_graph* h, const void* fn, void** args, const char* name, EngineCtl* ctl,
                             cudaStream_t st, int bps) {
    int blocks = 0;
    if (int rc = persistent_grid(h, fn, bps, &blocks)) return rc;
    const bool own = ctl == h->ctl;
    EngineCtl* initp = &h->ctl_init;
    for (int i = 0; i < kMaxRowSegments - 1; ++i)
        if (ctl == h->scratch->seg[i].ctl) initp = &h->ctl_init_seg[i];
    EngineCtl& init = *initp;
    memset(&init, 0, sizeof(init));
    init.step = -1;
    init.wait_ns = h->wait_ns;
    if (own) {
        init.trace = h->trace_dev;
        init.trace_cap = h->trace_cap;
        if (h->barrier_fault_block >= 0) {  // one launch only
            init.test_skip_block = h->barrier_fault_block + 1;
            h->barrier_fault_block = -1;
        }
    }
    DC_CUDA(cudaMemcpyAsync(ctl, &init, sizeof(EngineCtl), cudaMemcpyHostToDevice, st));
    if (own && h->trace_dev) DC_CUDA(cudaMemsetAsync(h->trace_dev, 0, 64ull * h->trace_cap, st));
    ++g_launches;
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kThreads), args, 0, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "%s: cooperative launch failed (%s)", name, cudaGetErrorString(e));
    }
    return DC_OK;
}

// Waits for a persistent kernel launched on stream st with control block ctl
// and converts its device status; the handle's own block also delivers the
// trace.  A failed phase may leave items in its ring, which is cleared.
static int finish_persistent(dc_graph* h, EngineCtl* ctl, cudaStream_t st, const char* name, EngineCtl* out) {
    int rc = check_ctl_on(ctl, st, out, name);
    const bool own = ctl == h->ctl;
    if (own && h->trace_dev && h->trace_host) {
        cudaMemcpy(h->trace_host, h->trace_dev, 64ull * h->trace_cap, cudaMemcpyDeviceToHost);
        h->trace_steps = (unsigned)std::max(0, out->step);
        if (h->trace_cb) h->trace_cb(name, h->trace_host, h->trace_steps, h->trace_user);
    }
    if (rc != DC_OK) {
        Scratch* s = h->scratch;
        unsigned long long* ring = s->tring;
        uint64_t cap = s->tring_cap;
        for (const RowSegment& g : s->seg)
            if (ctl == g.ctl) {
                ring = g.tring;
                cap = g.tring_cap;
            }
        cudaMemsetAsync(ring, 0xFF, sizeof(unsigned long long) * cap, st);
        cudaStreamSynchronize(st);
    }
    return rc;
}

// Launches a persistent kernel, waits, and converts its device status.
int run_persistent(dc_graph* h, const void* fn, void** args, const char* name, EngineCtl* out, int bps) {
    if (int rc = persistent_launch(h, fn, args, name, h->ctl, h->stream, bps)) return rc;
    return finish_persistent(h, h->ctl, h->stream, name, out);
}

// State of row segment i + 1 (seg[i]), sized for V vertices.
static int ensure_segment(dc_graph* h, int i, uint32_t V) {
    Scratch* s = h->scratch;
    RowSegment& g = s->seg[i];
    if (!g.stream) {
        DC_CUDA(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
        for (auto& e : g.ev) DC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (!g.ctl && dmalloc(h->stream, &g.ctl, 1)) return DC_ERR_NOMEM;
    if (g.cap_V < V || !g.cur) {
        dfree(h->stream, g.cur);
        dfree(h->stream, g.cnt_out);
        dfree(h->stream, g.cnt_in);
        dfree(h->stream, g.mark);
        dfree(h->stream, g.stamp);
        dfree(h->stream, g.logidx);
        g.cap_V = 0;
        const uint64_t n = (uint64_t)V + 1;
        if (dmalloc(h->stream, &g.cur, n) || dmalloc(h->stream, &g.cnt_out, n) || dmalloc(h->stream, &g.cnt_in, n) ||
            dmalloc(h->stream, &g.mark, n) || dmalloc(h->stream, &g.stamp, n) || dmalloc(h->stream, &g.logidx, n))
            return DC_ERR_NOMEM;
        g.cap_V = V;
    }
    uint64_t need = 2ull * V + (uint64_t)h->geom.sms * 64 + 4096, cap = 1024;
    while (cap < need) cap <<= 1;
    if (g.tring_cap < cap || !g.tring) {
        dfree(h->stream, g.tring);
        g.tring_cap = 0;
        if (dmalloc(h->stream, &g.tring, cap)) return DC_ERR_NOMEM;
        g.tring_cap = cap;
        DC_CUDA(cudaMemsetAsync(g.tring, 0xFF, sizeof(unsigned long long) * cap, h->stream));
    }
    return DC_OK;
}

// Allocates the state of the row segments the handle's cuts ask for, so
// that no later run of rows allocates it (maintenance batches included).
int prepare_row_segments(dc_graph* h) {
    const uint32_t V = h->g.V;
    if (!V) return DC_OK;
    int n = 0;
    while (n < kMaxRowSegments - 1 && h->rows_split[n] > 0) ++n;
    if (!n) return DC_OK;
    if (int rc = ensure_scratch(h, V)) return rc;
    for (int i = 0; i < n; ++i)
        if (int rc = ensure_segment(h, i, V)) return rc;
    DC_CUDA(cudaStreamSynchronize(h->stream));
    return DC_OK;
}

PeelInst make_inst(dc_graph* h, int which, const int32_t* member, int32_t k, int32_t* val, int slot) {
    DevGraph& g = h->g;
    Scratch* s = h->scratch;
    PeelInst I;
    if (which == 0) {
        I.a_off = g.in_off; I.a_len = g.in_len; I.a_nbr = g.in_nbr;
        I.b_off = g.out_off; I.b_len = g.out_len; I.b_nbr = g.out_nbr;
    } else {
        I.a_off = g.out_off; I.a_len = g.out_len; I.a_nbr = g.out_nbr;
        I.b_off = g.in_off; I.b_len = g.in_len; I.b_nbr = g.in_nbr;
    }
    I.member = member;
    I.k = k;
    I.val = val;
    if (slot == 0) {
        I.key = s->key; I.cdeg = s->cdeg; I.rem0 = s->rem0; I.rem1 = s->rem1;
    } else {
        I.key = s->key2; I.cdeg = s->cdeg2; I.rem0 = s->rem2; I.rem1 = s->rem3;
    }
    return I;
}

// Runs one or two peels in one persistent launch; maxv[i] = largest value.
int run_peel2(dc_graph* h, int ninst, const PeelInst* inst, int32_t* maxv) {
    Scratch* s = h->scratch;
    DevGraph& g = h->g;
    const unsigned chunk = h->peel_chunk ? h->peel_chunk : 64;
    uint64_t need = 2ull * g.V + 2ull * (g.out_cap + g.in_cap) / chunk + (uint64_t)h->geom.sms * 64 + 4096;
    if (int rc = ensure_tring(h, need)) return rc;
    Peel2Params p;
    p.V = g.V;
    p.ninst = ninst;
    p.chunk = chunk;
    p.in[0] = inst[0];
    p.in[1] = ninst > 1 ? inst[1] : inst[0];
    p.q.slots = s->tring;
    p.q.mask = (unsigned)(s->tring_cap - 1);
    p.ctl = h->ctl;
    void* args[] = {&p};
    EngineCtl hc;
    if (int rc = run_persistent(h, (const void*)k_peel2, args, "peel", &hc, h->peel_bps)) return rc;
    for (int i = 0; i < ninst; ++i) maxv[i] = hc.maxv[i];
    return DC_OK;
}

int peel_kmax_row0(dc_graph* h, int32_t* kmax, int32_t* lmax) {
    int32_t mv[2] = {0, 0};
    PeelInst I[2] = {make_inst(h, 0, nullptr, 0, h->d.kmax_v, 0), make_inst(h, 1, nullptr, 0, h->scratch->row0, 1)};
    if (int rc = run_peel2(h, 2, I, mv)) return rc;
    *kmax = mv[0];
    *lmax = mv[1];
    return DC_OK;
}

// which: 0 = kmax pass (peel in-degree), 1 = row pass (peel out-degree)
int run_peel(dc_graph* h, int which, const int32_t* member, int32_t k, int32_t* d_val, int32_t* maxval, int sync) {
    (void)sync;
    PeelInst I = make_inst(h, which, member, k, d_val, 0);
    int32_t mv = 0;
    if (int rc = run_peel2(h, 1, &I, &mv)) return rc;
    if (maxval) *maxval = mv;
    return DC_OK;
}

// Skyline from row 0 and the corner logs of the last run of rows: the
// first segment's nlog entries at the log's start and the other segments'
// ranges (h->seg_off / seg_n, voided entries skipped).
int build_skyline_from_log(dc_graph* h, uint64_t nlog) {
    Scratch* s = h->scratch;
    Decomp& d = h->d;
    uint32_t V = h->g.V;
    unsigned long long* cnt = (unsigned long long*)s->tmp64;
    uint64_t lo[kMaxRowSegments], n[kMaxRowSegments];
    int nr = 0;
    uint64_t total = (uint64_t)V;
    if (nlog) {
        lo[nr] = 0;
        n[nr++] = nlog;
        total += nlog;
    }
    for (int i = 0; i < h->nseg_extra; ++i)
        if (h->seg_n[i]) {
            lo[nr] = h->seg_off[i];
            n[nr++] = h->seg_n[i];
            total += h->seg_n[i] - h->seg_void[i];
        }
    ++g_launches;
    k_set_one<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, cnt);
    for (int r = 0; r < nr; ++r) {
        ++g_launches;
        k_sky_count<<<grid_for(h, n[r]), kThreads, 0, h->stream>>>(V, n[r], s->log_v + lo[r], s->log_k + lo[r], cnt);
    }
    if (int rc = scan_tmp64(h, V)) return rc;
    if (d.corner_cap < total || !d.sky_k) {
        // a quarter of headroom: maintenance batches rarely grow it again
        dfree(h->stream, d.sky_k);
        dfree(h->stream, d.sky_l);
        d.corner_cap = 0;
        const uint64_t want = total + total / 4 + 1;
        if (dmalloc(h->stream, &d.sky_k, want) || dmalloc(h->stream, &d.sky_l, want)) return DC_ERR_NOMEM;
        d.corner_cap = want;
    }
    if (!d.sky_off && dmalloc(h->stream, &d.sky_off, (uint64_t)V + 1)) return DC_ERR_NOMEM;
    ++g_launches;
    k_sky_fill_row0<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, cnt, s->row0, d.sky_k, d.sky_l, s->cursor);
    for (int r = 0; r < nr; ++r) {
        ++g_launches;
        k_sky_fill_log<<<grid_for(h, n[r]), kThreads, 0, h->stream>>>(n[r], s->log_v + lo[r], s->log_k + lo[r],
                                                                      s->log_l + lo[r], cnt, d.sky_k, d.sky_l,
                                                                      s->cursor);
    }
    ++g_launches;
    k_sky_sort<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, cnt, d.sky_k, d.sky_l, d.sky_off);
    d.n_corners = total;
    DC_CUDA(cudaGetLastError());
    return DC_OK;
}

static int ensure_rows(dc_graph* h, uint64_t elems) {
    Decomp& d = h->d;
    if (d.rows_cap >= elems && d.rows) return DC_OK;
    dfree(h->stream, d.rows);
    d.rows_cap = 0;
    if (dmalloc(h->stream, &d.rows, elems)) return DC_ERR_NOMEM;
    d.rows_cap = elems;
    return DC_OK;
}

int expand_rows(dc_graph* h, uint32_t k0, uint32_t n, int32_t* d_dst) {
    Decomp& d = h->d;
    if (!d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (n == 0) return DC_OK;
    ++g_launches;
    if (h->g.V % 4 == 0 && ((uintptr_t)d_dst & 15u) == 0)
        k_expand4<<<grid_for(h, h->g.V / 4), kThreads, 0, h->stream>>>(h->g.V, k0, n, d.kmax_v, d.sky_off, d.sky_k,
                                                                         d.sky_l, d_dst);
    else
        k_expand<<<grid_for(h, h->g.V), kThreads, 0, h->stream>>>(h->g.V, k0, n, d.kmax_v, d.sky_off, d.sky_k,
                                                                   d.sky_l, d_dst);
    DC_CUDA(cudaGetLastError());
    return DC_OK;
}

// Orders every adjacency list by neighbour kmax, descending.  *sorted = 0
// when kmax is too large for the long-list counting sort (lists then stay
// in arbitrary order and evaluations read them whole).
// Orders every list of one side by neighbour kmax, descending (kmax[u] of
// each entry u of the graph the lists belong to).  cap = entries the lists'
// array spans (the long-list sort stages through a scratch copy that size).
static int sort_side(dc_graph* h, int32_t K, uint32_t V, const uint32_t* off, const int32_t* len, uint32_t* nbr,
                     uint64_t cap, const int32_t* kmax, int side, ListSrc src) {
    Scratch* s = h->scratch;
    unsigned* cnt = s->cursor;
    DC_CUDA(cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned), h->stream));
    ++g_launches;
    k_sort_short<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, off, len, nbr, kmax, s->rem0, s->rem2, s->rem1, cnt,
                                                              src);
    // most lists go to the warp sort, which reads its count on the device
    ++g_launches;
    k_sort_warp<<<h->geom.sms * 8, kSortWarpThreads, 0, h->stream>>>(off, len, nbr, kmax, s->rem0, &cnt[0], src);
    unsigned hc[3] = {0, 0, 0};
    DC_CUDA(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, h->stream));
    DC_CUDA(cudaStreamSynchronize(h->stream));
    if (hc[1]) {
        const size_t shm = 4ull * (K + 1) + 8ull * kSortMid;
        // the kernel's limit is set to its largest need, the same value on
        // every call: handles sorting on other threads at the same time
        // (the serving loop) must never see it lowered below their launch
        constexpr size_t kMidMax = 4ull * kSortBigBins + 8ull * kSortMid;
        static_assert(kMidMax <= 227ull * 1024, "mid-list sort shared memory");
        DC_CUDA(cudaFuncSetAttribute(k_sort_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMidMax));
        int blocks = (int)std::min<unsigned>(hc[1], (unsigned)h->geom.sms * 8);
        ++g_launches;
        k_sort_mid<<<blocks, 256, shm, h->stream>>>(off, len, nbr, kmax, K, s->rem2, hc[1], src);
    }
    if (hc[2]) {
        uint32_t*& tmp = side == 0 ? s->w_out_nbr : s->w_in_nbr;
        uint64_t& tcap = side == 0 ? s->w_out_cap : s->w_in_cap;
        if (!src.order && (tcap < cap || !tmp)) {  // in place: staging copy of the lists' span
            dfree(h->stream, tmp);
            if (dmalloc(h->stream, &tmp, cap)) return DC_ERR_NOMEM;
            tcap = cap;
        }
        int blocks = (int)std::min<unsigned>(hc[2], (unsigned)h->geom.sms * 2);
        ++g_launches;
        k_sort_big<<<blocks, 512, 0, h->stream>>>(off, len, nbr, tmp, kmax, K, s->rem1, hc[2], src);
    }
    DC_CUDA(cudaGetLastError());
    return DC_OK;
}

// Orders every adjacency list of the graph by neighbour kmax, descending.
// *sorted = 0 when kmax is too large for the long-list counting sort (lists
// then stay in arbitrary order and evaluations read them whole).
static int sort_lists_by_kmax(dc_graph* h, int32_t K, int* sorted) {
    DevGraph& g = h->g;
    *sorted = 0;
    if (g.sorted_kmax) {
        *sorted = 1;
        return DC_OK;
    }
    if (K + 1 > kSortBigBins) return DC_OK;
    for (int side = 0; side < 2; ++side)
        if (int rc = sort_side(h, K, g.V, side == 0 ? g.out_off : g.in_off, side == 0 ? g.out_len : g.in_len,
                               side == 0 ? g.out_nbr : g.in_nbr, side == 0 ? g.out_cap : g.in_cap, h->d.kmax_v, side,
                               ListSrc{nullptr, nullptr, nullptr, nullptr}))
            return rc;
    g.sorted_kmax = true;
    *sorted = 1;
    return DC_OK;
}

// ---------------------------------------------------------------------------
// the graph relabeled in kmax order for the row kernel
// ---------------------------------------------------------------------------
// New id i = position of a vertex in kmax-descending order (s->order), so
// C_k = {new ids < |C_k|} is a prefix of the id space: the row kernel's scans
// of C_k read its state contiguously, and the dense core's state (the
// vertices of the heavy rows) packs into a small range that stays in the
// SMs' caches.  Lists hold new ids, ordered by neighbour kmax.
__global__ void k_relabel_gather(uint32_t V, const uint32_t* order, const int32_t* kmax, const int32_t* row0,
                                 const int32_t* out_len, const int32_t* in_len, uint32_t* pos, int32_t* kmax_r,
                                 int32_t* row0_r, int32_t* len_o, int32_t* len_i) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = order[i];
        pos[v] = (uint32_t)i;
        kmax_r[i] = kmax[v];
        row0_r[i] = row0[v];
        len_o[i] = out_len[v];
        len_i[i] = in_len[v];
    }
}

__global__ void k_len_to_u64e(uint32_t V, const int32_t* len, unsigned long long* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (unsigned long long)len[i];
}

// corner records of the relabeled run back to original ids
__global__ void k_unlabel_log(uint64_t n, const uint32_t* order, uint32_t* log_v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        log_v[i] = order[log_v[i]];
}

// Builds the relabeled graph (s->order must hold the kmax order of the
// current kmax) with its lists sorted by neighbour kmax, plus kmax and row 0
// by new id.
static int build_relabeled(dc_graph* h, int32_t K) {
    DevGraph& g = h->g;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    const uint64_t n = (uint64_t)V + 1;
    if (s->r_cap_V < V || !s->pos) {
        dfree(h->stream, s->pos);
        dfree(h->stream, s->kmax_r);
        dfree(h->stream, s->row0_r);
        for (int i = 0; i < 2; ++i) {
            dfree(h->stream, s->r_off[i]);
            dfree(h->stream, s->r_len[i]);
        }
        s->r_cap_V = 0;
        if (dmalloc(h->stream, &s->pos, n) || dmalloc(h->stream, &s->kmax_r, n) || dmalloc(h->stream, &s->row0_r, n) ||
            dmalloc(h->stream, &s->r_off[0], n) || dmalloc(h->stream, &s->r_off[1], n) ||
            dmalloc(h->stream, &s->r_len[0], n) || dmalloc(h->stream, &s->r_len[1], n))
            return DC_ERR_NOMEM;
        s->r_cap_V = V;
    }
    // list arrays: three spare entries in front for the 16-byte alignment of
    // the array start, four at the end for the last 16-byte id group
    const uint64_t cap = g.E + 8;
    if (s->r_cap < cap || !s->r_nbr_alloc[0]) {
        for (int i = 0; i < 2; ++i) {
            dfree(h->stream, s->r_nbr_alloc[i]);
            s->r_nbr[i] = nullptr;
        }
        s->r_cap = 0;
        const uint64_t want = cap + cap / 8;  // headroom for later, larger graphs of the handle
        for (int i = 0; i < 2; ++i) {
            if (dmalloc(h->stream, &s->r_nbr_alloc[i], want + 7)) return DC_ERR_NOMEM;
            s->r_nbr[i] = (uint32_t*)(((uintptr_t)s->r_nbr_alloc[i] + 15u) & ~(uintptr_t)15u);
        }
        s->r_cap = want;
    }
    ++g_launches;
    k_relabel_gather<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, s->order, h->d.kmax_v, s->row0, g.out_len,
                                                                  g.in_len, s->pos, s->kmax_r, s->row0_r, s->r_len[0],
                                                                  s->r_len[1]);
    for (int side = 0; side < 2; ++side) {
        ++g_launches;
        k_len_to_u64e<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, s->r_len[side], (unsigned long long*)s->tmp64);
        if (int rc = scan_tmp64(h, V)) return rc;
        ++g_launches;
        k_off_to_u32<<<grid_for(h, n), kThreads, 0, h->stream>>>(V, (unsigned long long*)s->tmp64, s->r_off[side]);
    }
    // every relabeled list is read from its original list, renamed and
    // sorted by neighbour kmax in one pass
    for (int side = 0; side < 2; ++side) {
        const ListSrc src{side == 0 ? g.out_off : g.in_off, side == 0 ? g.out_nbr : g.in_nbr, s->order, s->pos};
        if (int rc = sort_side(h, K, V, s->r_off[side], s->r_len[side], s->r_nbr[side], s->r_cap, s->kmax_r, side, src))
            return rc;
    }
    return DC_OK;
}

// Rows 1..Kstop from row 0 (scratch row0) and kmax (d.kmax_v): orders
// vertices by kmax, initialises the support counters and runs the
// row-to-row kernel.  Corners of rows 1..Kstop are left in the scratch log
// (*nlog entries).  allow_sort: order adjacency lists by neighbour kmax
// first (otherwise lists are read whole).
int rows_from_row0(dc_graph* h, int32_t K, int32_t Kstop, bool allow_sort, uint64_t* nlog_out, int32_t K0,
                   bool allow_relabel) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    *nlog_out = 0;
    h->nseg_extra = 0;
    cudaEventRecord(h->ev[2], h->stream);
    if (s->ck_cap < (uint32_t)K + 2) {
        dfree(h->stream, s->ck);
        if (dmalloc(h->stream, &s->ck, (uint64_t)K + 2)) return DC_ERR_NOMEM;
        s->ck_cap = K + 2;
    }
    uint32_t* hist = s->cursor;
    DC_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * ((uint64_t)K + 2), h->stream));
    ++g_launches;
    k_kmax_hist<<<grid_for(h, V), kThreads, K + 1 <= kHistShared ? 4 * (K + 1) : 0, h->stream>>>(V, d.kmax_v, hist, K);
    std::vector<uint32_t> hh((size_t)K + 2), ck((size_t)K + 2), start((size_t)K + 2);
    DC_CUDA(cudaMemcpyAsync(hh.data(), hist, sizeof(uint32_t) * ((size_t)K + 2), cudaMemcpyDeviceToHost, h->stream));
    unsigned long long* acc = (unsigned long long*)s->tmp64;
    DC_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), h->stream));
    ++g_launches;
    k_corner_bound<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, s->row0, acc);
    unsigned long long bound = 0;
    DC_CUDA(cudaMemcpyAsync(&bound, acc, sizeof(bound), cudaMemcpyDeviceToHost, h->stream));
    DC_CUDA(cudaStreamSynchronize(h->stream));
    {
        uint64_t run = 0;
        ck[K + 1] = 0;
        for (int32_t k = K; k >= 0; --k) {
            start[k] = (uint32_t)run;
            run += hh[k];
            ck[k] = (uint32_t)run;
        }
    }
    DC_CUDA(cudaMemcpyAsync(s->ck, ck.data(), sizeof(uint32_t) * ((size_t)K + 2), cudaMemcpyHostToDevice, h->stream));
    DC_CUDA(cudaMemcpyAsync(hist, start.data(), sizeof(uint32_t) * ((size_t)K + 2), cudaMemcpyHostToDevice, h->stream));
    ++g_launches;
    k_order_scatter<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, hist, s->order);
    // a run from row 1 (a full decomposition, or rows 1..R of a maintenance
    // batch) may be split in row segments run concurrently: segment 0 (rows
    // 1..cut[0]) on the handle's stream, segment i (rows cut[i-1]+1..cut[i],
    // starting there from row 0) on seg[i-1]'s stream, each with its own
    // state and its own range of the corner log; runs of fewer than
    // kMinSplitRows rows stay whole
    const int32_t k0 = std::max(1, K0);
    int32_t cut[kMaxRowSegments];
    int nseg = 1;
    if (k0 == 1 && Kstop >= kMinSplitRows)
        for (int i = 0; i < kMaxRowSegments - 1 && h->rows_split[i] > 0; ++i) {
            const int32_t c = (int32_t)((int64_t)K * h->rows_split[i] / 1000);
            if (c >= 1 && c < Kstop && (nseg == 1 || c > cut[nseg - 2])) cut[nseg++ - 1] = c;
        }
    cut[nseg - 1] = Kstop;
    int seg_bps = h->rows_bps;
    if (nseg > 1) {
        // every segment's blocks must be resident together for their grid barriers
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_trans2, kThreads, 0) != cudaSuccess)
            per_sm = 0;
        while (nseg > 1 && per_sm / nseg < 1) {
            cut[nseg - 2] = Kstop;
            --nseg;
        }
        const int want = seg_bps > 0 ? seg_bps : (h->blocks_per_sm > 0 ? h->blocks_per_sm : kDefaultBlocksPerSm);
        if (nseg > 1) seg_bps = std::min(want, per_sm / nseg);
    }
    // log ranges: [off[i], off[i] + cap[i]) per segment
    uint64_t off[kMaxRowSegments] = {}, capn[kMaxRowSegments] = {};
    uint64_t lc = bound + 1;
    if (nseg > 1) {
        SegBounds sb;
        sb.n = nseg;
        for (int i = 0; i < nseg; ++i) {
            sb.lo[i] = i == 0 ? k0 : cut[i - 1] + 1;
            sb.hi[i] = cut[i];
        }
        DC_CUDA(cudaMemsetAsync(acc, 0, nseg * sizeof(unsigned long long), h->stream));
        ++g_launches;
        k_corner_bounds<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, s->row0, sb, acc);
        unsigned long long bs[kMaxRowSegments] = {};
        DC_CUDA(cudaMemcpyAsync(bs, acc, nseg * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
        DC_CUDA(cudaStreamSynchronize(h->stream));
        lc = 0;
        for (int i = 0; i < nseg; ++i) {
            off[i] = lc;
            capn[i] = bs[i] + 1;
            lc += capn[i];
        }
    }
    if (s->log_cap < lc) {
        // a quarter of headroom: later runs (maintenance batches) rarely grow it again
        const uint64_t cap = lc + lc / 4;
        dfree(h->stream, s->log_v);
        dfree(h->stream, s->log_k);
        dfree(h->stream, s->log_l);
        s->log_cap = 0;
        if (dmalloc(h->stream, &s->log_v, cap) || dmalloc(h->stream, &s->log_k, cap) || dmalloc(h->stream, &s->log_l, cap)) return DC_ERR_NOMEM;
        s->log_cap = cap;
    }
    if (nseg == 1) capn[0] = s->log_cap;
    // The graph the row kernel reads: where sorting is allowed, the graph
    // relabeled in kmax order with kmax-sorted lists (C_k a prefix of the
    // ids); else the handle's own lists (kmax-sorted when they still are from
    // an earlier run) with C_k listed by `order`.
    int sorted = 0;
    const bool relabel = allow_sort && allow_relabel && K + 1 <= kSortBigBins;
    const uint32_t *G_out_off = g.out_off, *G_in_off = g.in_off, *G_order = s->order;
    int32_t *G_out_len = g.out_len, *G_in_len = g.in_len;
    uint32_t *G_out_nbr = g.out_nbr, *G_in_nbr = g.in_nbr;
    const int32_t *G_kmax = d.kmax_v, *G_row0 = s->row0;
    if (relabel) {
        if (int rc = build_relabeled(h, K)) return rc;
        sorted = 1;
        G_out_off = s->r_off[0];
        G_in_off = s->r_off[1];
        G_out_len = s->r_len[0];
        G_in_len = s->r_len[1];
        G_out_nbr = s->r_nbr[0];
        G_in_nbr = s->r_nbr[1];
        G_kmax = s->kmax_r;
        G_row0 = s->row0_r;
        G_order = nullptr;
    } else if (allow_sort || g.sorted_kmax) {
        if (int rc = sort_lists_by_kmax(h, K, &sorted)) return rc;
    }
    // starting values and counters of a run that starts at row a: row 0
    // inside C_a with the vertices outside already left (for a = 1 those of
    // kmax 0), so the run's first step has no leaving pass
    auto start_state = [&](cudaStream_t st, int32_t a, int32_t* cur, int32_t* co, int32_t* ci, uint32_t* mark,
                           int32_t* stamp) -> int {
        ++g_launches;
        k_preleft_cur<<<grid_for(h, V), kThreads, 0, st>>>(V, G_kmax, G_row0, a, cur);
        ++g_launches;
        k_counters_init<<<grid_for(h, (uint64_t)V * 32), kThreads, 0, st>>>(
            V, G_out_off, G_out_len, G_out_nbr, G_in_off, G_in_len, G_in_nbr, cur, co, ci, sorted);
        DC_CUDA(cudaMemsetAsync(mark, 0, sizeof(uint32_t) * V, st));
        DC_CUDA(cudaMemsetAsync(stamp, 0xFF, sizeof(int32_t) * V, st));
        return DC_OK;
    };
    if (int rc = start_state(h->stream, k0, s->cur, s->cnt_out, s->key, s->mark, s->stamp)) return rc;
    if (int rc = ensure_tring(h, 2ull * V + (uint64_t)h->geom.sms * 64 + 4096)) return rc;
    Trans2Params tp[kMaxRowSegments];
    tp[0].V = V;
    tp[0].out_off = G_out_off; tp[0].out_len = G_out_len; tp[0].out_nbr = G_out_nbr;
    tp[0].in_off = G_in_off; tp[0].in_len = G_in_len; tp[0].in_nbr = G_in_nbr;
    tp[0].kmax = G_kmax;
    tp[0].K = K;
    tp[0].K0 = k0;
    tp[0].preleft = 1;
    tp[0].Kstop = cut[0];
    tp[0].sorted = sorted;
    tp[0].order = G_order;
    tp[0].ck = s->ck;
    tp[0].cur = s->cur;
    tp[0].cnt_out = s->cnt_out;
    tp[0].cnt_in = s->key;
    tp[0].mark = s->mark;
    tp[0].stamp = s->stamp;
    tp[0].logidx = s->logidx;
    tp[0].log_v = s->log_v;
    tp[0].log_k = s->log_k;
    tp[0].log_l = s->log_l;
    tp[0].log_cap = capn[0];
    tp[0].q.slots = s->tring;
    tp[0].q.mask = (unsigned)(s->tring_cap - 1);
    tp[0].ctl = h->ctl;
    for (int i = 1; i < nseg; ++i)
        if (int rc = ensure_segment(h, i - 1, V)) return rc;
    if (nseg > 1) {
        // the other segments start once the shared preparation is done
        DC_CUDA(cudaEventRecord(s->seg[0].ev[0], h->stream));
        for (int i = 1; i < nseg; ++i) {
            RowSegment& sg = s->seg[i - 1];
            DC_CUDA(cudaStreamWaitEvent(sg.stream, s->seg[0].ev[0], 0));
            if (int rc = start_state(sg.stream, cut[i - 1] + 1, sg.cur, sg.cnt_out, sg.cnt_in, sg.mark, sg.stamp))
                return rc;
            Trans2Params& t = tp[i];
            t = tp[0];
            t.K0 = cut[i - 1] + 1;
            t.preleft = 1;
            t.Kstop = cut[i];
            t.cur = sg.cur;
            t.cnt_out = sg.cnt_out;
            t.cnt_in = sg.cnt_in;
            t.mark = sg.mark;
            t.stamp = sg.stamp;
            t.logidx = sg.logidx;
            t.log_v = s->log_v + off[i];
            t.log_k = s->log_k + off[i];
            t.log_l = s->log_l + off[i];
            t.log_cap = capn[i];
            t.q.slots = sg.tring;
            t.q.mask = (unsigned)(sg.tring_cap - 1);
            t.ctl = sg.ctl;
        }
    }
    uint64_t nlog = 0;
    uint64_t nseg_log[kMaxRowSegments] = {};
    unsigned long long voids[kMaxRowSegments] = {};
    cudaEventRecord(h->ev[3], h->stream);
    if (tp[0].Kstop >= tp[0].K0) {
        static const char* const kNames[8] = {"transitions",           "transitions (segment 2)",
                                              "transitions (segment 3)", "transitions (segment 4)",
                                              "transitions (segment 5)", "transitions (segment 6)",
                                              "transitions (segment 7)", "transitions (segment 8)"};
        static_assert(kMaxRowSegments <= 8, "one name per segment");
        void* args[kMaxRowSegments][1];
        int launched = 0, rc = DC_OK;
        for (int i = 0; i < nseg && rc == DC_OK; ++i) {
            args[i][0] = &tp[i];
            EngineCtl* ctl = i == 0 ? h->ctl : s->seg[i - 1].ctl;
            cudaStream_t st = i == 0 ? h->stream : s->seg[i - 1].stream;
            rc = persistent_launch(h, (const void*)k_trans2, args[i], kNames[i], ctl, st, seg_bps);
            if (rc == DC_OK) ++launched;
        }
        h->stat_evals = h->stat_drops = h->stat_entries = 0;
        for (int i = 0; i < launched; ++i) {
            EngineCtl hc;
            EngineCtl* ctl = i == 0 ? h->ctl : s->seg[i - 1].ctl;
            cudaStream_t st = i == 0 ? h->stream : s->seg[i - 1].stream;
            const int r = finish_persistent(h, ctl, st, kNames[i], &hc);
            if (r != DC_OK) {
                if (rc == DC_OK) rc = r;
                continue;
            }
            nseg_log[i] = hc.log_count;
            h->stat_evals += hc.evals;
            h->stat_drops += hc.drops;
            h->stat_entries += hc.edges_scanned;
        }
        if (rc) return rc;
        nlog = nseg_log[0];
        if (nseg > 1) {
            DC_CUDA(cudaMemsetAsync(acc, 0, nseg * sizeof(unsigned long long), h->stream));
            for (int i = 1; i < nseg; ++i) {
                RowSegment& sg = s->seg[i - 1];
                DC_CUDA(cudaEventRecord(sg.ev[1], sg.stream));
                DC_CUDA(cudaStreamWaitEvent(h->stream, sg.ev[1], 0));
                if (!nseg_log[i]) continue;
                // a corner at the segment's first row is void where the value
                // equals the previous segment's last row
                const int32_t* prev = i == 1 ? s->cur : s->seg[i - 2].cur;
                ++g_launches;
                k_seg_void<<<grid_for(h, nseg_log[i]), kThreads, 0, h->stream>>>(
                    nseg_log[i], s->log_v + off[i], s->log_k + off[i], s->log_l + off[i], cut[i - 1] + 1, prev,
                    acc + i);
            }
            DC_CUDA(cudaMemcpyAsync(voids, acc, nseg * sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
            DC_CUDA(cudaStreamSynchronize(h->stream));
            h->nseg_extra = nseg - 1;
            for (int i = 1; i < nseg; ++i) {
                h->seg_off[i - 1] = off[i];
                h->seg_n[i - 1] = nseg_log[i];
                h->seg_void[i - 1] = voids[i];
            }
        }
        if (relabel)  // corner records back to original ids (the seam check above compares relabeled state)
            for (int i = 0; i < nseg; ++i)
                if (nseg_log[i]) {
                    ++g_launches;
                    k_unlabel_log<<<grid_for(h, nseg_log[i]), kThreads, 0, h->stream>>>(nseg_log[i], s->order,
                                                                                       s->log_v + off[i]);
                }
    }
    cudaEventRecord(h->ev[4], h->stream);
    *nlog_out = nlog;
    return DC_OK;
}

int decompose(dc_graph* h, int method, int materialize_rows) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    const uint32_t V = g.V;
    d.valid = false;
    d.rows_valid = false;
    if (int rc = ensure_scratch(h, V)) return rc;
    Scratch* s = h->scratch;
    if (!d.kmax_v && dmalloc(h->stream, &d.kmax_v, (uint64_t)V + 1)) return DC_ERR_NOMEM;
    d.peel_valid = false;
    if (V == 0) {
        d.kmax = 0;
        d.lmax = 0;
        d.n_corners = 0;
        if (!d.sky_off && dmalloc(h->stream, &d.sky_off, 1)) return DC_ERR_NOMEM;
        DC_CUDA(cudaMemsetAsync(d.sky_off, 0, sizeof(uint32_t), h->stream));
        d.row_lo = 1;
        d.row_hi = 0;
        d.peel_valid = true;
        d.valid = true;
        return DC_OK;
    }
    cudaEventRecord(h->ev[0], h->stream);
    // kmax (in-degree peel) and row 0 (out-degree peel) in one grid
    int32_t mv[2] = {0, 0};
    {
        PeelInst I[2] = {make_inst(h, 0, nullptr, 0, d.kmax_v, 0), make_inst(h, 1, nullptr, 0, s->row0, 1)};
        if (int rc = run_peel2(h, 2, I, mv)) return rc;
    }
    cudaEventRecord(h->ev[1], h->stream);
    const int32_t K = mv[0];
    d.kmax = K;
    d.lmax = mv[1];
    if (!d.row0 && dmalloc(h->stream, &d.row0, (uint64_t)V + 1)) return DC_ERR_NOMEM;
    DC_CUDA(cudaMemcpyAsync(d.row0, s->row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
    d.peel_valid = true;
    d.row_lo = 1;
    d.row_hi = K;
    if (method == 1) {
        // one fresh peel per row (the reference's schedule, main.cu:238-244),
        // two rows per launch
        if (int rc = ensure_rows(h, (uint64_t)(K + 1) * V)) return rc;
        DC_CUDA(cudaMemcpyAsync(d.rows, s->row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
        for (int32_t k = 1; k <= K; k += 2) {
            int n = (k + 1 <= K) ? 2 : 1;
            PeelInst I[2] = {make_inst(h, 1, d.kmax_v, k, d.rows + (uint64_t)k * V, 0),
                             make_inst(h, 1, d.kmax_v, k + 1, d.rows + (uint64_t)(k + 1) * V, 1)};
            int32_t m2[2];
            if (int rc = run_peel2(h, n, I, m2)) return rc;
        }
        cudaEventRecord(h->ev[2], h->stream);
        cudaEventRecord(h->ev[3], h->stream);
        unsigned long long* cnt = (unsigned long long*)s->tmp64;
        ++g_launches;
        k_rows_corner_count<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, K, d.kmax_v, d.rows, cnt);
        if (int rc = scan_tmp64(h, V)) return rc;
        unsigned long long total = 0;
        DC_CUDA(cudaMemcpyAsync(&total, s->tmp64 + V, sizeof(total), cudaMemcpyDeviceToHost, h->stream));
        DC_CUDA(cudaStreamSynchronize(h->stream));
        if (d.corner_cap < total) {
            dfree(h->stream, d.sky_k);
            dfree(h->stream, d.sky_l);
            if (dmalloc(h->stream, &d.sky_k, total) || dmalloc(h->stream, &d.sky_l, total)) return DC_ERR_NOMEM;
            d.corner_cap = total;
        }
        if (!d.sky_off && dmalloc(h->stream, &d.sky_off, (uint64_t)V + 1)) return DC_ERR_NOMEM;
        ++g_launches;
        k_rows_corner_fill<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, d.rows, cnt, d.sky_k, d.sky_l,
                                                                        d.sky_off);
        d.n_corners = total;
        d.rows_valid = true;
        if (int rc = degree_kmax_sum(h, &h->full_work)) return rc;
        cudaEventRecord(h->ev[4], h->stream);
        cudaEventRecord(h->ev[5], h->stream);
        cudaEventRecord(h->ev[6], h->stream);
        DC_CUDA(cudaStreamSynchronize(h->stream));
        d.valid = true;
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
        h->times.kmax_ms = ms;
        h->times.row0_ms = 0;
        cudaEventElapsedTime(&ms, h->ev[1], h->ev[2]);
        h->times.trans_ms = ms;
        h->full_rows_ms = ms;
        cudaEventElapsedTime(&ms, h->ev[3], h->ev[4]);
        h->times.sky_ms = ms;
        h->times.expand_ms = 0;
        return DC_OK;
    }
    // ---- method 0: rows 1..K derived row to row
    uint64_t nlog = 0;
    if (int rc = rows_from_row0(h, K, K, true, &nlog)) return rc;
    if (int rc = degree_kmax_sum(h, &h->full_work)) return rc;
    if (int rc = build_skyline_from_log(h, nlog)) return rc;
    cudaEventRecord(h->ev[5], h->stream);
    d.valid = true;
    if (materialize_rows) {
        if (int rc = ensure_rows(h, (uint64_t)(K + 1) * V)) return rc;
        if (int rc = expand_rows(h, 0, (uint32_t)K + 1, d.rows)) return rc;
        d.rows_valid = true;
    }
    cudaEventRecord(h->ev[6], h->stream);
    DC_CUDA(cudaStreamSynchronize(h->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
    h->times.kmax_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[1], h->ev[3]);
    h->times.row0_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[3], h->ev[4]);
    h->times.trans_ms = ms;
    h->full_rows_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]);
    h->times.sky_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[5], h->ev[6]);
    h->times.expand_ms = ms;
    return DC_OK;
}

int row_weights(dc_graph* h, uint64_t* out) {
    const DevGraph& g = h->g;
    const Decomp& d = h->d;
    const int32_t K = d.kmax;
    unsigned long long* w = nullptr;
    if (dmalloc(h->stream, &w, (uint64_t)K + 1)) return DC_ERR_NOMEM;
    DC_CUDA(cudaMemsetAsync(w, 0, 8ull * (K + 1), h->stream));
    if (g.V) {
        ++g_launches;
        size_t shm = K + 1 <= 4096 ? 8ull * (K + 1) : 0;
        k_kmax_degree_hist<<<grid_for(h, g.V), kThreads, shm, h->stream>>>(g.V, d.kmax_v, g.in_len, g.out_len, K, w);
    }
    std::vector<uint64_t> hw((size_t)K + 1);
    DC_CUDA(cudaMemcpyAsync(hw.data(), w, 8ull * (K + 1), cudaMemcpyDeviceToHost, h->stream));
    dfree(h->stream, w);
    DC_CUDA(cudaStreamSynchronize(h->stream));
    uint64_t run = 0;
    for (int32_t k = K; k >= 0; --k) {
        run += hw[k];
        out[k] = run;
    }
    return DC_OK;
}

// sum over vertices of (in + out degree) x kmax: the list entries a per-row
// pass over rows 1..kmax scans, a deterministic measure of a graph's row work
__global__ void k_deg_kmax_sum(uint32_t V, const int32_t* kmax, const int32_t* in_len, const int32_t* out_len,
                               unsigned long long* acc) {
    unsigned long long w = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        w += (unsigned long long)(in_len[v] + out_len[v]) * (unsigned long long)max(kmax[v], 0);
#pragma unroll
    for (int s = 16; s; s >>= 1) w += __shfl_xor_sync(0xFFFFFFFFu, w, s);
    if ((threadIdx.x & 31u) == 0) atomicAdd(acc, w);
}

int degree_kmax_sum(dc_graph* h, uint64_t* out) {
    unsigned long long* acc = (unsigned long long*)h->scratch->tmp64;
    DC_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), h->stream));
    ++g_launches;
    k_deg_kmax_sum<<<grid_for(h, h->g.V), kThreads, 0, h->stream>>>(h->g.V, h->d.kmax_v, h->g.in_len, h->g.out_len,
                                                                     acc);
    unsigned long long w = 0;
    DC_CUDA(cudaMemcpyAsync(&w, acc, sizeof(w), cudaMemcpyDeviceToHost, h->stream));
    DC_CUDA(cudaStreamSynchronize(h->stream));
    *out = w;
    return DC_OK;
}

int decompose_range(dc_graph* h, int32_t k_first, int32_t k_last) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    const uint32_t V = g.V;
    if (k_first <= 0 || !d.peel_valid || !d.kmax_v || !d.row0) {
        // kmax and row 0 (fused peel)
        if (int rc = ensure_scratch(h, V)) return rc;
        Scratch* s = h->scratch;
        if (!d.kmax_v && dmalloc(h->stream, &d.kmax_v, (uint64_t)V + 1)) return DC_ERR_NOMEM;
        if (V == 0) return decompose(h, 0, 0);
        d.valid = false;
        d.rows_valid = false;
        cudaEventRecord(h->ev[0], h->stream);
        int32_t mv[2] = {0, 0};
        PeelInst I[2] = {make_inst(h, 0, nullptr, 0, d.kmax_v, 0), make_inst(h, 1, nullptr, 0, s->row0, 1)};
        if (int rc = run_peel2(h, 2, I, mv)) return rc;
        cudaEventRecord(h->ev[1], h->stream);
        d.kmax = mv[0];
        d.lmax = mv[1];
        if (!d.row0 && dmalloc(h->stream, &d.row0, (uint64_t)V + 1)) return DC_ERR_NOMEM;
        DC_CUDA(cudaMemcpyAsync(d.row0, s->row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
        DC_CUDA(cudaStreamSynchronize(h->stream));
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
        h->times.kmax_ms = ms;
        d.peel_valid = true;
    } else {
        h->times.kmax_ms = 0;
    }
    if (int rc = ensure_scratch(h, V)) return rc;
    Scratch* s = h->scratch;
    const int32_t K = d.kmax;
    const int32_t k0 = std::max(1, k_first), k1 = std::min(k_last, K);
    d.rows_valid = false;
    // the row kernel starts from row 0 in scratch
    DC_CUDA(cudaMemcpyAsync(s->row0, d.row0, 4ull * V, cudaMemcpyDeviceToDevice, h->stream));
    uint64_t nlog = 0;
    if (int rc = rows_from_row0(h, K, k1, true, &nlog, k0)) return rc;
    if (int rc = build_skyline_from_log(h, nlog)) return rc;
    cudaEventRecord(h->ev[5], h->stream);
    DC_CUDA(cudaStreamSynchronize(h->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev[3], h->ev[4]);
    h->times.trans_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]);
    h->times.sky_ms = ms;
    h->times.row0_ms = 0;
    h->times.expand_ms = 0;
    d.row_lo = k0;
    d.row_hi = k1;
    d.valid = true;
    return DC_OK;
}


}  // namespace dc
