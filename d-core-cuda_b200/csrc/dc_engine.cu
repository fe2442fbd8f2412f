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
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dc_engine.cuh"
#include "dc_internal.h"

namespace dc {

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

template <typename T>
static int dmalloc(T** p, uint64_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "device allocation of %llu bytes failed: %s",
                         (unsigned long long)(n * sizeof(T)), cudaGetErrorString(e));
    }
    return DC_OK;
}
template <typename T>
static void dfree(T*& p) {
    if (p) cudaFree((void*)p);
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
// persistent peel
// ---------------------------------------------------------------------------
struct PeelParams {
    uint32_t V;
    const uint32_t* a_off;
    const int32_t* a_len;
    const uint32_t* a_nbr;
    const uint32_t* b_off;
    const int32_t* b_len;
    const uint32_t* b_nbr;
    const int32_t* member;  // nullptr: every vertex is in the set
    int32_t k;              // constraint threshold (0: none)
    int32_t* key;
    int32_t* cdeg;
    int32_t* val;
    uint32_t* rem0;
    uint32_t* rem1;
    RingQueue q;
    EngineCtl* ctl;
};

// One pass of the reference's level loop (KListInplace, main.cu:171-195):
// level L removes every remaining vertex whose peeling degree is L (scan,
// main.cu:37-56) and then the cascade of vertices whose peeling degree falls
// to L or whose constraint degree falls below k (process, main.cu:100-135),
// all with value L.  Here the cascade runs through the device work queue and
// one software grid barrier separates levels.
__global__ void __launch_bounds__(kThreads) k_peel(PeelParams p) {
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const unsigned gwarp = blockIdx.x * kWarpsPerBlock + wib;
    const unsigned nwarps = gridDim.x * kWarpsPerBlock;
    EngineCtl* c = p.ctl;
    __shared__ uint32_t s_x[kWarpsPerBlock][32];
    __shared__ uint32_t s_start[kWarpsPerBlock][32];
    __shared__ int32_t s_la[kWarpsPerBlock][32];

    // ---- init: degrees restricted to the member set, remaining list
    for (uint64_t base = (uint64_t)gwarp * 32; base < p.V; base += (uint64_t)nwarps * 32) {
        uint64_t vi = base + lane;
        bool ok = vi < p.V, in = false;
        uint32_t v = (uint32_t)vi;
        if (ok) {
            in = !p.member || p.member[v] >= p.k;
            if (!in) {
                p.val[v] = 0;
            } else {
                p.val[v] = -1;
                int kd = 0, cd = 0;
                if (!p.member) {
                    kd = p.a_len[v];
                } else {
                    uint32_t o = p.a_off[v], e = o + (uint32_t)p.a_len[v];
                    for (; o < e; ++o) kd += (p.member[p.a_nbr[o]] >= p.k);
                    o = p.b_off[v];
                    e = o + (uint32_t)p.b_len[v];
                    for (; o < e; ++o) cd += (p.member[p.b_nbr[o]] >= p.k);
                }
                p.key[v] = kd;
                p.cdeg[v] = cd;
            }
        }
        unsigned pos = warp_append(&c->rcount[0], ok && in);
        if (ok && in) p.rem0[pos] = v;
    }
    if (!grid_sync(c)) return;

    uint32_t* rc = p.rem0;
    uint32_t* rn = p.rem1;
    int L = 0;
    for (;; ++L) {
        const unsigned cs = L % 3, ns = (L + 1) % 3, zs = (L + 2) % 3;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            c->rcount[zs] = 0;
            c->producers[ns] = 0;
        }
        const unsigned n_rem = ld_vol(&c->rcount[cs]);
        if (n_rem == 0) break;
        bool pushed_any = false;
        // ---- scan the remaining list
        for (unsigned base = gwarp * 32; base < n_rem; base += nwarps * 32) {
            unsigned i = base + lane;
            bool ok = i < n_rem;
            uint32_t v = ok ? rc[i] : 0;
            bool keep = false, push = false;
            if (ok && ld_vol(&p.val[v]) == -1) {
                if (ld_vol(&p.key[v]) <= L)
                    push = atomicCAS(&p.val[v], -1, L) == -1;
                else
                    keep = true;
            }
            unsigned pos = warp_append(&c->rcount[ns], keep);
            if (keep) rn[pos] = v;
            q_push_warp(c, p.q, push, v);
            pushed_any |= push;
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(&c->producers[cs], 1u);

        // ---- drain the cascade
        IdleClock clk;
        clk.start(c);
        for (;;) {
            unsigned first;
            bool fin;
            unsigned n = q_claim_warp(c, 32, nwarps, &c->producers[cs], &first, &fin);
            if (n == 0) {
                if (fin || ld_vol(&c->error)) break;
                if (!clk.tick(c)) break;
                continue;
            }
            uint32_t x = 0;
            int la = 0, lb = 0;
            if (lane < n) {
                x = q_take(c, p.q, first + lane);
                if (x != kEmptySlot) {
                    la = p.k > 0 ? p.a_len[x] : 0;
                    lb = p.b_len[x];
                }
            }
            unsigned tot = (unsigned)(la + lb);
            unsigned inc = warp_incl_scan(tot);
            unsigned T = __shfl_sync(0xFFFFFFFFu, inc, 31);
            s_x[wib][lane] = x;
            s_start[wib][lane] = inc - tot;
            s_la[wib][lane] = la;
            __syncwarp();
            for (unsigned base = 0; base < T; base += 32) {
                unsigned e = base + lane;
                bool push = false;
                uint32_t pv = 0;
                if (e < T) {
                    int lo = 0, hi = (int)n - 1;
                    while (lo < hi) {
                        int mid = (lo + hi + 1) >> 1;
                        if (s_start[wib][mid] <= e) lo = mid;
                        else hi = mid - 1;
                    }
                    uint32_t xj = s_x[wib][lo];
                    unsigned local = e - s_start[wib][lo];
                    int laj = s_la[wib][lo];
                    if ((int)local < laj) {
                        uint32_t u = p.a_nbr[p.a_off[xj] + local];
                        int old = atomicSub(&p.cdeg[u], 1);
                        if (old == p.k && ld_vol(&p.val[u]) == -1 && atomicCAS(&p.val[u], -1, L) == -1) {
                            push = true;
                            pv = u;
                        }
                    } else {
                        uint32_t w = p.b_nbr[p.b_off[xj] + (local - (unsigned)laj)];
                        int old = atomicSub(&p.key[w], 1);
                        if (old == L + 1 && ld_vol(&p.val[w]) == -1 && atomicCAS(&p.val[w], -1, L) == -1) {
                            push = true;
                            pv = w;
                        }
                    }
                }
                q_push_warp(c, p.q, push, pv);
                pushed_any |= push;
            }
            q_done_warp(c, n);
        }
        if (__any_sync(0xFFFFFFFFu, pushed_any) && lane == 0) atomicMax(&c->maxval, L);
        if (!grid_sync(c)) return;
        uint32_t* t = rc;
        rc = rn;
        rn = t;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) c->steps = L;
}

// ---------------------------------------------------------------------------
// incremental rows
// ---------------------------------------------------------------------------
struct TransParams {
    uint32_t V;
    const uint32_t* out_off;
    const int32_t* out_len;
    const uint32_t* out_nbr;
    const uint32_t* in_off;
    const int32_t* in_len;
    const uint32_t* in_nbr;
    const int32_t* kmax;
    int32_t K;
    const uint32_t* order;  // vertices by kmax descending
    const uint32_t* ck;     // ck[k] = |C_k|, k = 0..K+1
    int32_t* cur;           // row values, -1 outside C
    int32_t* cnt_in;        // #in-neighbours with cur >= cur[v]
    uint32_t* mark;
    int32_t* stamp;
    uint32_t* logidx;
    uint32_t* log_v;
    int32_t* log_k;
    int32_t* log_l;
    unsigned long long log_cap;
    RingQueue q;
    EngineCtl* ctl;
};

static constexpr int kWin = 64;

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

// cnt_in[v] = #{w in N_in(v) : cur[w] >= cur[v]}  (warp per vertex)
__global__ void k_cnt_in_init(uint32_t V, const uint32_t* in_off, const int32_t* in_len, const uint32_t* in_nbr,
                              const int32_t* cur, int32_t* cnt_in) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = gw; v < V; v += nw) {
        int cv = cur[v];
        uint32_t o = in_off[v];
        int n = in_len[v];
        int cnt = 0;
        for (int i = lane; i < n; i += 32) cnt += (cur[in_nbr[o + i]] >= cv);
#pragma unroll
        for (int s = 16; s; s >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, s);
        if (lane == 0) cnt_in[v] = cnt;
    }
}

// Warp evaluation of vertex x against in-count requirement kreq.
// New value = max L <= cap with #{out-nbrs u: cur[u] >= L} >= L and
// #{in-nbrs w: cur[w] >= L} >= kreq; found by windowed histograms of
// neighbour values, 64 levels per pass from the top.
// Returns new value; *cnt = #{in-nbrs w : cur[w] >= new value}.
__device__ int eval_vertex(const TransParams& p, uint32_t x, int cap, int kreq, int* s_ho, int* s_hi, int* cnt_out_in) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t oo = p.out_off[x], io = p.in_off[x];
    const int on = p.out_len[x], in = p.in_len[x];
    int carry_o = 0, carry_i = 0;
    int hi = cap;
    for (;;) {
        int lo = max(0, hi - (kWin - 1));
        s_ho[lane] = 0;
        s_ho[lane + 32] = 0;
        s_hi[lane] = 0;
        s_hi[lane + 32] = 0;
        __syncwarp();
        for (int i = lane; i < on; i += 32) {
            int cu = ld_vol(&p.cur[p.out_nbr[oo + i]]);
            if (cu >= lo) {
                if (cu >= hi) {
                    if (hi == cap || cu <= hi) atomicAdd(&s_ho[hi - lo], 1);
                } else {
                    atomicAdd(&s_ho[cu - lo], 1);
                }
            }
        }
        for (int i = lane; i < in; i += 32) {
            int cw = ld_vol(&p.cur[p.in_nbr[io + i]]);
            if (cw >= lo) {
                if (cw >= hi) {
                    if (hi == cap || cw <= hi) atomicAdd(&s_hi[hi - lo], 1);
                } else {
                    atomicAdd(&s_hi[cw - lo], 1);
                }
            }
        }
        __syncwarp();
        // suffix sums over bins [0, hi-lo]; lane handles bins 2*lane, 2*lane+1
        int b0 = 2 * lane, b1 = 2 * lane + 1;
        int o0 = s_ho[b0], o1 = s_ho[b1], i0 = s_hi[b0], i1 = s_hi[b1];
        int po = o0 + o1, pi = i0 + i1;
        // reverse inclusive scan (from lane 31 down to lane)
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
        // cum at bin b1 = carry + (suffix from lane+1) + o1 ; at b0 = that + o0
        int cum_o1 = carry_o + (so - po) + o1, cum_i1 = carry_i + (si - pi) + i1;
        int cum_o0 = cum_o1 + o0, cum_i0 = cum_i1 + i0;
        int L0 = lo + b0, L1 = lo + b1;
        bool ok1 = (L1 <= hi) && cum_o1 >= L1 && cum_i1 >= kreq;
        bool ok0 = (L0 <= hi) && cum_o0 >= L0 && cum_i0 >= kreq;
        unsigned m1 = __ballot_sync(0xFFFFFFFFu, ok1), m0 = __ballot_sync(0xFFFFFFFFu, ok0);
        int best = -1, bestcnt = 0;
        // highest L satisfying: compare top lanes of m1 and m0
        int t1 = m1 ? 31 - __clz(m1) : -1, t0 = m0 ? 31 - __clz(m0) : -1;
        int c1 = __shfl_sync(0xFFFFFFFFu, cum_i1, t1 < 0 ? 0 : t1);
        int c0 = __shfl_sync(0xFFFFFFFFu, cum_i0, t0 < 0 ? 0 : t0);
        if (t1 >= 0) {
            best = lo + 2 * t1 + 1;
            bestcnt = c1;
        }
        if (t0 >= 0 && lo + 2 * t0 > best) {
            best = lo + 2 * t0;
            bestcnt = c0;
        }
        if (best >= 0) {
            *cnt_out_in = bestcnt;
            return best;
        }
        // carry the whole window into the next one below
        int wo = __shfl_sync(0xFFFFFFFFu, so, 0), wi = __shfl_sync(0xFFFFFFFFu, si, 0);
        carry_o += wo;
        carry_i += wi;
        if (lo == 0) {  // cannot happen for members of C_kreq; report value 0
            *cnt_out_in = carry_i;
            return 0;
        }
        hi = lo - 1;
        __syncwarp();
    }
}

// Rows 1..K from row 0.  Row j is the greatest fixpoint below row j-1 of
//   l(v) = max L : |{u in N_out(v) : l(u) >= L}| >= L  and
//                  |{w in N_in(v)  : l(w) >= L}| >= j,  v in C_j,
// which is the (j, l)-core number of v (the value the reference's pass k = j
// produces, main.cu:238-244).  Starting from row j-1 (a pointwise upper
// bound, since the (j,l)-core is inside the (j-1,l)-core) the kernel only
// re-evaluates vertices whose bound can be violated: those leaving C_j
// (kmax == j-1), those whose in-count at their own level is below j, and,
// transitively, neighbours of every vertex whose value drops.
__global__ void __launch_bounds__(kThreads) k_transitions(TransParams p) {
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const unsigned gwarp = blockIdx.x * kWarpsPerBlock + wib;
    const unsigned nwarps = gridDim.x * kWarpsPerBlock;
    EngineCtl* c = p.ctl;
    __shared__ int s_ho[kWarpsPerBlock][kWin];
    __shared__ int s_hi[kWarpsPerBlock][kWin];
    unsigned long long my_evals = 0, my_drops = 0;

    for (int j = 1; j <= p.K; ++j) {
        const unsigned cs = j % 3, ns = (j + 1) % 3;
        if (blockIdx.x == 0 && threadIdx.x == 0) c->producers[ns] = 0;
        const uint32_t vj = p.ck[j], vprev = p.ck[j - 1];
        // ---- vertices leaving C_j: value -1, wake neighbours they supported
        for (uint32_t i = vj + gwarp; i < vprev; i += nwarps) {
            uint32_t x = p.order[i];
            int a = p.cur[x];
            __syncwarp();
            if (lane == 0) {
                p.cur[x] = -1;
                __threadfence();
            }
            __syncwarp();
            if (a < 1) continue;
            uint32_t o = p.out_off[x];
            int n = p.out_len[x];
            for (int b = 0; b < n; b += 32) {
                bool push = false;
                uint32_t z = 0;
                if (b + (int)lane < n) {
                    z = p.out_nbr[o + b + lane];
                    int cz = ld_vol(&p.cur[z]);
                    push = cz >= 1 && cz <= a && mark_request(&p.mark[z], c);
                }
                q_push_warp(c, p.q, push, z);
            }
            o = p.in_off[x];
            n = p.in_len[x];
            for (int b = 0; b < n; b += 32) {
                bool push = false;
                uint32_t y = 0;
                if (b + (int)lane < n) {
                    y = p.in_nbr[o + b + lane];
                    int cy = ld_vol(&p.cur[y]);
                    push = cy >= 1 && cy <= a && mark_request(&p.mark[y], c);
                }
                q_push_warp(c, p.q, push, y);
            }
        }
        // ---- seeds: members whose in-count at their level is below j
        for (uint32_t base = gwarp * 32; base < vj; base += nwarps * 32) {
            uint32_t i = base + lane;
            bool push = false;
            uint32_t v = 0;
            if (i < vj) {
                v = p.order[i];
                push = p.cur[v] >= 1 && p.cnt_in[v] < j && mark_request(&p.mark[v], c);
            }
            q_push_warp(c, p.q, push, v);
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(&c->producers[cs], 1u);

        // ---- drain
        IdleClock clk;
        clk.start(c);
        for (;;) {
            unsigned first;
            bool fin;
            unsigned n = q_claim_warp(c, 1, nwarps, &c->producers[cs], &first, &fin);
            if (n == 0) {
                if (fin || ld_vol(&c->error)) break;
                if (!clk.tick(c)) break;
                continue;
            }
            uint32_t x = 0;
            if (lane == 0) {
                x = q_take(c, p.q, first);
                if (x != kEmptySlot) {
                    atomicExch(&p.mark[x], 2u);
                    __threadfence();
                }
            }
            x = __shfl_sync(0xFFFFFFFFu, x, 0);
            if (x == kEmptySlot) {
                q_done_warp(c, n);
                continue;
            }
            int cap = ld_vol(&p.cur[x]);
            if (p.kmax[x] < j || cap < 1) {
                // outside C_j or at value 0: nothing can change
                if (lane == 0) atomicExch(&p.mark[x], 0u);
                q_done_warp(c, n);
                continue;
            }
            int cnt = 0;
            int nv = eval_vertex(p, x, cap, j, s_ho[wib], s_hi[wib], &cnt);
            ++my_evals;
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
                // wake neighbours whose support crossed: value in (nv, cap]
                uint32_t o = p.out_off[x];
                int m = p.out_len[x];
                for (int b = 0; b < m; b += 32) {
                    bool push = false;
                    uint32_t z = 0;
                    if (b + (int)lane < m) {
                        z = p.out_nbr[o + b + lane];
                        int cz = ld_vol(&p.cur[z]);
                        push = cz > nv && cz <= cap && mark_request(&p.mark[z], c);
                    }
                    q_push_warp(c, p.q, push, z);
                }
                o = p.in_off[x];
                m = p.in_len[x];
                for (int b = 0; b < m; b += 32) {
                    bool push = false;
                    uint32_t y = 0;
                    if (b + (int)lane < m) {
                        y = p.in_nbr[o + b + lane];
                        int cy = ld_vol(&p.cur[y]);
                        push = cy > nv && cy <= cap && mark_request(&p.mark[y], c);
                    }
                    q_push_warp(c, p.q, push, y);
                }
            }
            // release x; after a drop it is re-run once more, so that values
            // of neighbours that dropped concurrently are seen
            bool requeue = false;
            if (lane == 0) {
                p.cnt_in[x] = cnt;
                __threadfence();
                if (nv < cap && nv >= 1) {
                    atomicExch(&p.mark[x], 1u);
                    requeue = true;
                } else {
                    unsigned o = atomicCAS(&p.mark[x], 2u, 0u);
                    if (o == 3u) {
                        if (nv >= 1) {
                            atomicExch(&p.mark[x], 1u);
                            requeue = true;
                        } else {
                            atomicExch(&p.mark[x], 0u);
                        }
                    }
                }
            }
            q_push_warp(c, p.q, requeue, x);
            q_done_warp(c, n);
        }
        if (!grid_sync(c)) break;
    }
    if (lane == 0) {
        atomicAdd(&c->evals, my_evals);
        atomicAdd(&c->drops, my_drops);
    }
}

// ---------------------------------------------------------------------------
// order by kmax, skyline assembly, expansion
// ---------------------------------------------------------------------------
__global__ void k_kmax_hist(uint32_t V, const int32_t* kmax, uint32_t* hist) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&hist[kmax[v]], 1u);
}

// cursor[k] = first position of bucket k in descending-kmax order
__global__ void k_order_scatter(uint32_t V, const int32_t* kmax, uint32_t* cursor, uint32_t* order) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t p = atomicAdd(&cursor[kmax[v]], 1u);
        order[p] = (uint32_t)v;
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

__global__ void k_sky_count(uint32_t V, uint64_t nlog, const uint32_t* log_v, unsigned long long* cnt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlog; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[log_v[i]], 1ull);
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

static int check_ctl(dc_graph* h, EngineCtl* hc, const char* what) {
    DC_CUDA(cudaMemcpyAsync(hc, h->ctl, sizeof(EngineCtl), cudaMemcpyDeviceToHost, h->stream));
    DC_CUDA(cudaStreamSynchronize(h->stream));
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
    cudaDeviceProp prop;
    DC_CUDA(cudaGetDeviceProperties(&prop, h->device));
    if (!prop.cooperativeLaunch) return set_error(DC_ERR_NO_DEVICE, "device lacks cooperative launch");
    h->geom.sms = prop.multiProcessorCount;
    h->geom.threads = kThreads;
    DC_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    if (dmalloc(&h->ctl, 1)) return DC_ERR_NOMEM;
    for (auto& e : h->ev) DC_CUDA(cudaEventCreate(&e));
    return DC_OK;
}

void free_graph_arrays(DevGraph& g) {
    dfree(g.out_off);
    dfree(g.out_len);
    dfree(g.out_nbr);
    dfree(g.in_off);
    dfree(g.in_len);
    dfree(g.in_nbr);
    g.out_cap = g.in_cap = 0;
}

void free_decomp(Decomp& d) {
    dfree(d.kmax_v);
    dfree(d.sky_off);
    dfree(d.sky_k);
    dfree(d.sky_l);
    dfree(d.rows);
    d.rows_cap = 0;
    d.corner_cap = 0;
    d.valid = false;
    d.rows_valid = false;
}

void free_scratch(dc_graph* h) {
    Scratch* s = h->scratch;
    if (!s) return;
    dfree(s->key);
    dfree(s->cdeg);
    dfree(s->cur);
    dfree(s->row0);
    dfree(s->mark);
    dfree(s->stamp);
    dfree(s->logidx);
    dfree(s->rem0);
    dfree(s->rem1);
    dfree(s->order);
    dfree(s->ck);
    dfree(s->ring);
    dfree(s->log_v);
    dfree(s->log_k);
    dfree(s->log_l);
    dfree(s->tmp64);
    dfree(s->partial);
    dfree(s->cursor);
    if (s->tmp_edges) cudaFree(s->tmp_edges);
    delete s;
    h->scratch = nullptr;
}

int ensure_scratch(dc_graph* h, uint32_t V) {
    if (!h->scratch) h->scratch = new Scratch();
    Scratch* s = h->scratch;
    if (s->cap_V >= V && s->key) return DC_OK;
    uint32_t keep_ck = s->ck_cap;
    (void)keep_ck;
    // release V-sized buffers and reallocate
    dfree(s->key); dfree(s->cdeg); dfree(s->cur); dfree(s->row0); dfree(s->mark); dfree(s->stamp);
    dfree(s->logidx); dfree(s->rem0); dfree(s->rem1); dfree(s->order); dfree(s->ring); dfree(s->tmp64);
    dfree(s->partial); dfree(s->cursor);
    uint64_t n = (uint64_t)V + 1;
    if (dmalloc(&s->key, n) || dmalloc(&s->cdeg, n) || dmalloc(&s->cur, n) || dmalloc(&s->row0, n) ||
        dmalloc(&s->mark, n) || dmalloc(&s->stamp, n) || dmalloc(&s->logidx, n) || dmalloc(&s->rem0, n) ||
        dmalloc(&s->rem1, n) || dmalloc(&s->order, n) || dmalloc(&s->tmp64, n + 1) ||
        dmalloc(&s->partial, (uint64_t)h->geom.sms * 64 + 64) || dmalloc(&s->cursor, n + 1))
        return DC_ERR_NOMEM;
    uint64_t need = (uint64_t)V + (uint64_t)h->geom.sms * 64 * 32 + 64;
    uint64_t rc = 1024;
    while (rc < need) rc <<= 1;
    if (dmalloc(&s->ring, rc)) return DC_ERR_NOMEM;
    s->ring_mask = (uint32_t)(rc - 1);
    s->cap_V = V;
    return DC_OK;
}

// Exclusive scan of n u64 values in s->tmp64 (tmp64[n] receives the total).
static int scan_tmp64(dc_graph* h, uint64_t n) {
    Scratch* s = h->scratch;
    unsigned long long* data = (unsigned long long*)s->tmp64;
    unsigned long long* part = (unsigned long long*)s->partial;
    void* args[] = {&data, &n, &part, &h->ctl};
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_scan_coop, 256, 0);
    per_sm = std::max(1, std::min(per_sm, 8));
    DC_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
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
        if (dmalloc(off, (uint64_t)V + 1) || dmalloc(nbr, total)) return DC_ERR_NOMEM;
        k_off_to_u32<<<grid_for(h, (uint64_t)V + 1), kThreads, 0, h->stream>>>(V, (unsigned long long*)s->tmp64, *off);
        if (side == 0) g.out_cap = total;
        else g.in_cap = total;
    }
    DC_CUDA(cudaMemsetAsync(g.out_len, 0, sizeof(int32_t) * V, h->stream));
    DC_CUDA(cudaMemsetAsync(g.in_len, 0, sizeof(int32_t) * V, h->stream));
    if (E)
        k_scatter_edges<<<grid_for(h, E), kThreads, 0, h->stream>>>(E, d_src, d_dst, g.out_off, g.out_len, g.out_nbr,
                                                                     g.in_off, g.in_len, g.in_nbr);
    DC_CUDA(cudaGetLastError());
    g.V = V;
    g.E = E;
    return DC_OK;
}

int build_from_device_edges(dc_graph* h, uint32_t V, uint64_t E, const uint32_t* d_src, const uint32_t* d_dst) {
    free_graph_arrays(h->g);
    free_decomp(h->d);
    if (int rc = ensure_scratch(h, V)) return rc;
    DevGraph& g = h->g;
    if (dmalloc(&g.out_len, (uint64_t)V + 1) || dmalloc(&g.in_len, (uint64_t)V + 1)) return DC_ERR_NOMEM;
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
    free_graph_arrays(h->g);
    free_decomp(h->d);
    if (int rc = ensure_scratch(h, V)) return rc;
    uint32_t *d_off = nullptr, *d_nbr = nullptr, *d_src = nullptr, *d_dst = nullptr;
    int32_t* d_deg = nullptr;
    int rc = DC_OK;
    if ((rc = dmalloc(&d_off, (uint64_t)V + 1)) || (rc = dmalloc(&d_nbr, nbr_len)) || (rc = dmalloc(&d_deg, V)) ||
        (rc = dmalloc(&d_src, E)) || (rc = dmalloc(&d_dst, E))) {
        dfree(d_off); dfree(d_nbr); dfree(d_deg); dfree(d_src); dfree(d_dst);
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
        dfree(d_off); dfree(d_nbr); dfree(d_deg); dfree(d_src); dfree(d_dst);
        return set_error(DC_ERR_INVALID, "binary graph: out-degrees sum to %llu, header says %llu", acc,
                         (unsigned long long)E);
    }
    cudaMemcpyAsync(s->tmp64, eo.data(), sizeof(unsigned long long) * ((size_t)V + 1), cudaMemcpyHostToDevice,
                    h->stream);
    k_csr_to_edges<<<grid_for(h, (uint64_t)V * 32), kThreads, 0, h->stream>>>(
        V, d_off, d_deg, (const unsigned long long*)s->tmp64, d_nbr, d_src, d_dst, 0);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    dfree(d_off);
    dfree(d_nbr);
    dfree(d_deg);
    if (e != cudaSuccess) {
        dfree(d_src); dfree(d_dst);
        return set_error(DC_ERR_CUDA, "binary graph upload failed: %s", cudaGetErrorString(e));
    }
    rc = build_from_device_edges(h, V, E, d_src, d_dst);
    cudaStreamSynchronize(h->stream);
    dfree(d_src);
    dfree(d_dst);
    return rc;
}

// which: 0 = kmax pass (peel in-degree), 1 = row pass (peel out-degree)
int run_peel(dc_graph* h, int which, const int32_t* member, int32_t k, int32_t* d_val, int32_t* maxval, int sync) {
    DevGraph& g = h->g;
    Scratch* s = h->scratch;
    PeelParams p;
    p.V = g.V;
    if (which == 0) {
        p.a_off = g.in_off; p.a_len = g.in_len; p.a_nbr = g.in_nbr;
        p.b_off = g.out_off; p.b_len = g.out_len; p.b_nbr = g.out_nbr;
    } else {
        p.a_off = g.out_off; p.a_len = g.out_len; p.a_nbr = g.out_nbr;
        p.b_off = g.in_off; p.b_len = g.in_len; p.b_nbr = g.in_nbr;
    }
    p.member = member;
    p.k = k;
    p.key = s->key;
    p.cdeg = s->cdeg;
    p.val = d_val;
    p.rem0 = s->rem0;
    p.rem1 = s->rem1;
    p.q.slots = s->ring;
    p.q.mask = s->ring_mask;
    p.ctl = h->ctl;
    DC_CUDA(cudaMemsetAsync(s->ring, 0xFF, sizeof(uint32_t) * ((uint64_t)s->ring_mask + 1), h->stream));
    void* args[] = {&p};
    if (int rc = coop_launch(h, (const void*)k_peel, args, kThreads, "peel")) return rc;
    if (!sync) return DC_OK;
    EngineCtl hc;
    if (int rc = check_ctl(h, &hc, "peel")) return rc;
    if (maxval) *maxval = hc.maxval;
    return DC_OK;
}

static int build_skyline_from_log(dc_graph* h, uint64_t nlog) {
    Scratch* s = h->scratch;
    Decomp& d = h->d;
    uint32_t V = h->g.V;
    unsigned long long* cnt = (unsigned long long*)s->tmp64;
    k_set_one<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, cnt);
    if (nlog) k_sky_count<<<grid_for(h, nlog), kThreads, 0, h->stream>>>(V, nlog, s->log_v, cnt);
    if (int rc = scan_tmp64(h, V)) return rc;
    uint64_t total = (uint64_t)V + nlog;
    if (d.corner_cap < total) {
        dfree(d.sky_k);
        dfree(d.sky_l);
        if (dmalloc(&d.sky_k, total) || dmalloc(&d.sky_l, total)) return DC_ERR_NOMEM;
        d.corner_cap = total;
    }
    if (!d.sky_off && dmalloc(&d.sky_off, (uint64_t)V + 1)) return DC_ERR_NOMEM;
    k_sky_fill_row0<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, cnt, s->row0, d.sky_k, d.sky_l, s->cursor);
    if (nlog)
        k_sky_fill_log<<<grid_for(h, nlog), kThreads, 0, h->stream>>>(nlog, s->log_v, s->log_k, s->log_l, cnt, d.sky_k,
                                                                      d.sky_l, s->cursor);
    k_sky_sort<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, cnt, d.sky_k, d.sky_l, d.sky_off);
    d.n_corners = total;
    DC_CUDA(cudaGetLastError());
    return DC_OK;
}

static int ensure_rows(dc_graph* h, uint64_t elems) {
    Decomp& d = h->d;
    if (d.rows_cap >= elems && d.rows) return DC_OK;
    dfree(d.rows);
    d.rows_cap = 0;
    if (dmalloc(&d.rows, elems)) return DC_ERR_NOMEM;
    d.rows_cap = elems;
    return DC_OK;
}

int expand_rows(dc_graph* h, uint32_t k0, uint32_t n, int32_t* d_dst) {
    Decomp& d = h->d;
    if (!d.valid) return set_error(DC_ERR_STATE, "no decomposition on this graph");
    if (n == 0) return DC_OK;
    k_expand<<<grid_for(h, h->g.V), kThreads, 0, h->stream>>>(h->g.V, k0, n, d.kmax_v, d.sky_off, d.sky_k, d.sky_l,
                                                               d_dst);
    DC_CUDA(cudaGetLastError());
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
    if (!d.kmax_v && dmalloc(&d.kmax_v, (uint64_t)V + 1)) return DC_ERR_NOMEM;
    if (V == 0) {
        d.kmax = 0;
        d.lmax = 0;
        d.n_corners = 0;
        if (!d.sky_off && dmalloc(&d.sky_off, 1)) return DC_ERR_NOMEM;
        DC_CUDA(cudaMemsetAsync(d.sky_off, 0, sizeof(uint32_t), h->stream));
        d.valid = true;
        return DC_OK;
    }
    cudaEventRecord(h->ev[0], h->stream);
    int32_t K = 0;
    if (int rc = run_peel(h, 0, nullptr, 0, d.kmax_v, &K, 1)) return rc;
    cudaEventRecord(h->ev[1], h->stream);
    d.kmax = K;
    if (method == 1) {
        // one fresh peel per row (the reference's schedule, main.cu:238-244)
        if (int rc = ensure_rows(h, (uint64_t)(K + 1) * V)) return rc;
        int32_t lm = 0;
        for (int32_t k = 0; k <= K; ++k) {
            int32_t mv = 0;
            if (int rc = run_peel(h, 1, k == 0 ? nullptr : d.kmax_v, k, d.rows + (uint64_t)k * V, &mv, 1)) return rc;
        }
        EngineCtl hc;
        if (int rc = check_ctl(h, &hc, "row peel")) return rc;
        int* dmax = (int*)s->cursor;
        DC_CUDA(cudaMemsetAsync(dmax, 0, sizeof(int), h->stream));
        k_max_reduce<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.rows, dmax);
        DC_CUDA(cudaMemcpyAsync(&lm, dmax, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        cudaEventRecord(h->ev[2], h->stream);
        cudaEventRecord(h->ev[3], h->stream);
        // skyline from rows
        unsigned long long* cnt = (unsigned long long*)s->tmp64;
        k_rows_corner_count<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, K, d.kmax_v, d.rows, cnt);
        if (int rc = scan_tmp64(h, V)) return rc;
        unsigned long long total = 0;
        DC_CUDA(cudaMemcpyAsync(&total, s->tmp64 + V, sizeof(total), cudaMemcpyDeviceToHost, h->stream));
        DC_CUDA(cudaStreamSynchronize(h->stream));
        if (d.corner_cap < total) {
            dfree(d.sky_k);
            dfree(d.sky_l);
            if (dmalloc(&d.sky_k, total) || dmalloc(&d.sky_l, total)) return DC_ERR_NOMEM;
            d.corner_cap = total;
        }
        if (!d.sky_off && dmalloc(&d.sky_off, (uint64_t)V + 1)) return DC_ERR_NOMEM;
        k_rows_corner_fill<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, d.rows, cnt, d.sky_k, d.sky_l,
                                                                        d.sky_off);
        d.n_corners = total;
        d.lmax = lm;
        d.rows_valid = true;
        cudaEventRecord(h->ev[4], h->stream);
        cudaEventRecord(h->ev[5], h->stream);
        DC_CUDA(cudaStreamSynchronize(h->stream));
        d.valid = true;
        return DC_OK;
    }
    // ---- method 0: row 0 by peel, rows 1..K by incremental transitions
    int32_t l0 = 0;
    if (int rc = run_peel(h, 1, nullptr, 0, s->row0, &l0, 1)) return rc;
    cudaEventRecord(h->ev[2], h->stream);
    d.lmax = l0;
    // order by kmax descending; ck[k] = |{v : kmax >= k}|
    if (s->ck_cap < (uint32_t)K + 2) {
        dfree(s->ck);
        if (dmalloc(&s->ck, (uint64_t)K + 2)) return DC_ERR_NOMEM;
        s->ck_cap = K + 2;
    }
    uint32_t* hist = s->cursor;
    DC_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * ((uint64_t)K + 2), h->stream));
    k_kmax_hist<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, hist);
    std::vector<uint32_t> hh((size_t)K + 2), ck((size_t)K + 2), start((size_t)K + 2);
    DC_CUDA(cudaMemcpyAsync(hh.data(), hist, sizeof(uint32_t) * ((size_t)K + 2), cudaMemcpyDeviceToHost, h->stream));
    // corner bound
    unsigned long long* acc = (unsigned long long*)s->tmp64;
    DC_CUDA(cudaMemsetAsync(acc, 0, sizeof(unsigned long long), h->stream));
    k_corner_bound<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, s->row0, acc);
    unsigned long long bound = 0;
    DC_CUDA(cudaMemcpyAsync(&bound, acc, sizeof(bound), cudaMemcpyDeviceToHost, h->stream));
    DC_CUDA(cudaStreamSynchronize(h->stream));
    {
        uint64_t run = 0;
        ck[K + 1] = 0;
        for (int32_t k = K; k >= 0; --k) {
            start[k] = (uint32_t)run;  // descending order: bucket K first
            run += hh[k];
            ck[k] = (uint32_t)run;
        }
    }
    DC_CUDA(cudaMemcpyAsync(s->ck, ck.data(), sizeof(uint32_t) * ((size_t)K + 2), cudaMemcpyHostToDevice, h->stream));
    DC_CUDA(cudaMemcpyAsync(hist, start.data(), sizeof(uint32_t) * ((size_t)K + 2), cudaMemcpyHostToDevice, h->stream));
    k_order_scatter<<<grid_for(h, V), kThreads, 0, h->stream>>>(V, d.kmax_v, hist, s->order);
    // log capacity = corner bound
    uint64_t lc = bound + 1;
    if (s->log_cap < lc) {
        dfree(s->log_v);
        dfree(s->log_k);
        dfree(s->log_l);
        if (dmalloc(&s->log_v, lc) || dmalloc(&s->log_k, lc) || dmalloc(&s->log_l, lc)) return DC_ERR_NOMEM;
        s->log_cap = lc;
    }
    // transition state
    DC_CUDA(cudaMemcpyAsync(s->cur, s->row0, sizeof(int32_t) * V, cudaMemcpyDeviceToDevice, h->stream));
    k_cnt_in_init<<<grid_for(h, (uint64_t)V * 32), kThreads, 0, h->stream>>>(V, g.in_off, g.in_len, g.in_nbr, s->cur,
                                                                             s->key);
    DC_CUDA(cudaMemsetAsync(s->mark, 0, sizeof(uint32_t) * V, h->stream));
    DC_CUDA(cudaMemsetAsync(s->stamp, 0xFF, sizeof(int32_t) * V, h->stream));
    DC_CUDA(cudaMemsetAsync(s->ring, 0xFF, sizeof(uint32_t) * ((uint64_t)s->ring_mask + 1), h->stream));
    TransParams tp;
    tp.V = V;
    tp.out_off = g.out_off; tp.out_len = g.out_len; tp.out_nbr = g.out_nbr;
    tp.in_off = g.in_off; tp.in_len = g.in_len; tp.in_nbr = g.in_nbr;
    tp.kmax = d.kmax_v;
    tp.K = K;
    tp.order = s->order;
    tp.ck = s->ck;
    tp.cur = s->cur;
    tp.cnt_in = s->key;
    tp.mark = s->mark;
    tp.stamp = s->stamp;
    tp.logidx = s->logidx;
    tp.log_v = s->log_v;
    tp.log_k = s->log_k;
    tp.log_l = s->log_l;
    tp.log_cap = s->log_cap;
    tp.q.slots = s->ring;
    tp.q.mask = s->ring_mask;
    tp.ctl = h->ctl;
    cudaEventRecord(h->ev[3], h->stream);
    uint64_t nlog = 0;
    if (K >= 1) {
        void* args[] = {&tp};
        if (int rc = coop_launch(h, (const void*)k_transitions, args, kThreads, "transitions")) return rc;
        EngineCtl hc;
        if (int rc = check_ctl(h, &hc, "transitions")) return rc;
        nlog = hc.log_count;
        h->stat_evals = hc.evals;
        h->stat_drops = hc.drops;
    }
    cudaEventRecord(h->ev[4], h->stream);
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
    cudaEventElapsedTime(&ms, h->ev[1], h->ev[2]);
    h->times.row0_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[3], h->ev[4]);
    h->times.trans_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[4], h->ev[5]);
    h->times.sky_ms = ms;
    cudaEventElapsedTime(&ms, h->ev[5], h->ev[6]);
    h->times.expand_ms = ms;
    return DC_OK;
}

}  // namespace dc
