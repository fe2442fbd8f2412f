// Local row repair after edge deletions.
//
// Deleting edges (and the vertices that leave C_k because their kmax fell)
// can only lower row values: new row k is the greatest fixpoint of the row-k
// operator of the updated graph that lies below old row k.  Each block takes
// whole rows k = 1..R from a counter and repairs one row at a time, starting
// from the old row (read from the old skyline) and touching only the vertices
// the deletions reach:
//
//   seeds    the endpoints of deleted edges that are still in C_k, and the
//            neighbours that a vertex leaving C_k was supporting
//   evaluate l(x) = max L <= cur(x) with #{out-nbrs w in C_k, l(w) >= L} >= L
//            and #{in-nbrs u in C_k, l(u) >= L} >= k, by windowed histograms
//            over x's lists, neighbour values from the block's overrides or
//            the old skyline
//   drop     write the lower value, queue the neighbours whose support it
//            was (values in (new, old])
//
// Overrides and the work queue live in shared memory (one open-addressed
// table per block); a row that touches more vertices than the table holds
// aborts the repair and the caller recomputes the rows instead.  The changed
// (v, k, value) triples go to a log from which the new skyline is merged with
// the old one.
//
// The row semantics are those of the reference's per-row pass
// (KListInplace, main.cu:171-195, driven by dcore, main.cu:236-243); the
// reference itself re-peels rows after maintenance (maintenanceFast,
// main.cu:1735-1743) and its exact l-list maintenance is disabled code
// (main.cu:929-1242).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "dc_engine.cuh"
#include "dc_internal.h"

namespace dc {

extern std::atomic<unsigned long long> g_launches;

namespace {

constexpr int kRThreads = 256;
constexpr int kRWarps = kRThreads / 32;
constexpr int kHashBits = 13;
constexpr int kHash = 1 << kHashBits;  // vertices a block can touch in one row
constexpr unsigned kHashLimit = kHash * 3 / 4;  // more than this aborts the repair
constexpr uint32_t kEmptyKey = 0xFFFFFFFFu;
constexpr int kUnset = 0x7FFFFFFF;   // no override: the old value applies
constexpr uint32_t kEmptySlot = 0xFFFFFFFFu;
constexpr int kRWin = 64;

struct RepairParams {
    uint32_t V;
    const uint32_t* out_off;
    const int32_t* out_len;
    const uint32_t* out_nbr;
    const uint32_t* in_off;
    const int32_t* in_len;
    const uint32_t* in_nbr;
    const int32_t* kmax_new;
    const int32_t* kmax_old;
    const uint32_t* sky_off;  // old skyline
    const int32_t* sky_k;
    const int32_t* sky_l;
    const uint32_t* del_u;  // deleted edges u -> v (insertions: inserted edges)
    const uint32_t* del_v;
    uint32_t n_del;
    const uint32_t* leave;  // vertices whose kmax fell (insertions: rose)
    uint32_t n_leave;
    const int32_t* row0_new;  // insertions: row 0 after the batch
    unsigned long long deadline_ns;  // a block still busy this long after its start gives up (0: never)
    int32_t R;
    // captured batches: R and the vertex count of `leave` read on the device
    // when set, and a flag that must be nonzero for the kernel to act
    const int32_t* R_dev;
    const unsigned* n_leave_dev;
    const unsigned long long* deadline_dev;
    const int* run;
    uint32_t* log_v;
    int32_t* log_k;
    int32_t* log_l;
    unsigned long long log_cap;
    EngineCtl* ctl;  // level = row counter, log_count, error
};

template <int NW>
struct RowStateT {
    uint32_t key[kHash];
    int cur[kHash];
    unsigned st[kHash];  // 0 idle, 1 queued or being evaluated, 2 re-run requested
    uint32_t ring[kHash];
    unsigned qhead, qtail, used;
    int out;    // queued + running items
    int abort;  // table full, a wait ran out, or (insertions) the scan budget is spent
    int k;
    int hist[NW][2][kRWin];
    // one list scan shared by the block's idle warps (a hub's list): the
    // owner posts it, every warp waiting for work claims chunks of it
    unsigned job_busy;            // 0 free, 1 posted
    unsigned job_id;              // bumped per posted scan
    unsigned long long job_ctr;   // (job id << 32) | next chunk to claim
    unsigned job_done;            // chunks finished
    int job_support;              // release scans: neighbours at or above nv
    const uint32_t* job_a;
    int job_n, job_kind, job_k, job_lo, job_hi, job_first, job_nv, job_cap;
    unsigned job_nchunks;
    int* job_bins;
    // re-check sweep: hubs checked by the whole block after the others
    unsigned nbig;
    uint32_t bigv[32];
    int big_so, big_si;
};
using RowState = RowStateT<kRWarps>;

__device__ __forceinline__ int vld(const int* p) { return *(const volatile int*)p; }
__device__ __forceinline__ unsigned vldu(const unsigned* p) { return *(const volatile unsigned*)p; }

// Old row-k value of v: the last corner at or below k (binary search).
__device__ __forceinline__ int sky_at(const RepairParams& p, uint32_t v, int k) {
    uint32_t a = p.sky_off[v], b = p.sky_off[v + 1];
    int val = 0;
    while (a < b) {
        uint32_t m = (a + b) >> 1;
        if (p.sky_k[m] <= k) {
            val = p.sky_l[m];
            a = m + 1;
        } else {
            b = m;
        }
    }
    return val;
}

__device__ __forceinline__ unsigned hslot0(uint32_t v) { return (v * 2654435761u) >> (32 - kHashBits); }

// Table slot of v (inserting it when asked); -1 when absent / table full.
template <class St>
__device__ int h_slot(St& S, uint32_t v, bool insert) {
    unsigned i = hslot0(v) & (kHash - 1);
    for (int probe = 0; probe < kHash; ++probe) {
        uint32_t key = vldu(&S.key[i]);
        if (key == v) return (int)i;
        if (key == kEmptyKey) {
            if (!insert) return -1;
            uint32_t prev = atomicCAS(&S.key[i], kEmptyKey, v);
            if (prev == kEmptyKey) {
                if (atomicAdd(&S.used, 1u) >= kHashLimit) atomicExch(&S.abort, 1);
                return (int)i;
            }
            if (prev == v) return (int)i;
        }
        i = (i + 1) & (kHash - 1);
    }
    atomicExch(&S.abort, 1);
    return -1;
}

// Row-k value of w: -1 outside C_k, else the override or the old value.
template <class St>
__device__ __forceinline__ int rv(const RepairParams& p, St& S, uint32_t w, int k) {
    if (p.kmax_new[w] < k) return -1;
    int i = h_slot(S, w, false);
    if (i >= 0) {
        int c = vld(&S.cur[i]);
        if (c != kUnset) return c;
    }
    return sky_at(p, w, k);
}

template <class St>
__device__ __forceinline__ void enqueue(St& S, unsigned slot) {
    atomicAdd(&S.out, 1);
    unsigned pos = atomicAdd(&S.qtail, 1u);
    __threadfence_block();
    *(volatile uint32_t*)&S.ring[pos & (kHash - 1)] = slot;
}

// Any thread: asks for an evaluation of w at this row.
template <class St>
__device__ __forceinline__ void push(St& S, uint32_t w) {
    int slot = h_slot(S, w, true);
    if (slot < 0) return;
    unsigned old = atomicCAS(&S.st[slot], 0u, 1u);
    if (old == 0u) enqueue(S, (unsigned)slot);
    else if (old == 1u) atomicCAS(&S.st[slot], 1u, 2u);
}

// Row-k values of up to W vertices at once (rv for each w[q] with ok[q];
// -1 elsewhere): the table probes first, then the W binary searches over the
// old skyline in lockstep, so a lane has W independent chains of loads in
// flight instead of one.
template <int W, class St>
__device__ __forceinline__ void rvw(const RepairParams& p, St& S, const uint32_t w[W], const bool ok[W], int k,
                                    int out[W]) {
    uint32_t lo[W], hi[W];
    int val[W];
    bool need[W];
    int km[W];
#pragma unroll
    for (int q = 0; q < W; ++q) km[q] = ok[q] ? p.kmax_new[w[q]] : -1;
#pragma unroll
    for (int q = 0; q < W; ++q) {
        out[q] = -1;
        need[q] = false;
        lo[q] = hi[q] = 0;
        val[q] = 0;
        if (km[q] < k) continue;
        const int i = h_slot(S, w[q], false);
        if (i >= 0) {
            const int c = vld(&S.cur[i]);
            if (c != kUnset) {
                out[q] = c;
                continue;
            }
        }
        need[q] = true;
        lo[q] = p.sky_off[w[q]];
        hi[q] = p.sky_off[w[q] + 1];
    }
    for (;;) {
        bool any = false;
#pragma unroll
        for (int q = 0; q < W; ++q) {
            if (need[q] && lo[q] < hi[q]) {
                any = true;
                const uint32_t m = (lo[q] + hi[q]) >> 1;
                if (p.sky_k[m] <= k) {
                    val[q] = p.sky_l[m];
                    lo[q] = m + 1;
                } else {
                    hi[q] = m;
                }
            }
        }
        if (!any) break;
    }
#pragma unroll
    for (int q = 0; q < W; ++q)
        if (need[q]) out[q] = val[q];
}
constexpr int kRv = 8;  // lookups per lane in flight

// Converged warp: one histogram pass over a list for the window [lo, hi];
// values above hi land in the top bin on the first window only.  kRv
// entries per lane and step (rvw).
template <class St>
__device__ __forceinline__ void r_hist(const RepairParams& p, St& S, const uint32_t* a, int n, int k, int lo,
                                       int hi, bool first, int* bins) {
    const unsigned lane = threadIdx.x & 31u;
    int top = 0;
    for (int b = 0; b < n; b += 32 * kRv) {
        uint32_t w[kRv];
        bool ok[kRv];
        int x[kRv];
#pragma unroll
        for (int q = 0; q < kRv; ++q) {
            const int e = b + 32 * q + (int)lane;
            ok[q] = e < n;
            w[q] = ok[q] ? a[e] : 0;
        }
        rvw<kRv>(p, S, w, ok, k, x);
#pragma unroll
        for (int q = 0; q < kRv; ++q) {
            if (!ok[q]) continue;
            if (x[q] > hi) top += first;
            else if (x[q] == hi) ++top;
            else if (x[q] >= lo) atomicAdd(&bins[x[q] - lo], 1);
        }
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) top += __shfl_xor_sync(0xFFFFFFFFu, top, s);
    if (lane == 0 && top) atomicAdd(&bins[hi - lo], top);
}

// Converged warp: how many entries of a list hold at least val (rvw).
template <class St>
__device__ __forceinline__ int r_count_at_least(const RepairParams& p, St& S, const uint32_t* a, int n, int k,
                                                int val) {
    int cnt = 0;
    for (int b = 0; b < n; b += 32 * kRv) {
        uint32_t w[kRv];
        bool ok[kRv];
        int x[kRv];
#pragma unroll
        for (int q = 0; q < kRv; ++q) {
            const int e = b + 32 * q + (int)(threadIdx.x & 31u);
            ok[q] = e < n;
            w[q] = ok[q] ? a[e] : 0;
        }
        rvw<kRv>(p, S, w, ok, k, x);
#pragma unroll
        for (int q = 0; q < kRv; ++q) cnt += ok[q] && x[q] >= val;
    }
    return cnt;
}

// Converged warp, after x dropped from cap to nv (value already written):
// queues the neighbours in a list whose value lies in (nv, cap] and returns
// how many neighbours hold at least nv, read after the write.  The recount
// closes the race in which x and a neighbour drop at the same time and each
// read the other's old value: whichever reads second sees the other's write.
template <class St>
__device__ __forceinline__ int r_release(const RepairParams& p, St& S, const uint32_t* a, int n, int k, int nv,
                                         int cap) {
    int support = 0;
    for (int b = 0; b < n && !vld(&S.abort); b += 32 * kRv) {
        uint32_t w[kRv];
        bool ok[kRv];
        int x[kRv];
#pragma unroll
        for (int q = 0; q < kRv; ++q) {
            const int e = b + 32 * q + (int)(threadIdx.x & 31u);
            ok[q] = e < n;
            w[q] = ok[q] ? a[e] : 0;
        }
        rvw<kRv>(p, S, w, ok, k, x);
#pragma unroll
        for (int q = 0; q < kRv; ++q) {
            if (!ok[q]) continue;
            support += x[q] >= nv;
            if (x[q] > nv && x[q] <= cap) push(S, w[q]);
        }
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) support += __shfl_xor_sync(0xFFFFFFFFu, support, s);
    return support;
}

// ---- list scans shared by the block -------------------------------------
// A hub's lists hold up to ~10^5 entries; one warp scanning them leaves the
// block's other warps idle in the queue.  A warp about to scan a list longer
// than kHubMin posts the scan in the block's job slot instead; warps waiting
// for work claim chunks of it (r_take), the owner claims chunks too and then
// waits until every chunk is done.  A chunk is claimed by a CAS on
// (job id, next chunk), so a warp that read an older job's fields can never
// claim a chunk of a newer one; the owner reuses the slot only after all
// chunks of its job are done, so no claimer still reads its fields.
constexpr int kHubMin = 4096;
constexpr int kChunk = 2048;

// Converged warp: chunk [c0, c1) of the posted scan.  kind 0: histogram of
// the window [lo, hi] into bins (r_hist); kind 1: release (r_release), the
// support count added to job_support.
template <class St>
__device__ void job_chunk(const RepairParams& p, St& S, int kind, const uint32_t* a, int c0, int c1, int k, int lo,
                          int hi, bool first, int nv, int cap, int* bins) {
    const unsigned lane = threadIdx.x & 31u;
    int acc = 0;  // histogram: top-bin count; release: support
    for (int b = c0; b < c1 && !vld(&S.abort); b += 32 * kRv) {
        uint32_t w[kRv];
        bool ok[kRv];
        int x[kRv];
#pragma unroll
        for (int q = 0; q < kRv; ++q) {
            const int e = b + 32 * q + (int)lane;
            ok[q] = e < c1;
            w[q] = ok[q] ? a[e] : 0;
        }
        rvw<kRv>(p, S, w, ok, k, x);
#pragma unroll
        for (int q = 0; q < kRv; ++q) {
            if (!ok[q]) continue;
            if (kind == 0) {
                if (x[q] > hi) acc += first;
                else if (x[q] == hi) ++acc;
                else if (x[q] >= lo) atomicAdd(&bins[x[q] - lo], 1);
            } else {
                acc += x[q] >= nv;
                if (x[q] > nv && x[q] <= cap) push(S, w[q]);
            }
        }
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, s);
    if (lane == 0 && acc) {
        if (kind == 0) atomicAdd(&bins[hi - lo], acc);
        else atomicAdd(&S.job_support, acc);
    }
}

// Converged warp: claims and scans chunks of the posted job until none is
// left.
template <class St>
__device__ void job_help(const RepairParams& p, St& S) {
    const unsigned lane = threadIdx.x & 31u;
    for (;;) {
        int chunk = -1;
        unsigned long long aptr = 0;
        int n = 0, kind = 0, k = 0, lo = 0, hi = 0, first = 0, nv = 0, cap = 0;
        unsigned long long bptr = 0;
        if (lane == 0 && vldu(&S.job_busy)) {
            const unsigned id = vldu(&S.job_id);
            __threadfence_block();
            aptr = (unsigned long long)*(const uint32_t* volatile*)&S.job_a;
            n = vld(&S.job_n);
            kind = vld(&S.job_kind);
            k = vld(&S.job_k);
            lo = vld(&S.job_lo);
            hi = vld(&S.job_hi);
            first = vld(&S.job_first);
            nv = vld(&S.job_nv);
            cap = vld(&S.job_cap);
            bptr = (unsigned long long)*(int* volatile*)&S.job_bins;
            const unsigned nch = vldu(&S.job_nchunks);
            __threadfence_block();
            for (int tries = 0; tries < 64; ++tries) {
                const unsigned long long c = *(volatile unsigned long long*)&S.job_ctr;
                if ((unsigned)(c >> 32) != id || (unsigned)c >= nch) break;
                if (atomicCAS(&S.job_ctr, c, c + 1) == c) {
                    chunk = (int)(unsigned)c;
                    break;
                }
            }
        }
        chunk = __shfl_sync(0xFFFFFFFFu, chunk, 0);
        if (chunk < 0) return;
        aptr = __shfl_sync(0xFFFFFFFFu, aptr, 0);
        bptr = __shfl_sync(0xFFFFFFFFu, bptr, 0);
        n = __shfl_sync(0xFFFFFFFFu, n, 0);
        kind = __shfl_sync(0xFFFFFFFFu, kind, 0);
        k = __shfl_sync(0xFFFFFFFFu, k, 0);
        lo = __shfl_sync(0xFFFFFFFFu, lo, 0);
        hi = __shfl_sync(0xFFFFFFFFu, hi, 0);
        first = __shfl_sync(0xFFFFFFFFu, first, 0);
        nv = __shfl_sync(0xFFFFFFFFu, nv, 0);
        cap = __shfl_sync(0xFFFFFFFFu, cap, 0);
        const int c0 = chunk * kChunk, c1 = min(n, c0 + kChunk);
        job_chunk(p, S, kind, (const uint32_t*)aptr, c0, c1, k, lo, hi, first != 0, nv, cap, (int*)bptr);
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            atomicAdd(&S.job_done, 1u);
        }
    }
}

// A posted job with chunks left to claim (a hint; the claim decides).
template <class St>
__device__ __forceinline__ bool job_open(St& S) {
    if (!vldu(&S.job_busy)) return false;
    const unsigned long long c = *(volatile unsigned long long*)&S.job_ctr;
    return (unsigned)(c >> 32) == vldu(&S.job_id) && (unsigned)c < vldu(&S.job_nchunks);
}

// Converged warp: a scan of list a (kind 0 histogram, kind 1 release) shared
// with the block's idle warps when the list is long and the job slot free,
// else scanned alone.  Returns the release's support count (kind 1).
template <class St>
__device__ int scan_shared(const RepairParams& p, St& S, int kind, const uint32_t* a, int n, int k, int lo, int hi,
                           bool first, int nv, int cap, int* bins) {
    const unsigned lane = threadIdx.x & 31u;
    bool mine = false;
    if (n > kHubMin) {
        if (lane == 0) mine = atomicCAS(&S.job_busy, 0u, 1u) == 0u;
        mine = __shfl_sync(0xFFFFFFFFu, mine, 0);
    }
    if (!mine) {
        if (kind == 0) {
            r_hist(p, S, a, n, k, lo, hi, first, bins);
            return 0;
        }
        return r_release(p, S, a, n, k, nv, cap);
    }
    const unsigned nch = (unsigned)((n + kChunk - 1) / kChunk);
    if (lane == 0) {
        S.job_a = a;
        S.job_n = n;
        S.job_kind = kind;
        S.job_k = k;
        S.job_lo = lo;
        S.job_hi = hi;
        S.job_first = first;
        S.job_nv = nv;
        S.job_cap = cap;
        S.job_bins = bins;
        S.job_nchunks = nch;
        S.job_done = 0;
        S.job_support = 0;
        const unsigned id = S.job_id + 1;
        __threadfence_block();
        *(volatile unsigned*)&S.job_id = id;
        __threadfence_block();
        atomicExch(&S.job_ctr, (unsigned long long)id << 32);
    }
    __syncwarp();
    job_help(p, S);  // the owner scans chunks too
    int support = 0;
    if (lane == 0) {
        const unsigned long long t0 = gtimer();
        for (unsigned spins = 0; vldu(&S.job_done) < nch; ++spins) {
            if ((spins & 63) == 63 && gtimer() - t0 > wait_limit(p.ctl)) {
                set_dev_error(p.ctl, DC_DEV_ERR_TIMEOUT, 43);
                atomicExch(&S.abort, 1);
                break;
            }
            __nanosleep(32);
        }
        __threadfence_block();
        support = vld(&S.job_support);
        atomicExch(&S.job_busy, 0u);
    }
    __syncwarp();
    return __shfl_sync(0xFFFFFFFFu, support, 0);
}

// Converged warp: takes a queued slot; false when the row is finished or
// abandoned.
template <class St>
__device__ bool r_take(const RepairParams& p, St& S, unsigned* slot) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(&S.qhead, 1u);
    unsigned long long t0 = 0;
    unsigned spins = 0;
    for (;;) {
        int state = 0;  // 1 item, 2 row finished or abandoned, 3 help with a shared scan
        unsigned got = 0;
        if (lane == 0) {
            volatile uint32_t* cell = (volatile uint32_t*)&S.ring[t & (kHash - 1)];
            for (;; ++spins) {
                uint32_t it = *cell;
                if (it != kEmptySlot) {
                    *cell = kEmptySlot;
                    got = it;
                    state = 1;
                    break;
                }
                if (vld(&S.out) == 0 || vld(&S.abort) || ld_vol(&p.ctl->error)) {
                    state = 2;
                    break;
                }
                if (job_open(S)) {
                    state = 3;
                    spins = 0;  // helping is progress: the wait's clock restarts
                    break;
                }
                if (spins == 64) t0 = gtimer();
                if (spins > 64 && (spins & 63) == 0 && gtimer() - t0 > wait_limit(p.ctl)) {
                    set_dev_error(p.ctl, DC_DEV_ERR_TIMEOUT, 40);
                    atomicExch(&S.abort, 1);
                    state = 2;
                    break;
                }
                if (spins > 16) __nanosleep(64);
            }
        }
        state = __shfl_sync(0xFFFFFFFFu, state, 0);
        if (state == 3) {
            job_help(p, S);
            continue;
        }
        *slot = __shfl_sync(0xFFFFFFFFu, got, 0);
        __threadfence_block();
        return state == 1;
    }
}

__global__ void __launch_bounds__(kRThreads, 1) k_row_repair(RepairParams p) {
    if (p.run && !*p.run) return;
    const int32_t R = p.R_dev ? *p.R_dev : p.R;
    const uint32_t n_leave = p.n_leave_dev ? *p.n_leave_dev : p.n_leave;
    const unsigned long long deadline = p.deadline_dev ? *p.deadline_dev : p.deadline_ns;
    extern __shared__ __align__(16) unsigned char s_raw[];
    RowState& S = *reinterpret_cast<RowState*>(s_raw);
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const unsigned long long t_start = gtimer();
    int* ho = S.hist[wib][0];
    int* hi_ = S.hist[wib][1];
    if (threadIdx.x == 0) {
        S.job_busy = 0;
        S.job_id = 0;
        S.job_ctr = 0;
        S.job_nchunks = 0;
    }
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) S.k = ld_vol(&p.ctl->error) ? R + 1 : atomicAdd(&p.ctl->level, 1) + 1;
        for (int i = threadIdx.x; i < kHash; i += kRThreads) {
            S.key[i] = kEmptyKey;
            S.cur[i] = kUnset;
            S.st[i] = 0;
            S.ring[i] = kEmptySlot;
        }
        if (threadIdx.x == 0) {
            S.qhead = S.qtail = S.used = 0;
            S.out = 1;  // held by the seeding phase
            S.abort = 0;
        }
        __syncthreads();
        const int k = S.k;
        if (k > R) break;
        // ---- seeds: endpoints of deleted edges still in C_k
        for (uint32_t i = threadIdx.x; i < p.n_del && !vld(&S.abort); i += kRThreads) {
            uint32_t u = p.del_u[i], v = p.del_v[i];
            if (p.kmax_new[u] >= k) push(S, u);
            if (p.kmax_new[v] >= k) push(S, v);
        }
        // ---- vertices leaving C_k: the neighbours they supported
        for (uint32_t i = wib; i < n_leave; i += kRWarps) {
            if (__any_sync(0xFFFFFFFFu, vld(&S.abort))) break;
            uint32_t x = p.leave[i];
            if (!(p.kmax_old[x] >= k && p.kmax_new[x] < k)) continue;
            int ox = sky_at(p, x, k);
            const uint32_t* a = p.out_nbr + p.out_off[x];
            int n = p.out_len[x];
            for (int e = (int)lane; e < n && !vld(&S.abort); e += 32) {
                uint32_t z = a[e];
                int vz = rv(p, S, z, k);
                if (vz >= 1 && vz <= ox) push(S, z);
            }
            a = p.in_nbr + p.in_off[x];
            n = p.in_len[x];
            for (int e = (int)lane; e < n && !vld(&S.abort); e += 32) {
                uint32_t y = a[e];
                int vy = rv(p, S, y, k);
                if (vy >= 1 && vy <= ox) push(S, y);
            }
        }
        for (int sweep = 0;; ++sweep) {
            __syncthreads();
            if (threadIdx.x == 0) atomicSub(&S.out, 1);
            __syncthreads();
            // ---- drain
            unsigned slot;
            while (r_take(p, S, &slot)) {
                if (lane == 0 && deadline && gtimer() - t_start > deadline) atomicExch(&S.abort, 1);
                const uint32_t x = vldu(&S.key[slot]);
                int cap = vld(&S.cur[slot]);
                if (cap == kUnset) cap = sky_at(p, x, k);
                int nv = cap;
                if (cap >= 1 && p.kmax_new[x] >= k) {
                    const uint32_t* ao = p.out_nbr + p.out_off[x];
                    const uint32_t* ai = p.in_nbr + p.in_off[x];
                    const int no = p.out_len[x], ni = p.in_len[x];
                    int carry_o = 0, carry_i = 0, hi = cap;
                    bool first = true;
                    for (;;) {
                        const int lo = max(0, hi - (kRWin - 1));
                        ho[lane] = 0;
                        ho[lane + 32] = 0;
                        hi_[lane] = 0;
                        hi_[lane + 32] = 0;
                        __syncwarp();
                        scan_shared(p, S, 0, ao, no, k, lo, hi, first, 0, 0, ho);
                        scan_shared(p, S, 0, ai, ni, k, lo, hi, first, 0, 0, hi_);
                        __syncwarp();
                        int found = -1;
                        if (lane == 0) {
                            for (int L = hi; L >= lo; --L) {
                                carry_o += ho[L - lo];
                                carry_i += hi_[L - lo];
                                if (carry_o >= L && carry_i >= k) {
                                    found = L;
                                    break;
                                }
                            }
                        }
                        found = __shfl_sync(0xFFFFFFFFu, found, 0);
                        carry_o = __shfl_sync(0xFFFFFFFFu, carry_o, 0);
                        carry_i = __shfl_sync(0xFFFFFFFFu, carry_i, 0);
                        __syncwarp();
                        if (found >= 0) {
                            nv = found;
                            break;
                        }
                        if (lo == 0) {  // a member keeps at least 0
                            nv = 0;
                            break;
                        }
                        hi = lo - 1;
                        first = false;
                    }
                    if (nv < cap) {
                        if (lane == 0) atomicExch(&S.cur[slot], nv);
                        __syncwarp();
                        __threadfence_block();
                        const int so = scan_shared(p, S, 1, ao, no, k, 0, 0, false, nv, cap, nullptr);
                        const int si = scan_shared(p, S, 1, ai, ni, k, 0, 0, false, nv, cap, nullptr);
                        // a neighbour fell below nv meanwhile: evaluate x again
                        if (lane == 0 && nv >= 1 && (so < nv || si < k)) atomicCAS(&S.st[slot], 1u, 2u);
                    }
                }
                __syncwarp();
                if (lane == 0) {
                    if (atomicCAS(&S.st[slot], 1u, 0u) == 2u) {
                        atomicExch(&S.st[slot], 1u);
                        enqueue(S, slot);
                    }
                    __threadfence_block();
                    atomicSub(&S.out, 1);
                }
                __syncwarp();
            }
            __syncthreads();
            if (S.abort) break;
            if (sweep == 32) {  // bounded: a row that keeps failing is recomputed
                if (threadIdx.x == 0) S.abort = 1;
                __syncthreads();
                break;
            }
            // ---- the row is quiet: every touched vertex must hold its value
            // against the final values of its neighbours; queue any that does
            // not and drain again
            if (threadIdx.x == 0) {
                S.qhead = S.qtail = 0;
                S.out = 1;  // held by the sweep
                S.k = 0;    // vertices found unstable
            }
            for (int i = threadIdx.x; i < kHash; i += kRThreads) S.ring[i] = kEmptySlot;
            if (threadIdx.x == 0) S.nbig = 0;
            __syncthreads();
            for (int i = wib; i < kHash; i += kRWarps) {
                const uint32_t x = S.key[i];
                if (x == kEmptyKey || p.kmax_new[x] < k) continue;
                int val = S.cur[i];
                if (val == kUnset) val = sky_at(p, x, k);
                if (val < 1) continue;
                // a hub is checked by the whole block below (up to 32 per sweep)
                if (p.out_len[x] + p.in_len[x] > 2 * kHubMin) {
                    unsigned b = 0;
                    if (lane == 0) b = atomicAdd(&S.nbig, 1u);
                    b = __shfl_sync(0xFFFFFFFFu, b, 0);
                    if (b < 32u) {
                        if (lane == 0) S.bigv[b] = (uint32_t)i;
                        continue;
                    }
                }
                int so = 0, si = 0;
                const uint32_t* ao = p.out_nbr + p.out_off[x];
                const uint32_t* ai = p.in_nbr + p.in_off[x];
                so = r_count_at_least(p, S, ao, p.out_len[x], k, val);
                si = r_count_at_least(p, S, ai, p.in_len[x], k, val);
    #pragma unroll
                for (int s = 16; s; s >>= 1) {
                    so += __shfl_xor_sync(0xFFFFFFFFu, so, s);
                    si += __shfl_xor_sync(0xFFFFFFFFu, si, s);
                }
                if (lane == 0 && (so < val || si < k)) {
                    atomicAdd(&S.k, 1);
                    push(S, x);
                }
            }
            __syncthreads();
            const unsigned nbig = min(S.nbig, 32u);
            for (unsigned bi = 0; bi < nbig; ++bi) {
                const uint32_t slot = S.bigv[bi];
                const uint32_t x = S.key[slot];
                int val = S.cur[slot];
                if (val == kUnset) val = sky_at(p, x, k);
                if (threadIdx.x == 0) {
                    S.big_so = 0;
                    S.big_si = 0;
                }
                __syncthreads();
                // every warp counts its share of both lists
                for (int side = 0; side < 2; ++side) {
                    const uint32_t* a = side ? p.in_nbr + p.in_off[x] : p.out_nbr + p.out_off[x];
                    const int n = side ? p.in_len[x] : p.out_len[x];
                    int cnt = 0;
                    for (int b = (int)wib * 32 * kRv; b < n; b += kRWarps * 32 * kRv) {
                        uint32_t w[kRv];
                        bool ok[kRv];
                        int xv[kRv];
#pragma unroll
                        for (int q = 0; q < kRv; ++q) {
                            const int e = b + 32 * q + (int)lane;
                            ok[q] = e < n;
                            w[q] = ok[q] ? a[e] : 0;
                        }
                        rvw<kRv>(p, S, w, ok, k, xv);
#pragma unroll
                        for (int q = 0; q < kRv; ++q) cnt += ok[q] && xv[q] >= val;
                    }
#pragma unroll
                    for (int s = 16; s; s >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, s);
                    if (lane == 0 && cnt) atomicAdd(side ? &S.big_si : &S.big_so, cnt);
                }
                __syncthreads();
                if (threadIdx.x == 0 && (S.big_so < val || S.big_si < k)) {
                    atomicAdd(&S.k, 1);
                    push(S, x);
                }
                __syncthreads();
            }
            const bool again = S.k != 0;
            __syncthreads();
            if (threadIdx.x == 0) S.k = k;
            if (!again) {
                __syncthreads();
                break;
            }
        }
        __syncthreads();
        if (S.abort) {
            if (threadIdx.x == 0) set_dev_error(p.ctl, DC_DEV_ERR_CAPACITY, 41);
            break;
        }
        // ---- changed values of this row to the log
        for (int i = threadIdx.x; i < kHash; i += kRThreads) {
            uint32_t v = S.key[i];
            int c = S.cur[i];
            if (v == kEmptyKey || c == kUnset) continue;
            if (c >= sky_at(p, v, k)) continue;
            unsigned long long li = atomicAdd(&p.ctl->log_count, 1u);
            if (li < p.log_cap) {
                p.log_v[li] = v;
                p.log_k[li] = k;
                p.log_l[li] = c;
            } else {
                set_dev_error(p.ctl, DC_DEV_ERR_CAPACITY, 42);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// insertions
// ---------------------------------------------------------------------------
// Inserting edges (and vertices joining C_k because their kmax rose) can only
// raise row values.  Row k is repaired after row k-1 (one block takes the rows
// in order), because the new row k-1 bounds the new row k from above:
//
//   region   grown from the seeds -- endpoints of inserted edges with both
//            ends in C_k, and the vertices that joined C_k -- along edges
//            (either direction) to every member w with
//                old_k(w) < bound(x)   for a region vertex x next to it, and
//                old_k(w) < new row_{k-1}(w)   (w could rise at all);
//            each region vertex starts at its bound, new row_{k-1}
//   refine   the greatest fixpoint below the bounds, as for deletions, with
//            every vertex outside the region fixed at its old value
//
// Why the region holds every vertex that rises: let w rise to L > old_k(w).
// In the new (k, L)-core, the vertices that were not in the old one split
// into groups joined by edges; a group without a seed would, with the old
// (k, L)-core, already satisfy the (k, L) conditions in the old graph (its
// members' edges are all old and reach no other group), so it would have
// been in the old core.  Hence a path of risen vertices joins w to a seed,
// and every step of it passes the two conditions above (each of them ends at
// or above L, started below L, and is bounded by its new row k-1).  The
// refinement then starts at or above every new value and stops at the
// greatest fixpoint, which is the new row.
constexpr int kIThreads = 512;
constexpr int kIWarps = kIThreads / 32;

struct InsState {
    RowStateT<kIWarps> S;
    uint32_t pkey[kHash];  // the previous row's region (slots as S.key had them)
    int pval[kHash];       // and its new values in that row
    unsigned long long scanned;  // list entries read, all rows
    unsigned pused;        // entries of the previous row's region
};

// New row-(k-1) value of a member w of C_k: the previous row's region holds
// every value that rose there; row 0 is the updated row-0 array.
__device__ __forceinline__ int prev_val(const RepairParams& p, const InsState& I, uint32_t w, int k) {
    if (k == 1) return p.row0_new[w];
    if (I.pused) {
        unsigned i = hslot0(w) & (kHash - 1);
        for (int probe = 0; probe < kHash; ++probe) {
            const uint32_t key = I.pkey[i];
            if (key == w) return I.pval[i];
            if (key == kEmptyKey) break;
            i = (i + 1) & (kHash - 1);
        }
    }
    return sky_at(p, w, k - 1);
}

// Row-k value of w before the batch; -1 when w was outside C_k.
__device__ __forceinline__ int old_val(const RepairParams& p, uint32_t w, int k) {
    return p.kmax_old[w] >= k ? sky_at(p, w, k) : -1;
}

// Adds w to the region with bound u (once) and queues it for expansion.
__device__ __forceinline__ void ins_add(InsState& I, uint32_t w, int u) {
    auto& S = I.S;
    const int slot = h_slot(S, w, true);
    if (slot < 0) return;
    if (atomicCAS(&S.st[slot], 0u, 1u) == 0u) {
        atomicExch(&S.cur[slot], u);
        __threadfence_block();
        enqueue(S, (unsigned)slot);
    }
}

// Converged warp, after x fell from cap to nv: queues the region members of
// a list whose value lies in (nv, cap]; returns how many neighbours in C_k
// hold at least nv (read after the write, as in r_release).
template <class St>
__device__ __forceinline__ int r_release_region(const RepairParams& p, St& S, const uint32_t* a, int n, int k, int nv,
                                                int cap) {
    int support = 0;
    for (int e = (int)(threadIdx.x & 31u); e < n && !vld(&S.abort); e += 32) {
        const uint32_t w = a[e];
        if (p.kmax_new[w] < k) continue;
        const int sl = h_slot(S, w, false);
        int x = sl >= 0 ? vld(&S.cur[sl]) : kUnset;
        if (x == kUnset) x = sky_at(p, w, k);
        support += x >= nv;
        if (sl >= 0 && x > nv && x <= cap) {
            const unsigned o = atomicCAS(&S.st[sl], 0u, 1u);
            if (o == 0u) enqueue(S, (unsigned)sl);
            else if (o == 1u) atomicCAS(&S.st[sl], 1u, 2u);
        }
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) support += __shfl_xor_sync(0xFFFFFFFFu, support, s);
    return support;
}

// Converged warp: largest L <= cap with #{out-nbrs in C_k at >= L} >= L and
// #{in-nbrs in C_k at >= L} >= k, by 64-value windows from the top.
template <class St>
__device__ int r_eval(const RepairParams& p, St& S, uint32_t x, int k, int cap, int* ho, int* hi_) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t* ao = p.out_nbr + p.out_off[x];
    const uint32_t* ai = p.in_nbr + p.in_off[x];
    const int no = p.out_len[x], ni = p.in_len[x];
    int carry_o = 0, carry_i = 0, hi = cap;
    bool first = true;
    for (;;) {
        const int lo = max(0, hi - (kRWin - 1));
        ho[lane] = 0;
        ho[lane + 32] = 0;
        hi_[lane] = 0;
        hi_[lane + 32] = 0;
        __syncwarp();
        r_hist(p, S, ao, no, k, lo, hi, first, ho);
        r_hist(p, S, ai, ni, k, lo, hi, first, hi_);
        __syncwarp();
        int found = -1;
        if (lane == 0) {
            for (int L = hi; L >= lo; --L) {
                carry_o += ho[L - lo];
                carry_i += hi_[L - lo];
                if (carry_o >= L && carry_i >= k) {
                    found = L;
                    break;
                }
            }
        }
        found = __shfl_sync(0xFFFFFFFFu, found, 0);
        carry_o = __shfl_sync(0xFFFFFFFFu, carry_o, 0);
        carry_i = __shfl_sync(0xFFFFFFFFu, carry_i, 0);
        __syncwarp();
        if (found >= 0) return found;
        if (lo == 0) return 0;  // a member keeps at least 0
        hi = lo - 1;
        first = false;
    }
}

__global__ void __launch_bounds__(kIThreads, 1) k_row_repair_ins(RepairParams p) {
    if (p.run && !*p.run) return;
    const int32_t R = p.R_dev ? *p.R_dev : p.R;
    const uint32_t n_leave = p.n_leave_dev ? *p.n_leave_dev : p.n_leave;
    const unsigned long long deadline = p.deadline_dev ? *p.deadline_dev : p.deadline_ns;
    extern __shared__ __align__(16) unsigned char s_raw[];
    InsState& I = *reinterpret_cast<InsState*>(s_raw);
    auto& S = I.S;
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    int* ho = S.hist[wib][0];
    int* hi_ = S.hist[wib][1];
    const unsigned long long t_start = gtimer();
    for (int i = threadIdx.x; i < kHash; i += kIThreads) {
        S.key[i] = kEmptyKey;
        S.cur[i] = kUnset;
        S.st[i] = 0;
        S.ring[i] = kEmptySlot;
    }
    if (threadIdx.x == 0) {
        S.used = 0;
        S.abort = 0;
        S.job_busy = 0;  // no shared scans in this kernel
        S.job_id = 0;
        S.job_ctr = 0;
        S.job_nchunks = 0;
        I.scanned = 0;
        I.pused = 0;
    }
    for (int k = 1; k <= R; ++k) {
        __syncthreads();
        if (threadIdx.x == 0 && ld_vol(&p.ctl->error)) S.abort = 1;
        __syncthreads();
        if (S.abort) break;
        if (S.used) {  // the last row left entries: clear the table
            __syncthreads();
            for (int i = threadIdx.x; i < kHash; i += kIThreads) {
                S.key[i] = kEmptyKey;
                S.cur[i] = kUnset;
                S.st[i] = 0;
                S.ring[i] = kEmptySlot;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            S.qhead = S.qtail = S.used = 0;
            S.out = 1;  // held by the seeding phase
            S.k = k;
        }
        __syncthreads();
        // ---- seeds: inserted edges inside C_k, vertices that joined C_k
        for (uint32_t i = threadIdx.x; i < p.n_del && !vld(&S.abort); i += kIThreads) {
            const uint32_t a = p.del_u[i], b = p.del_v[i];
            if (p.kmax_new[a] < k || p.kmax_new[b] < k) continue;
            int u = prev_val(p, I, a, k);
            if (u > old_val(p, a, k)) ins_add(I, a, u);
            u = prev_val(p, I, b, k);
            if (u > old_val(p, b, k)) ins_add(I, b, u);
        }
        for (uint32_t i = threadIdx.x; i < n_leave && !vld(&S.abort); i += kIThreads) {
            const uint32_t x = p.leave[i];
            if (p.kmax_old[x] < k && p.kmax_new[x] >= k) ins_add(I, x, prev_val(p, I, x, k));
        }
        __syncthreads();
        if (S.used == 0) {
            // nothing can rise in this row; the next row reads the old row
            if (threadIdx.x == 0) I.pused = 0;
            continue;
        }
        // ---- region: expand from every queued vertex
        if (threadIdx.x == 0) atomicSub(&S.out, 1);
        __syncthreads();
        unsigned slot;
        while (r_take(p, S, &slot)) {
            const uint32_t x = vldu(&S.key[slot]);
            const int t = vld(&S.cur[slot]);
            for (int side = 0; side < 2; ++side) {
                const uint32_t* a = side ? p.in_nbr + p.in_off[x] : p.out_nbr + p.out_off[x];
                const int n = side ? p.in_len[x] : p.out_len[x];
                for (int e = (int)lane; e < n && !vld(&S.abort); e += 32) {
                    const uint32_t w = a[e];
                    if (p.kmax_new[w] < k || h_slot(S, w, false) >= 0) continue;
                    const int o = old_val(p, w, k);
                    if (o >= t) continue;
                    const int u = prev_val(p, I, w, k);
                    if (u > o) ins_add(I, w, u);
                }
            }
            __syncwarp();
            if (lane == 0) {
                atomicAdd(&I.scanned, (unsigned long long)(p.out_len[x] + p.in_len[x]));
                if (deadline && gtimer() - t_start > deadline) atomicExch(&S.abort, 1);
                __threadfence_block();
                atomicSub(&S.out, 1);
            }
            __syncwarp();
        }
        __syncthreads();
        if (S.abort) break;
        // ---- refinement from the bounds: queue the whole region
        if (threadIdx.x == 0) {
            S.qhead = S.qtail = 0;
            S.out = 1;
        }
        for (int i = threadIdx.x; i < kHash; i += kIThreads) {
            S.ring[i] = kEmptySlot;
            S.st[i] = 0;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kHash; i += kIThreads)
            if (S.key[i] != kEmptyKey) {
                S.st[i] = 1u;
                enqueue(S, (unsigned)i);
            }
        for (int sweep = 0;; ++sweep) {
            __syncthreads();
            if (threadIdx.x == 0) atomicSub(&S.out, 1);
            __syncthreads();
            while (r_take(p, S, &slot)) {
                const uint32_t x = vldu(&S.key[slot]);
                const int cap = vld(&S.cur[slot]);
                const int nv = cap >= 1 ? r_eval(p, S, x, k, cap, ho, hi_) : cap;
                if (nv < cap) {
                    if (lane == 0) atomicExch(&S.cur[slot], nv);
                    __syncwarp();
                    __threadfence_block();
                    const int so = r_release_region(p, S, p.out_nbr + p.out_off[x], p.out_len[x], k, nv, cap);
                    const int si = r_release_region(p, S, p.in_nbr + p.in_off[x], p.in_len[x], k, nv, cap);
                    if (lane == 0 && nv >= 1 && (so < nv || si < k)) atomicCAS(&S.st[slot], 1u, 2u);
                }
                __syncwarp();
                if (lane == 0) {
                    atomicAdd(&I.scanned, 2ull * (unsigned long long)(p.out_len[x] + p.in_len[x]));
                    if (deadline && gtimer() - t_start > deadline) atomicExch(&S.abort, 1);
                    if (atomicCAS(&S.st[slot], 1u, 0u) == 2u) {
                        atomicExch(&S.st[slot], 1u);
                        enqueue(S, slot);
                    }
                    __threadfence_block();
                    atomicSub(&S.out, 1);
                }
                __syncwarp();
            }
            __syncthreads();
            if (S.abort) break;
            if (sweep == 32) {  // bounded: a row that keeps failing is recomputed
                if (threadIdx.x == 0) S.abort = 1;
                __syncthreads();
                break;
            }
            // ---- the row is quiet: every region vertex must hold its value
            // against the final values; queue any that does not, drain again
            if (threadIdx.x == 0) {
                S.qhead = S.qtail = 0;
                S.out = 1;  // held by the sweep
                S.k = 0;    // vertices found unstable
            }
            for (int i = threadIdx.x; i < kHash; i += kIThreads) S.ring[i] = kEmptySlot;
            __syncthreads();
            for (int i = wib; i < kHash; i += kIWarps) {
                const uint32_t x = S.key[i];
                if (x == kEmptyKey) continue;
                const int val = S.cur[i];
                if (val < 1) continue;
                int so = 0, si = 0;
                const uint32_t* ao = p.out_nbr + p.out_off[x];
                const uint32_t* ai = p.in_nbr + p.in_off[x];
                so = r_count_at_least(p, S, ao, p.out_len[x], k, val);
                si = r_count_at_least(p, S, ai, p.in_len[x], k, val);
#pragma unroll
                for (int s = 16; s; s >>= 1) {
                    so += __shfl_xor_sync(0xFFFFFFFFu, so, s);
                    si += __shfl_xor_sync(0xFFFFFFFFu, si, s);
                }
                if (lane == 0 && (so < val || si < k)) {
                    atomicAdd(&S.k, 1);
                    const unsigned o = atomicCAS(&S.st[i], 0u, 1u);
                    if (o == 0u) enqueue(S, (unsigned)i);
                }
            }
            __syncthreads();
            const bool again = S.k != 0;
            __syncthreads();
            if (threadIdx.x == 0) S.k = k;
            if (!again) {
                __syncthreads();
                break;
            }
        }
        __syncthreads();
        if (S.abort) break;
        // ---- values that differ from the old skyline's reading go to the
        // log (a vertex that joined C_k is read as its last old corner,
        // which is how the merged skyline reads rows above its old kmax);
        // the region becomes the next row's "previous row"
        for (int i = threadIdx.x; i < kHash; i += kIThreads) {
            const uint32_t v = S.key[i];
            const int c = S.cur[i];
            I.pkey[i] = v;
            I.pval[i] = c;
            if (v == kEmptyKey || c == sky_at(p, v, k)) continue;
            const unsigned long long li = atomicAdd(&p.ctl->log_count, 1u);
            if (li < p.log_cap) {
                p.log_v[li] = v;
                p.log_k[li] = k;
                p.log_l[li] = c;
            } else {
                set_dev_error(p.ctl, DC_DEV_ERR_CAPACITY, 45);
            }
        }
        if (threadIdx.x == 0) I.pused = S.used;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (S.abort && !ld_vol(&p.ctl->error)) set_dev_error(p.ctl, DC_DEV_ERR_CAPACITY, 44);
        p.ctl->edges_scanned = I.scanned;
    }
}

// Work of a repair: sum over the endpoints x of the deleted edges of
// deg(x) * kmax(x), the list entries a row-by-row repair scans at least once.
__global__ void k_repair_work(uint32_t n, const uint32_t* u, const uint32_t* v, const int32_t* kmax,
                              const int32_t* in_len, const int32_t* out_len, unsigned long long* acc) {
    unsigned long long w = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t a = u[i], b = v[i];
        w += (unsigned long long)(in_len[a] + out_len[a]) * (unsigned long long)max(kmax[a], 0);
        w += (unsigned long long)(in_len[b] + out_len[b]) * (unsigned long long)max(kmax[b], 0);
    }
#pragma unroll
    for (int s = 16; s; s >>= 1) w += __shfl_xor_sync(0xFFFFFFFFu, w, s);
    if ((threadIdx.x & 31u) == 0) atomicAdd(acc, w);
}

// Vertices whose kmax fell (rise = false) or rose (rise = true), compacted.
__global__ void k_collect_leave(uint32_t V, const int32_t* kold, const int32_t* knew, uint32_t* out, unsigned* n,
                                bool rise) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        if (rise ? knew[v] > kold[v] : knew[v] < kold[v]) out[atomicAdd(n, 1u)] = (uint32_t)v;
}

// Per-vertex change lists from the log: count, fill, sort by k.  Captured
// batches read n on the device (n_dev) and act only while *run != 0.
__global__ void k_chg_count(unsigned long long n, const uint32_t* lv, unsigned long long* cnt,
                            const unsigned long long* n_dev, const int* run) {
    if (run && !*run) return;
    if (n_dev) n = *n_dev;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[lv[i]], 1ull);
}
__global__ void k_chg_fill(unsigned long long n, const uint32_t* lv, const int32_t* lk, const int32_t* ll,
                           const unsigned long long* off, uint32_t* fill, int32_t* ck, int32_t* cl,
                           const unsigned long long* n_dev, const int* run) {
    if (run && !*run) return;
    if (n_dev) n = *n_dev;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v = lv[i];
        uint64_t o = off[v] + atomicAdd(&fill[v], 1u);
        ck[o] = lk[i];
        cl[o] = ll[i];
    }
}
__global__ void k_chg_sort(uint32_t V, const unsigned long long* off, int32_t* ck, int32_t* cl, uint32_t* off32,
                           const int* run) {
    if (run && !*run) return;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t a = off[v], b = off[v + 1];
        for (uint64_t i = a + 1; i < b; ++i) {
            int kk = ck[i], ll = cl[i];
            uint64_t j = i;
            while (j > a && ck[j - 1] > kk) {
                ck[j] = ck[j - 1];
                cl[j] = cl[j - 1];
                --j;
            }
            ck[j] = kk;
            cl[j] = ll;
        }
        off32[v] = (uint32_t)a;
        if (v == V - 1) off32[V] = (uint32_t)b;
    }
}

// New skyline of v: corner (0, new row 0), then at every row k <= new kmax
// where the old skyline has a corner, the change list has an entry, or a
// change run ends, the new value (change or old value) when it differs from
// the previous corner's.  FILL = false counts, true writes.  Change lists:
// none when coff is null or *chg_run is 0.  A vertex with no change, the
// same row 0 and every old corner at or below its kmax keeps its corners as
// they are (counted from the offsets, copied without the merge walk).
template <bool FILL>
__global__ void k_rep_merge(uint32_t V, const int32_t* kmax, const int32_t* row0, const uint32_t* ooff,
                            const int32_t* ok, const int32_t* ol, const uint32_t* coff, const int32_t* ck,
                            const int32_t* cl, unsigned long long* cnt_off, int32_t* nk, int32_t* nl,
                            uint32_t* noff, const int* run, const int* chg_run) {
    if (run && !*run) return;
    const bool chg = coff && (!chg_run || *chg_run);
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const int km = kmax[v];
        const uint32_t i0 = ooff[v], ie = ooff[v + 1];
        uint32_t i = i0;
        uint32_t j = chg ? coff[v] : 0, je = chg ? coff[v + 1] : 0;
        uint64_t o = FILL ? cnt_off[v] : 0;
        uint64_t c = 0;
        int last = row0[v];
        int oldv = (i < ie) ? ol[i] : 0;  // old row-0 corner
        if (j == je && i < ie && oldv == last && ok[ie - 1] <= km) {
            // unchanged: the old corners as they are
            c = ie - i0;
            if (FILL) {
                for (uint32_t t = 0; t < c; ++t) {
                    nk[o + t] = ok[i0 + t];
                    nl[o + t] = ol[i0 + t];
                }
                noff[v] = (uint32_t)o;
                if (v == V - 1) noff[V] = (uint32_t)(o + c);
            } else {
                cnt_off[v] = c;
            }
            continue;
        }
        if (FILL) {
            nk[o] = 0;
            nl[o] = last;
        }
        ++c;
        ++i;
        // row after a change run; a changed row 0 is one (an unchanged row 1
        // keeps its old value, which may now differ from row 0)
        int after = oldv != last ? 1 : 0x7FFFFFFF;
        for (;;) {
            int kc = 0x7FFFFFFF;
            if (i < ie) kc = min(kc, ok[i]);
            if (j < je) kc = min(kc, ck[j]);
            kc = min(kc, after);
            if (kc > km) break;
            while (i < ie && ok[i] <= kc) oldv = ol[i++];
            int val = oldv;
            after = 0x7FFFFFFF;
            if (j < je && ck[j] == kc) {
                val = cl[j++];
                after = kc + 1;
            }
            if (val != last) {
                if (FILL) {
                    nk[o + c] = kc;
                    nl[o + c] = val;
                }
                ++c;
                last = val;
            }
        }
        if (FILL) {
            noff[v] = (uint32_t)o;
            if (v == V - 1) noff[V] = (uint32_t)(o + c);
        } else {
            cnt_off[v] = c;
        }
    }
}

// ---------------------------------------------------------------------------
// decisions of a captured batch (BatchStatus)
// ---------------------------------------------------------------------------
// After the kmax / row-0 update: R, and whether rows 1..R are repaired in
// place, only row 0's corners merged, or recomputed by the host -- the
// decisions rows_repair / rows_repair_ins and the maintenance driver take.
__global__ void k_gb_decide(BatchStatus* st, const int* dbuf, unsigned long long full_work, int rmode,
                            uint32_t n_edges, float full_rows_ms, int K_old) {
    if (!st->run_apply) return;
    const int Knew = dbuf[1];
    const int R = min(dbuf[0], Knew);
    st->R = R;
    st->Knew = Knew;
    st->lmax = dbuf[2];
    if (R < 0) return;  // nothing changed
    if (R == 0) {       // rows above 0 keep their values
        st->run_merge = 1;
        st->nlog = 0;
        return;
    }
    const bool fits = 2ull * n_edges + st->n_leave <= kHashLimit;
    const bool worth = rmode >= 2 || (full_work > 0 && 160ull * st->work < full_work);
    if (fits && worth) {
        st->run_repair = 1;
        // the time limit repair_deadline_ns sets on the host path
        const float ms = 2.f + full_rows_ms * fminf(1.f, (float)R / (float)max(K_old, 1)) + 0.1f * full_rows_ms;
        st->deadline_ns = rmode == 2 ? 0ull : (unsigned long long)(ms * 1e6f);
    } else {
        st->fallback = 1;
    }
}

// After the repair: merge its log, or hand the rows to the host.
__global__ void k_gb_after_repair(const EngineCtl* c, BatchStatus* st) {
    if (!st->run_repair) return;
    const unsigned e = c->error;
    st->run_repair = 0;
    if (e & DC_DEV_ERR_TIMEOUT) {
        st->err |= e;
        st->err_where = c->err_where;
        return;
    }
    if (e) {  // table full or past the time limit: recompute
        st->fallback = 1;
        return;
    }
    st->run_merge = 1;
    st->nlog = c->log_count;
    st->run_chg = st->nlog > 0;
    st->scanned = c->edges_scanned;
}

// The merged skyline's size against its buffer.
__global__ void k_gb_total(BatchStatus* st, const unsigned long long* cnt, uint32_t V) {
    if (!st->run_merge) return;
    st->total = cnt[V];
    if (st->total > st->cap) {
        st->run_merge = 0;
        st->merge_overflow = 1;
    }
}

}  // namespace


static int rgrid(dc_graph* h, uint64_t n) {
    uint64_t b = (n + kRThreads - 1) / kRThreads;
    uint64_t cap = (uint64_t)h->geom.sms * 16;
    return (int)std::max<uint64_t>(1, std::min(b, cap));
}

// Largest deletion batch whose seeds fit a row's table (callers split mixed
// batches only below it).
uint32_t row_repair_max_deletions() { return kHashLimit / 4; }

// Whether repairing the rows after deleting these edges (device arrays) is
// expected to beat recomputing them: the entries the repair scans (sum over
// the edges' endpoints of degree x kmax) against the graph's sum of degree x
// kmax at its last full decomposition.  The row-to-row derivation scans about
// a twentieth of the latter and the repair makes ~8 passes over its entries
// (histogram, release, re-check), hence the factor 160.  Deterministic: the
// same graph and batch always take the same path.
bool row_repair_worthwhile(dc_graph* h, const uint32_t* d_u, const uint32_t* d_v, uint32_t n) {
    if (n == 0 || 2ull * n > kHashLimit || h->full_work == 0 || !h->d.kmax_v) return false;
    unsigned long long* acc = (unsigned long long*)h->scratch->tmp64;
    if (cudaMemsetAsync(acc, 0, sizeof(unsigned long long), h->stream) != cudaSuccess) return false;
    ++g_launches;
    k_repair_work<<<rgrid(h, n), kRThreads, 0, h->stream>>>(n, d_u, d_v, h->d.kmax_v, h->g.in_len, h->g.out_len,
                                                              acc);
    unsigned long long w = 0;
    if (cudaMemcpyAsync(&w, acc, sizeof(w), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return 160ull * w < h->full_work;
}

#define RP_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess) {                                                            \
            cudaGetLastError();                                                             \
            return set_error(DC_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
        }                                                                                   \
    } while (0)

// The change log of a repair: the scratch corner log (sized by the last
// decomposition), at least 2^20 entries.
int ensure_change_log(dc_graph* h, uint64_t* cap_out) {
    Scratch* s = h->scratch;
    uint64_t cap = s->log_cap;
    if (cap < (1u << 20)) {
        cudaFreeAsync(s->log_v, h->stream);
        cudaFreeAsync(s->log_k, h->stream);
        cudaFreeAsync(s->log_l, h->stream);
        s->log_v = nullptr;
        s->log_k = nullptr;
        s->log_l = nullptr;
        s->log_cap = 0;
        cap = 1u << 20;
        if (cudaMallocAsync((void**)&s->log_v, 4 * cap, h->stream) != cudaSuccess ||
            cudaMallocAsync((void**)&s->log_k, 4 * cap, h->stream) != cudaSuccess ||
            cudaMallocAsync((void**)&s->log_l, 4 * cap, h->stream) != cudaSuccess) {
            cudaGetLastError();
            return set_error(DC_ERR_NOMEM, "row repair: change log allocation failed");
        }
        s->log_cap = cap;
    }
    *cap_out = cap;
    return DC_OK;
}

// Merges the change log (v, k, new value) of a repair with the current
// skyline into the new skyline (kmax and row 0 already updated) and makes it
// current; *applied tells whether it did.
int apply_change_log(dc_graph* h, uint64_t nlog, bool* applied) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    // per-vertex change lists
    // the change lists go to spare skyline slot 0 and the merged skyline to
    // slot 1 (no allocation once the slots have grown to the graph's size)
    unsigned long long* cnt = (unsigned long long*)s->tmp64;
    uint32_t *coff = nullptr, *fill = s->cursor, *noff = nullptr;
    int32_t *ck = nullptr, *cl = nullptr, *nk = nullptr, *nl = nullptr;
    uint64_t ccap = 0, ncap = 0;
    // (no change lists when only row 0 changed)
    int rc = nlog ? sky_take_spare(h, 0, nlog, &coff, &ck, &cl, &ccap) : DC_OK;
    unsigned long long total = 0;
    if (rc == DC_OK && nlog) {
        cudaMemsetAsync(cnt, 0, 8ull * (V + 1), h->stream);
        cudaMemsetAsync(fill, 0, 4ull * V, h->stream);
        g_launches += 3;
        k_chg_count<<<rgrid(h, nlog), kRThreads, 0, h->stream>>>(nlog, s->log_v, cnt, nullptr, nullptr);
        rc = scan_tmp64(h, V);
        if (rc == DC_OK) {
            k_chg_fill<<<rgrid(h, nlog), kRThreads, 0, h->stream>>>(nlog, s->log_v, s->log_k, s->log_l, cnt, fill, ck,
                                                                    cl, nullptr, nullptr);
            k_chg_sort<<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, cnt, ck, cl, coff, nullptr);
        }
    }
    if (rc == DC_OK) {
        // new skyline: count, scan, fill
        ++g_launches;
        k_rep_merge<false><<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, d.kmax_v, d.row0, d.sky_off, d.sky_k, d.sky_l,
                                                                     coff, ck, cl, cnt, nullptr, nullptr, nullptr,
                                                                     nullptr, nullptr);
        rc = scan_tmp64(h, V);
    }
    if (rc == DC_OK) {
        if (cudaMemcpyAsync(&total, cnt + V, sizeof(total), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess) {
            cudaGetLastError();
            rc = set_error(DC_ERR_CUDA, "row repair: corner count download failed");
        }
    }
    if (rc == DC_OK) rc = sky_take_spare(h, 1, total, &noff, &nk, &nl, &ncap);
    if (rc == DC_OK) {
        ++g_launches;
        k_rep_merge<true><<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, d.kmax_v, d.row0, d.sky_off, d.sky_k, d.sky_l,
                                                                    coff, ck, cl, cnt, nk, nl, noff, nullptr, nullptr);
        if (cudaGetLastError() != cudaSuccess) rc = set_error(DC_ERR_CUDA, "row repair: merge launch failed");
    }
    if (coff || ck) sky_put_spare(h, 0, coff, ck, cl, ccap);
    if (rc != DC_OK) {
        if (noff || nk) sky_put_spare(h, 1, noff, nk, nl, ncap);
        return rc;
    }
    // the old skyline becomes the spare of slot 1
    sky_put_spare(h, 1, d.sky_off, d.sky_k, d.sky_l, d.corner_cap);
    d.sky_off = noff;
    d.sky_k = nk;
    d.sky_l = nl;
    d.n_corners = total;
    d.corner_cap = ncap;
    *applied = true;
    return DC_OK;
}

// Rows 1..R after a deletion-only batch (graph, kmax and row 0 already
// updated; kmax before the batch in scratch kmax_old).  Replaces the skyline
// and sets *applied; leaves everything untouched with *applied = false when a
// row touched more vertices than a block's table holds or the change log ran
// out (the caller then recomputes the rows).
int rows_repair(dc_graph* h, int32_t R, const uint32_t* d_du, const uint32_t* d_dv, uint32_t n_del,
                unsigned long long deadline_ns, bool* applied) {
    *applied = false;
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    if (R < 1 || V == 0) return DC_OK;
    if (2ull * n_del > kHashLimit) return DC_OK;  // the seeds alone overflow a row's table
    unsigned* n_leave_d = (unsigned*)s->cursor;
    RP_CUDA(cudaMemsetAsync(n_leave_d, 0, sizeof(unsigned), h->stream));
    ++g_launches;
    k_collect_leave<<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, s->kmax_old, d.kmax_v, s->rem0, n_leave_d, false);
    unsigned n_leave = 0;
    RP_CUDA(cudaMemcpyAsync(&n_leave, n_leave_d, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    RP_CUDA(cudaStreamSynchronize(h->stream));
    if (2ull * n_del + n_leave > kHashLimit) return DC_OK;
    uint64_t cap = 0;
    if (int rc = ensure_change_log(h, &cap)) return rc;
    RP_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
    if (h->wait_ns)
        RP_CUDA(cudaMemcpyAsync(&h->ctl->wait_ns, &h->wait_ns, sizeof(h->wait_ns), cudaMemcpyHostToDevice, h->stream));
    RP_CUDA(cudaStreamSynchronize(h->stream));
    RepairParams p;
    p.V = V;
    p.out_off = g.out_off; p.out_len = g.out_len; p.out_nbr = g.out_nbr;
    p.in_off = g.in_off; p.in_len = g.in_len; p.in_nbr = g.in_nbr;
    p.kmax_new = d.kmax_v;
    p.kmax_old = s->kmax_old;
    p.sky_off = d.sky_off; p.sky_k = d.sky_k; p.sky_l = d.sky_l;
    p.del_u = d_du; p.del_v = d_dv; p.n_del = n_del;
    p.leave = s->rem0; p.n_leave = n_leave;
    p.row0_new = nullptr;
    p.deadline_ns = deadline_ns;
    p.R = R;
    p.R_dev = nullptr;
    p.n_leave_dev = nullptr;
    p.deadline_dev = nullptr;
    p.run = nullptr;
    p.log_v = s->log_v; p.log_k = s->log_k; p.log_l = s->log_l; p.log_cap = cap;
    p.ctl = h->ctl;
    static_assert(sizeof(RowState) <= 200 * 1024, "row table exceeds shared memory");
    RP_CUDA(cudaFuncSetAttribute(k_row_repair, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RowState)));
    const int blocks = std::max(1, std::min<int>(R, h->geom.sms));
    ++g_launches;
    k_row_repair<<<blocks, kRThreads, sizeof(RowState), h->stream>>>(p);
    RP_CUDA(cudaGetLastError());
    EngineCtl hc;
    RP_CUDA(cudaMemcpyAsync(&hc, h->ctl, sizeof(EngineCtl), cudaMemcpyDeviceToHost, h->stream));
    RP_CUDA(cudaStreamSynchronize(h->stream));
    if (hc.error & DC_DEV_ERR_TIMEOUT)
        return set_error(DC_ERR_TIMEOUT, "row repair: bounded device wait expired (site %u)", hc.err_where);
    if (hc.error) return DC_OK;  // capacity: the caller recomputes the rows
    return apply_change_log(h, hc.log_count, applied);
}

// Largest insertion batch whose seeds fit a row's table.
uint32_t row_repair_max_insertions() { return kHashLimit / 4; }

// Rows 1..R after an insertion-only batch (graph, kmax and row 0 already
// updated; kmax before the batch in scratch kmax_old).  Replaces the skyline
// and sets *applied; leaves everything untouched with *applied = false when a
// row's region outgrew the table, the repair ran past deadline_ns (the
// recomputation is then expected to be cheaper), or the change log ran out.
// *scanned: list entries the repair read.
int rows_repair_ins(dc_graph* h, int32_t R, const uint32_t* d_iu, const uint32_t* d_iv, uint32_t n_ins,
                    unsigned long long deadline_ns, bool* applied, unsigned long long* scanned) {
    *applied = false;
    *scanned = 0;
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    if (R < 1 || V == 0) return DC_OK;
    if (2ull * n_ins > kHashLimit) return DC_OK;
    unsigned* n_join_d = (unsigned*)s->cursor;
    RP_CUDA(cudaMemsetAsync(n_join_d, 0, sizeof(unsigned), h->stream));
    ++g_launches;
    k_collect_leave<<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, s->kmax_old, d.kmax_v, s->rem0, n_join_d, true);
    unsigned n_join = 0;
    RP_CUDA(cudaMemcpyAsync(&n_join, n_join_d, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    RP_CUDA(cudaStreamSynchronize(h->stream));
    if (2ull * n_ins + n_join > kHashLimit) return DC_OK;
    uint64_t cap = 0;
    if (int rc = ensure_change_log(h, &cap)) return rc;
    RP_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(EngineCtl), h->stream));
    if (h->wait_ns)
        RP_CUDA(cudaMemcpyAsync(&h->ctl->wait_ns, &h->wait_ns, sizeof(h->wait_ns), cudaMemcpyHostToDevice, h->stream));
    RepairParams p;
    memset(&p, 0, sizeof(p));
    p.V = V;
    p.out_off = g.out_off; p.out_len = g.out_len; p.out_nbr = g.out_nbr;
    p.in_off = g.in_off; p.in_len = g.in_len; p.in_nbr = g.in_nbr;
    p.kmax_new = d.kmax_v;
    p.kmax_old = s->kmax_old;
    p.sky_off = d.sky_off; p.sky_k = d.sky_k; p.sky_l = d.sky_l;
    p.del_u = d_iu; p.del_v = d_iv; p.n_del = n_ins;
    p.leave = s->rem0; p.n_leave = n_join;
    p.row0_new = d.row0;
    p.deadline_ns = deadline_ns;
    p.R = R;
    p.log_v = s->log_v; p.log_k = s->log_k; p.log_l = s->log_l; p.log_cap = cap;
    p.ctl = h->ctl;
    static_assert(sizeof(InsState) <= 227 * 1024, "insertion repair state exceeds shared memory");
    RP_CUDA(cudaFuncSetAttribute(k_row_repair_ins, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(InsState)));
    ++g_launches;
    k_row_repair_ins<<<1, kIThreads, sizeof(InsState), h->stream>>>(p);
    RP_CUDA(cudaGetLastError());
    EngineCtl hc;
    RP_CUDA(cudaMemcpyAsync(&hc, h->ctl, sizeof(EngineCtl), cudaMemcpyDeviceToHost, h->stream));
    RP_CUDA(cudaStreamSynchronize(h->stream));
    *scanned = hc.edges_scanned;
    if (hc.error & DC_DEV_ERR_TIMEOUT)
        return set_error(DC_ERR_TIMEOUT, "row repair: bounded device wait expired (site %u)", hc.err_where);
    if (hc.error) return DC_OK;  // capacity or budget: the caller recomputes the rows
    return apply_change_log(h, hc.log_count, applied);
}

// ---------------------------------------------------------------------------
// captured batches: the same row maintenance with its decisions on the device
// ---------------------------------------------------------------------------
int repair_prepare(dc_graph* h) {
    (void)h;
    RP_CUDA(cudaFuncSetAttribute(k_row_repair, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RowState)));
    RP_CUDA(cudaFuncSetAttribute(k_row_repair_ins, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(InsState)));
    return DC_OK;
}

int decide_enqueue(dc_graph* h, BatchStatus* st, const int* dbuf, int rmode, uint32_t n_edges, bool insertions) {
    g_launches += 2;
    k_collect_leave<<<rgrid(h, h->g.V), kRThreads, 0, h->stream>>>(h->g.V, h->scratch->kmax_old, h->d.kmax_v,
                                                                   h->scratch->rem0, &st->n_leave, insertions);
    k_gb_decide<<<1, 1, 0, h->stream>>>(st, dbuf, h->full_work, rmode, n_edges, h->full_rows_ms, h->d.kmax);
    RP_CUDA(cudaGetLastError());
    return DC_OK;
}

// The repair of rows 1..st->R (deletions or insertions; the vertices whose
// kmax fell / rose already in scratch rem0, their count in st->n_leave),
// acting only when st->run_repair, within st->deadline_ns; its change log
// holds at most log_cap entries.
int repair_enqueue(dc_graph* h, bool insertions, const uint32_t* d_u, const uint32_t* d_v, uint32_t n,
                   uint64_t log_cap, BatchStatus* st) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    RepairParams p;
    memset(&p, 0, sizeof(p));
    p.V = g.V;
    p.out_off = g.out_off; p.out_len = g.out_len; p.out_nbr = g.out_nbr;
    p.in_off = g.in_off; p.in_len = g.in_len; p.in_nbr = g.in_nbr;
    p.kmax_new = d.kmax_v;
    p.kmax_old = s->kmax_old;
    p.sky_off = d.sky_off; p.sky_k = d.sky_k; p.sky_l = d.sky_l;
    p.del_u = d_u; p.del_v = d_v; p.n_del = n;
    p.leave = s->rem0;
    p.row0_new = insertions ? d.row0 : nullptr;
    p.deadline_ns = 0;
    p.deadline_dev = &st->deadline_ns;
    p.R = 0;
    p.R_dev = &st->R;
    p.n_leave_dev = &st->n_leave;
    p.run = &st->run_repair;
    p.log_v = s->log_v; p.log_k = s->log_k; p.log_l = s->log_l; p.log_cap = log_cap;
    p.ctl = h->ctl;
    if (int rc = ctl_init_enqueue(h, h->ctl, h->stream)) return rc;
    ++g_launches;
    if (insertions) k_row_repair_ins<<<1, kIThreads, sizeof(InsState), h->stream>>>(p);
    else k_row_repair<<<std::max(1, h->geom.sms), kRThreads, sizeof(RowState), h->stream>>>(p);
    RP_CUDA(cudaGetLastError());
    ++g_launches;
    k_gb_after_repair<<<1, 1, 0, h->stream>>>(h->ctl, st);
    RP_CUDA(cudaGetLastError());
    return DC_OK;
}

// apply_change_log's passes with the log length read from st->nlog, acting
// only when st->run_merge: change lists into (coff, ck, cl), the merged
// skyline into (noff, nk, nl) of st->cap corners (a larger result clears
// run_merge and sets merge_overflow).
int merge_enqueue(dc_graph* h, BatchStatus* st, uint32_t* coff, int32_t* ck, int32_t* cl, uint32_t* noff,
                  int32_t* nk, int32_t* nl) {
    DevGraph& g = h->g;
    Decomp& d = h->d;
    Scratch* s = h->scratch;
    const uint32_t V = g.V;
    unsigned long long* cnt = (unsigned long long*)s->tmp64;
    uint32_t* fill = s->cursor;
    const int grid_log = rgrid(h, s->log_cap);
    // change lists only when the repair logged changes (st->run_chg)
    RP_CUDA(cudaMemsetAsync(cnt, 0, 8ull * (V + 1), h->stream));
    RP_CUDA(cudaMemsetAsync(fill, 0, 4ull * V, h->stream));
    g_launches += 2;
    k_chg_count<<<grid_log, kRThreads, 0, h->stream>>>(0, s->log_v, cnt, &st->nlog, &st->run_chg);
    if (int rc = scan_tmp64(h, V)) return rc;
    g_launches += 3;
    k_chg_fill<<<grid_log, kRThreads, 0, h->stream>>>(0, s->log_v, s->log_k, s->log_l, cnt, fill, ck, cl, &st->nlog,
                                                      &st->run_chg);
    k_chg_sort<<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, cnt, ck, cl, coff, &st->run_chg);
    k_rep_merge<false><<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, d.kmax_v, d.row0, d.sky_off, d.sky_k, d.sky_l,
                                                                 coff, ck, cl, cnt, nullptr, nullptr, nullptr,
                                                                 &st->run_merge, &st->run_chg);
    if (int rc = scan_tmp64(h, V)) return rc;
    g_launches += 2;
    k_gb_total<<<1, 1, 0, h->stream>>>(st, cnt, V);
    k_rep_merge<true><<<rgrid(h, V), kRThreads, 0, h->stream>>>(V, d.kmax_v, d.row0, d.sky_off, d.sky_k, d.sky_l,
                                                                coff, ck, cl, cnt, nk, nl, noff, &st->run_merge,
                                                                &st->run_chg);
    RP_CUDA(cudaGetLastError());
    return DC_OK;
}

}  // namespace dc
