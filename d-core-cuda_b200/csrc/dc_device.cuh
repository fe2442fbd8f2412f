// Device-side building blocks shared by the persistent engine kernels:
//   - EngineCtl: counters, error word and grid-barrier state in device memory
//   - grid_sync: software grid barrier with a bounded wait (cooperative launch)
//   - work queue: ring of vertex ids with claim / done counters and a
//     termination test, so cascades run without per-round barriers
//   - warp-aggregated append
// Every spin in here is bounded by kWaitNs of %globaltimer time; on expiry
// the waiter sets DC_DEV_ERR_TIMEOUT in EngineCtl::error and returns, so a
// fault in the protocol ends the kernel with a status instead of a hang.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dc {

constexpr unsigned DC_DEV_ERR_TIMEOUT = 1u;   // a bounded wait ran out
constexpr unsigned DC_DEV_ERR_QUEUE = 2u;     // queue capacity exceeded
constexpr unsigned DC_DEV_ERR_BADID = 4u;     // vertex id out of range
constexpr unsigned DC_DEV_ERR_CAPACITY = 8u;  // a log or list buffer overflowed
constexpr unsigned DC_DEV_ERR_NOTFOUND = 16u; // delete of an absent edge

constexpr uint32_t kEmptySlot = 0xFFFFFFFFu;
constexpr unsigned long long kWaitNs = 4000000000ull;  // 4 s per wait

struct EngineCtl {
    // grid barrier
    unsigned bar_count;
    unsigned bar_gen;
    unsigned error;
    unsigned err_where;
    // work queue (monotone within one phase)
    unsigned q_head;
    unsigned q_tail;
    unsigned q_done;
    unsigned pad0;
    // per-step counters, rotated over three slots
    unsigned producers[3];
    unsigned rcount[3];
    // results / statistics
    int maxval;
    int steps;
    unsigned log_count;
    unsigned pad1;
    unsigned long long evals;
    unsigned long long drops;
    unsigned long long pushes;
    unsigned long long edges_scanned;
};

__device__ __forceinline__ unsigned ld_vol(const unsigned* p) {
    return *reinterpret_cast<const volatile unsigned*>(p);
}
__device__ __forceinline__ int ld_vol(const int* p) {
    return *reinterpret_cast<const volatile int*>(p);
}
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void set_dev_error(EngineCtl* c, unsigned code, unsigned where) {
    atomicOr(&c->error, code);
    atomicExch(&c->err_where, where);
}

// Software grid barrier.  All blocks of a cooperative launch are co-resident,
// so every block reaches it unless one has already bailed out on an error;
// waiters then leave on the error word or after kWaitNs.
// Returns true when the grid may continue.
__device__ __forceinline__ bool grid_sync(EngineCtl* c) {
    __shared__ unsigned s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x;
        unsigned gen = ld_vol(&c->bar_gen);
        __threadfence();
        unsigned arrived = atomicAdd(&c->bar_count, 1u);
        if (arrived == nb - 1) {
            atomicExch(&c->bar_count, 0u);
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            unsigned long long t0 = gtimer();
            while (ld_vol(&c->bar_gen) == gen) {
                if (ld_vol(&c->error)) break;
                if (gtimer() - t0 > kWaitNs) {
                    set_dev_error(c, DC_DEV_ERR_TIMEOUT, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = (ld_vol(&c->error) == 0u);
    }
    __syncthreads();
    return s_ok != 0u;
}

// Warp-aggregated append: every lane of a converged warp calls this; lanes
// with pred get consecutive positions from *counter.
__device__ __forceinline__ unsigned warp_append(unsigned* counter, bool pred, unsigned* total = nullptr) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned mask = __ballot_sync(0xFFFFFFFFu, pred);
    if (total) *total = __popc(mask);
    if (!mask) return 0;
    unsigned leader = __ffs(mask) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Ring of vertex ids.  Producers reserve slots with q_tail and store the id;
// a consumer claims [h, h+n) by CAS on q_head, waits for each slot to be
// filled, resets it to kEmptySlot and, after its work (including its own
// pushes) is visible, adds n to q_done.  The phase is over when every
// producer has finished its seeding share and q_done == q_tail.
struct RingQueue {
    uint32_t* slots;
    unsigned mask;
};

// Converged-warp push of v for lanes with pred.
__device__ __forceinline__ void q_push_warp(EngineCtl* c, RingQueue q, bool pred, uint32_t v) {
    unsigned pos = warp_append(&c->q_tail, pred);
    if (pred) {
        atomicExch(&q.slots[pos & q.mask], v);
    }
}

// Single-thread push (divergent contexts).
__device__ __forceinline__ void q_push_one(EngineCtl* c, RingQueue q, uint32_t v) {
    unsigned pos = atomicAdd(&c->q_tail, 1u);
    atomicExch(&q.slots[pos & q.mask], v);
}

// Lane 0 of a converged warp tries to claim up to maxn items.  Returns the
// claimed count (broadcast) and the first index in *first.  0 with
// *finished = true means the phase is complete; 0 with *finished = false
// means nothing to claim right now.
__device__ __forceinline__ unsigned q_claim_warp(EngineCtl* c, unsigned maxn, unsigned total_producers,
                                                 unsigned* producers, unsigned* first, bool* finished) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned n = 0, h = 0, fin = 0;
    if (lane == 0) {
        h = ld_vol(&c->q_head);
        unsigned t = ld_vol(&c->q_tail);
        if (h < t) {
            unsigned want = min(maxn, t - h);
            if (atomicCAS(&c->q_head, h, h + want) == h) n = want;
        } else {
            unsigned p = ld_vol(producers);
            __threadfence();
            unsigned d = ld_vol(&c->q_done);
            __threadfence();
            unsigned t2 = ld_vol(&c->q_tail);
            if (p == total_producers && d == t2) fin = 1;
        }
    }
    n = __shfl_sync(0xFFFFFFFFu, n, 0);
    h = __shfl_sync(0xFFFFFFFFu, h, 0);
    fin = __shfl_sync(0xFFFFFFFFu, fin, 0);
    *first = h;
    *finished = fin != 0;
    return n;
}

// Reads a claimed slot, waiting (bounded) for its producer's store.
__device__ __forceinline__ uint32_t q_take(EngineCtl* c, RingQueue q, unsigned idx) {
    uint32_t* s = &q.slots[idx & q.mask];
    uint32_t v = atomicExch(s, kEmptySlot);
    if (v != kEmptySlot) return v;
    unsigned long long t0 = gtimer();
    for (;;) {
        v = atomicExch(s, kEmptySlot);
        if (v != kEmptySlot) return v;
        if (ld_vol(&c->error)) return kEmptySlot;
        if (gtimer() - t0 > kWaitNs) {
            set_dev_error(c, DC_DEV_ERR_TIMEOUT, 2);
            return kEmptySlot;
        }
        __nanosleep(16);
    }
}

// Marks n claimed items as done after the calling warp's writes are visible.
__device__ __forceinline__ void q_done_warp(EngineCtl* c, unsigned n) {
    __threadfence();
    __syncwarp();
    if ((threadIdx.x & 31u) == 0 && n) atomicAdd(&c->q_done, n);
}

// Idle-wait helper for the drain loops: returns false once the phase has made
// no progress for kWaitNs (error recorded).
struct IdleClock {
    unsigned long long t0;
    unsigned last_done;
    __device__ __forceinline__ void start(EngineCtl* c) {
        t0 = gtimer();
        last_done = ld_vol(&c->q_done);
    }
    __device__ __forceinline__ bool tick(EngineCtl* c) {
        unsigned d = ld_vol(&c->q_done);
        if (d != last_done) {
            last_done = d;
            t0 = gtimer();
            return true;
        }
        if (gtimer() - t0 > kWaitNs) {
            set_dev_error(c, DC_DEV_ERR_TIMEOUT, 3);
            return false;
        }
        __nanosleep(64);
        return true;
    }
};

}  // namespace dc
