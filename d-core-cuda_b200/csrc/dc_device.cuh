// Device-side building blocks shared by the persistent engine kernels:
//   - EngineCtl: counters, error word and grid-barrier state in device memory
//   - grid_sync: software grid barrier with a bounded wait (cooperative launch)
//   - work queue: ring of vertex ids with claim / done counters and a
//     termination test, so cascades run without per-round barriers
//   - warp-aggregated append
// Every spin in here is bounded by the control block's wait limit
// (EngineCtl::wait_ns, kWaitNs when 0) of %globaltimer time; on expiry the
// waiter sets DC_DEV_ERR_TIMEOUT in EngineCtl::error and returns, so a fault
// in the protocol ends the kernel with a status instead of a hang.
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
constexpr unsigned long long kWaitNs = 4000000000ull;  // default limit of one wait: 4 s
constexpr int kMaxRowSegments = 8;  // concurrent launches a full run of rows may split into
constexpr int kMinSplitRows = 32;   // runs of fewer rows are never split

// A counter on a 128-byte line of its own.
struct alignas(128) PadU {
    unsigned v;
};
struct alignas(128) PadI {
    int v;
};

// The counters every warp hits (ticket head and tail, the outstanding count,
// the barrier) and the flags idle warps poll (phase_done, error) each sit in
// a 128-byte line of their own: on one line they all land in one L2 slice,
// which then serialises the grid.
struct EngineCtl {
    // grid barrier
    alignas(128) unsigned bar_count;
    unsigned bar_gen;
    // polled by idle warps
    alignas(128) unsigned error;
    unsigned err_where;
    unsigned phase_done;    // set by whoever brings outstanding to 0
    // work queue (monotone within one phase)
    alignas(128) unsigned q_head;
    unsigned q_tail;
    unsigned q_done;
    unsigned pad0;
    // per-step counters, rotated over three slots
    unsigned producers[3];
    unsigned rcount[3];
    // results / statistics
    int maxval;
    int steps;
    alignas(128) unsigned log_count;
    unsigned pad1;
    unsigned long long evals;
    unsigned long long drops;
    unsigned long long pushes;
    unsigned long long edges_scanned;
    // ticket queue (see TicketQueue)
    alignas(128) unsigned t_head;  // next ticket
    alignas(128) unsigned t_tail;  // next slot to reserve
    alignas(128) int outstanding;  // unfinished producers + pushed, unfinished items
    alignas(128) unsigned rc_cur[2];  // remaining-list sizes per peel instance
    PadU rc_next[2];        // next level's remaining-list sizes (appended by every warp)
    int maxv[2];            // largest value per peel instance
    int step;               // level / transition index
    unsigned nworkers;      // producers per phase (warps in the grid)
    int level;              // current level / row of the persistent loop
    int next_min;           // smallest level / row a skipped step may jump to
    PadI minkey[2];         // per peel instance: least peeling degree kept by the scan
    // optional per-step timing trace: 8 words per step
    //   [0] %globaltimer at step start, [1] when its work ran out,
    //   [2] queue items of the step, [3] %globaltimer at the closing barrier,
    //   [4] latest block wake-up after the opening barrier,
    //   [5] latest block seeding done, [6] earliest block wake-up
    unsigned long long* trace;
    unsigned trace_cap;
    unsigned trace_tail0;
    // limit of one bounded wait in ns (0: kWaitNs)
    unsigned long long wait_ns;
    // failure-detection tests: block test_skip_block - 1 leaves at its first
    // grid barrier without arriving, so every other block's barrier wait runs
    // out (0: off)
    int test_skip_block;
};

// Decisions and results of one maintenance batch run as a captured CUDA
// graph: every branch the host-driven batch takes between its kernels is
// taken on the device, by small kernels writing these fields, and the
// kernels after a branch act only while their run flag is set.
struct BatchStatus {
    int run_apply;      // the batch is valid: no missing deletion, insertions fit their free slots
    int run_repair;     // rows 1..R are repaired in place
    int run_merge;      // a new skyline is merged (the repair's changes, or new row-0 corners only)
    int run_chg;        // the merge reads change lists (the repair logged changes)
    int fallback;       // rows 1..R must be recomputed (repair not expected to pay, or it gave up)
    int merge_overflow; // the merged skyline outgrew its buffer: the host merges instead
    int notfound;       // a deleted edge is not in the graph (nothing applied)
    int need_rebuild;   // an inserted edge does not fit its list (nothing applied)
    int R, Knew, lmax;  // row bound, kmax and lmax after the batch
    unsigned err, err_where;  // device error bits of the persistent kernels
    unsigned n_leave;   // vertices whose kmax fell (deletions) or rose (insertions)
    unsigned pad;
    unsigned long long nlog, total, cap, work, region, scanned;
    unsigned long long deadline_ns;  // time limit of the repair (0: none)
};

__device__ __forceinline__ unsigned long long wait_limit(const EngineCtl* c) {
    const unsigned long long w = *reinterpret_cast<const volatile unsigned long long*>(&c->wait_ns);
    return w ? w : kWaitNs;
}

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
// waiters then leave on the error word or after the wait limit.
// Returns true when the grid may continue.
__device__ __forceinline__ bool grid_sync(EngineCtl* c) {
    __shared__ unsigned s_ok;
    if (c->test_skip_block && (int)blockIdx.x == c->test_skip_block - 1) return false;
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
            const unsigned long long t0 = gtimer(), lim = wait_limit(c);
            while (ld_vol(&c->bar_gen) == gen) {
                if (ld_vol(&c->error)) break;
                if (gtimer() - t0 > lim) {
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

// Grid barrier whose last arriving block runs hook(c) before releasing the
// others, so per-phase counters can be reset with no other block running.
template <typename Hook>
__device__ __forceinline__ bool grid_sync_hook(EngineCtl* c, Hook hook) {
    __shared__ unsigned s_ok2;
    if (c->test_skip_block && (int)blockIdx.x == c->test_skip_block - 1) return false;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nb = gridDim.x;
        unsigned gen = ld_vol(&c->bar_gen);
        __threadfence();
        unsigned arrived = atomicAdd(&c->bar_count, 1u);
        if (arrived == nb - 1) {
            hook(c);
            atomicExch(&c->bar_count, 0u);
            __threadfence();
            atomicAdd(&c->bar_gen, 1u);
        } else {
            const unsigned long long t0 = gtimer(), lim = wait_limit(c);
            while (ld_vol(&c->bar_gen) == gen) {
                if (ld_vol(&c->error)) break;
                if (gtimer() - t0 > lim) {
                    set_dev_error(c, DC_DEV_ERR_TIMEOUT, 4);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok2 = (ld_vol(&c->error) == 0u);
        if (c->trace) {
            int st = ld_vol(&c->step);
            if (st >= 0 && (unsigned)st < c->trace_cap) {
                unsigned long long now = gtimer();
                atomicMax(&c->trace[8 * st + 4], now);
                atomicMin(&c->trace[8 * st + 6], now);
            }
        }
    }
    __syncthreads();
    return s_ok2 != 0u;
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
    const unsigned long long t0 = gtimer(), lim = wait_limit(c);
    for (;;) {
        v = atomicExch(s, kEmptySlot);
        if (v != kEmptySlot) return v;
        if (ld_vol(&c->error)) return kEmptySlot;
        if (gtimer() - t0 > lim) {
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

// ---------------------------------------------------------------------------
// Ticket queue.  Items are 64-bit words in a ring of slots (kEmptyItem =
// free).  A consumer warp takes a ticket with one atomicAdd on t_head and
// polls only its own slot, so idle warps do not contend on shared counters.
// Termination uses one counter: `outstanding` starts at the number of
// producer warps; each producer subtracts 1 when its seeding share is done,
// each push adds the number of pushed items before they become visible, and
// each finished item subtracts 1 after its own pushes.  Whoever brings it to
// 0 sets phase_done; a consumer whose slot is still empty then leaves.  At
// the barrier that ends the phase the abandoned tickets are skipped by
// setting t_tail = t_head (grid_sync_hook).
// ---------------------------------------------------------------------------
constexpr unsigned long long kEmptyItem = ~0ull;

struct TicketQueue {
    unsigned long long* slots;
    unsigned mask;
};

__device__ __forceinline__ void tq_finish(EngineCtl* c, int n) {
    __threadfence();
    if (atomicSub(&c->outstanding, n) == n) {
        atomicExch(&c->phase_done, 1u);
        if (c->trace && (unsigned)c->step < c->trace_cap) c->trace[8 * c->step + 1] = gtimer();
    }
}

// Called by the last block of a phase-ending barrier: closes the step's
// trace record and opens the next one.
__device__ __forceinline__ void trace_step_end(EngineCtl* c) {
    unsigned long long now = gtimer();
    if (c->trace && c->step >= 0 && (unsigned)c->step < c->trace_cap) {
        c->trace[8 * c->step + 2] = c->t_tail - c->trace_tail0;
        c->trace[8 * c->step + 3] = now;
    }
    c->step++;
    if (c->trace && (unsigned)c->step < c->trace_cap) {
        c->trace[8 * c->step] = now;
        c->trace[8 * c->step + 6] = ~0ull;
    }
    c->trace_tail0 = c->t_tail;
}

// Converged warp: lanes with pred push `cnt` consecutive items item0,
// item0 + inc, ... (cnt may be 0).
__device__ __forceinline__ void tq_push_warp_multi(EngineCtl* c, TicketQueue q, unsigned cnt,
                                                   unsigned long long item0, unsigned long long inc) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    unsigned total = __shfl_sync(0xFFFFFFFFu, x, 31);
    if (total == 0) return;
    unsigned base = 0;
    if (lane == 0) {
        atomicAdd(&c->outstanding, (int)total);
        base = atomicAdd(&c->t_tail, total);
    }
    base = __shfl_sync(0xFFFFFFFFu, base, 0) + (x - cnt);
    if (cnt) __threadfence();
    for (unsigned i = 0; i < cnt; ++i) {
        volatile unsigned long long* s = &q.slots[(base + i) & q.mask];
        *s = item0 + inc * i;
    }
}

__device__ __forceinline__ void tq_push_warp(EngineCtl* c, TicketQueue q, bool pred, unsigned long long item) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned m = __ballot_sync(0xFFFFFFFFu, pred);
    if (!m) return;
    unsigned base = 0;
    if (lane == 0) {
        atomicAdd(&c->outstanding, (int)__popc(m));
        base = atomicAdd(&c->t_tail, (unsigned)__popc(m));
    }
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (pred) {
        __threadfence();
        volatile unsigned long long* s = &q.slots[(base + __popc(m & ((1u << lane) - 1u))) & q.mask];
        *s = item;
    }
}

// Converged warp: each lane pushes its first cnt (<= 4) entries of items[].
__device__ __forceinline__ void tq_push_warp4(EngineCtl* c, TicketQueue q, unsigned cnt, const uint32_t* items) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    unsigned total = __shfl_sync(0xFFFFFFFFu, x, 31);
    if (total == 0) return;
    unsigned base = 0;
    if (lane == 0) {
        atomicAdd(&c->outstanding, (int)total);
        base = atomicAdd(&c->t_tail, total);
    }
    base = __shfl_sync(0xFFFFFFFFu, base, 0) + (x - cnt);
    if (cnt) __threadfence();
#pragma unroll
    for (unsigned i = 0; i < 4; ++i) {
        if (i < cnt) {
            volatile unsigned long long* s = &q.slots[(base + i) & q.mask];
            *s = (unsigned long long)items[i];
        }
    }
}

// Converged warp: each lane pushes items[r] for every bit r set in mask
// (r < 4), in bit order.
__device__ __forceinline__ void tq_push_warp_mask4(EngineCtl* c, TicketQueue q, unsigned mask,
                                                   const uint32_t items[4]) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned cnt = __popc(mask);
    unsigned x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    unsigned total = __shfl_sync(0xFFFFFFFFu, x, 31);
    if (total == 0) return;
    unsigned base = 0;
    if (lane == 0) {
        atomicAdd(&c->outstanding, (int)total);
        base = atomicAdd(&c->t_tail, total);
    }
    base = __shfl_sync(0xFFFFFFFFu, base, 0) + (x - cnt);
    if (cnt) __threadfence();
#pragma unroll
    for (unsigned r = 0; r < 4; ++r) {
        if (mask & (1u << r)) {
            volatile unsigned long long* s = &q.slots[(base + __popc(mask & ((1u << r) - 1u))) & q.mask];
            *s = (unsigned long long)items[r];
        }
    }
}

// Converged warp: returns true with *item set, or false when the phase is
// over (or an error / timeout occurred).  *ticket holds the warp's current
// ticket between calls (kNoTicket initially).
constexpr unsigned kNoTicket = 0xFFFFFFFFu;
__device__ __forceinline__ bool tq_take_warp(EngineCtl* c, TicketQueue q, unsigned* ticket,
                                             unsigned long long* item) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long it = kEmptyItem;
    int state = 0;  // 1 = got item, 2 = phase over
    if (lane == 0) {
        if (*ticket == kNoTicket) *ticket = atomicAdd(&c->t_head, 1u);
        volatile unsigned long long* s = &q.slots[*ticket & q.mask];
        unsigned long long t0 = 0;
        unsigned spins = 0, seen_tail = 0;
        int seen_out = 0;
        for (;;) {
            it = *s;
            if (it != kEmptyItem) {
                *s = kEmptyItem;
                *ticket = kNoTicket;
                state = 1;
                break;
            }
            // the shared flags are polled every 4th spin once the wait is long
            if ((spins < 16 || (spins & 3) == 0) && (ld_vol(&c->phase_done) || ld_vol(&c->error))) {
                // abandon the ticket: the phase-ending barrier skips it
                *ticket = kNoTicket;
                state = 2;
                break;
            }
            if (++spins == 64) {
                t0 = gtimer();
                seen_tail = ld_vol(&c->t_tail);
                seen_out = ld_vol(&c->outstanding);
            }
            // the limit bounds a wait without progress: while the phase's
            // other warps still push or finish items the clock restarts
            if (spins > 64 && (spins & 63) == 0) {
                const unsigned tl = ld_vol(&c->t_tail);
                const int ou = ld_vol(&c->outstanding);
                if (tl != seen_tail || ou != seen_out) {
                    seen_tail = tl;
                    seen_out = ou;
                    t0 = gtimer();
                } else if (gtimer() - t0 > wait_limit(c)) {
                    set_dev_error(c, DC_DEV_ERR_TIMEOUT, 5);
                    *ticket = kNoTicket;
                    state = 2;
                    break;
                }
            }
            if (spins > 16) __nanosleep(spins > 256 ? 256 : 32);
        }
    }
    state = __shfl_sync(0xFFFFFFFFu, state, 0);
    it = __shfl_sync(0xFFFFFFFFu, it, 0);
    __threadfence();
    *item = it;
    return state == 1;
}

// tq_take_warp with lazily counted finishes: *pending (lane 0's count of
// items this warp finished but has not yet subtracted from `outstanding`) is
// subtracted in one atomic when the warp's slot is not filled at once, i.e.
// before the warp can wait; a warp that keeps finding items never touches
// `outstanding` for them until then.  On a false return *pending is 0.
__device__ __forceinline__ bool tq_take_warp_lazy(EngineCtl* c, TicketQueue q, unsigned* ticket,
                                                  unsigned long long* item, unsigned* pending) {
    const unsigned lane = threadIdx.x & 31u;
    if (lane == 0) {
        if (*ticket == kNoTicket) *ticket = atomicAdd(&c->t_head, 1u);
        volatile unsigned long long* s = &q.slots[*ticket & q.mask];
        if (*s == kEmptyItem && *pending) {
            tq_finish(c, (int)*pending);
            *pending = 0;
        }
    }
    return tq_take_warp(c, q, ticket, item);
}

// Idle-wait helper for the drain loops: returns false once the phase has made
// no progress for the wait limit (error recorded).
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
        if (gtimer() - t0 > wait_limit(c)) {
            set_dev_error(c, DC_DEV_ERR_TIMEOUT, 3);
            return false;
        }
        __nanosleep(64);
        return true;
    }
};

}  // namespace dc
