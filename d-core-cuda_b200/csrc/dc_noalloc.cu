// kmax (in-degree core numbers) without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: code that owns all
// device memory through its own arena or pool and forbids other allocations,
// serving loops where cudaMalloc's implicit device-wide synchronisation
// would stall unrelated streams, and setups that must not grow the device
// footprint after start-up.  dc_kmax_noalloc serves them: the caller passes
// the graph (plain CSR and CSC arrays already on the device) and the output
// array, and every intermediate buffer of the peel lives in one fixed-size
// device array that is part of this library's module.
//
// Limits: at most kNaMaxV vertices and kNaMaxE edges per call.  The scratch
// array (about 11 MB) is reserved on every GPU that loads the library and
// stays reserved until the process exits.  All calls share it, so calls that
// overlap on the GPU (different streams or threads) race and must be
// serialised by the caller.  The first call on a device looks up the array's
// device address with cudaGetSymbolAddress; that call should come before any
// stream capture on that device.
#include <cstdint>
#include <cstring>
#include <mutex>

#include "dc_device.cuh"
#include "dc_internal.h"

namespace dc {
namespace {

constexpr uint32_t kNaMaxV = 1u << 18;     // 262,144 vertices
constexpr uint64_t kNaMaxE = 1ull << 22;   // 4,194,304 edges
constexpr unsigned kNaChunk = 64;          // adjacency entries per queue item
constexpr uint64_t kNaRingSlots = 1ull << 20;
constexpr int kNaThreads = 256;

// byte layout of the scratch array
constexpr size_t kNaCtlBytes = 2048;
constexpr size_t kNaKeyOff = kNaCtlBytes;
constexpr size_t kNaRem0Off = kNaKeyOff + 4ull * kNaMaxV;
constexpr size_t kNaRem1Off = kNaRem0Off + 4ull * kNaMaxV;
constexpr size_t kNaRingOff = kNaRem1Off + 4ull * kNaMaxV;
constexpr size_t kNaBytes = kNaRingOff + 8ull * kNaRingSlots;
static_assert(sizeof(EngineCtl) <= kNaCtlBytes, "control block does not fit its slot");
static_assert(kNaRingSlots >= kNaMaxV + kNaMaxE / kNaChunk + 4 * 148 * 64, "ring too small for the limits");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

struct NaParams {
    uint32_t V;
    const uint32_t* in_off;   // V+1 (peeling degree = in-degree)
    const uint32_t* out_off;  // V+1
    const uint32_t* out_nbr;  // out-neighbours lose one in-degree unit per removal
    int32_t* kmax;            // output [V]
    EngineCtl* ctl;
    int32_t* key;
    uint32_t* rem0;
    uint32_t* rem1;
    TicketQueue q;
};

struct NaHook {
    unsigned nworkers;
    __device__ void operator()(EngineCtl* c) const {
        c->rc_cur[0] = c->rc_next[0].v;
        c->rc_next[0].v = 0;
        c->t_tail = c->t_head;
        c->outstanding = (int)nworkers;
        c->phase_done = 0;
        __threadfence();
    }
};

__device__ __forceinline__ unsigned na_items(const NaParams& p, uint32_t x) {
    unsigned len = p.out_off[x + 1] - p.out_off[x];
    return (len + kNaChunk - 1) / kNaChunk;
}

// Level-by-level peel of the in-degree (the kmax pass of the engine's fused
// peel, restricted to one instance and plain CSR/CSC input).
__global__ void __launch_bounds__(kNaThreads) k_kmax_noalloc(NaParams p) {
    const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const unsigned gwarp = blockIdx.x * (kNaThreads / 32) + wib;
    const unsigned nwarps = gridDim.x * (kNaThreads / 32);
    EngineCtl* c = p.ctl;
    NaHook hook{gridDim.x};
    __shared__ unsigned s_prod;
    if (threadIdx.x == 0) s_prod = 0;
    for (uint64_t base = (uint64_t)gwarp * 32; base < p.V; base += (uint64_t)nwarps * 32) {
        uint64_t vi = base + lane;
        bool ok = vi < p.V;
        uint32_t v = (uint32_t)vi;
        if (ok) {
            p.kmax[v] = -1;
            p.key[v] = (int)(p.in_off[v + 1] - p.in_off[v]);
        }
        unsigned pos = warp_append(&c->rc_next[0].v, ok);
        if (ok) p.rem0[pos] = v;
    }
    if (!grid_sync_hook(c, hook)) return;
    unsigned ticket = kNoTicket;
    for (int L = 0;; ++L) {
        const unsigned n_rem = ld_vol(&c->rc_cur[0]);
        if (n_rem == 0) break;
        const uint32_t* rc = (L & 1) ? p.rem1 : p.rem0;
        uint32_t* rn = (L & 1) ? p.rem0 : p.rem1;
        bool pushed = false;
        for (unsigned base = gwarp * 32; base < n_rem; base += nwarps * 32) {
            unsigned idx = base + lane;
            bool okk = idx < n_rem;
            uint32_t v = okk ? rc[idx] : 0;
            bool keep = false, push = false;
            if (okk && ld_vol(&p.kmax[v]) == -1) {
                if (ld_vol(&p.key[v]) <= L)
                    push = atomicCAS(&p.kmax[v], -1, L) == -1;
                else
                    keep = true;
            }
            unsigned pos = warp_append(&c->rc_next[0].v, keep);
            if (keep) rn[pos] = v;
            unsigned cnt = push ? na_items(p, v) : 0u;
            tq_push_warp_multi(c, p.q, cnt, (unsigned long long)v, 1ull << 32);
            pushed |= __any_sync(0xFFFFFFFFu, push);
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            if (atomicAdd(&s_prod, 1u) == (kNaThreads / 32) - 1) {
                s_prod = 0;
                tq_finish(c, 1);
            }
        }
        __syncwarp();
        unsigned long long item;
        while (tq_take_warp(c, p.q, &ticket, &item)) {
            const uint32_t x = (uint32_t)item;
            const unsigned ch = (unsigned)(item >> 32);
            const uint32_t o = p.out_off[x];
            const unsigned len = p.out_off[x + 1] - o;
            const unsigned e0 = ch * kNaChunk, e1 = min(len, e0 + kNaChunk);
            for (unsigned b = e0; b < e1; b += 32) {
                unsigned e = b + lane;
                bool push = false;
                uint32_t w = 0;
                if (e < e1) {
                    w = p.out_nbr[o + e];
                    int old = atomicSub(&p.key[w], 1);
                    push = old == L + 1 && ld_vol(&p.kmax[w]) == -1 && atomicCAS(&p.kmax[w], -1, L) == -1;
                }
                unsigned cnt = push ? na_items(p, w) : 0u;
                tq_push_warp_multi(c, p.q, cnt, (unsigned long long)w, 1ull << 32);
                pushed |= __any_sync(0xFFFFFFFFu, push);
            }
            __syncwarp();
            if (lane == 0) tq_finish(c, 1);
        }
        if (lane == 0 && pushed) atomicMax(&c->maxv[0], L);
        if (!grid_sync_hook(c, hook)) return;
    }
}

// Device address of the scratch array, looked up once per device.
std::mutex g_na_mutex;
constexpr int kNaMaxDevices = 64;
unsigned char* g_na_base[kNaMaxDevices] = {};

int na_scratch_base(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kNaMaxDevices) return set_error(DC_ERR_INVALID, "dc_kmax_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_na_mutex);
    if (!g_na_base[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            cudaGetLastError();
            return set_error(DC_ERR_CUDA, "dc_kmax_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        }
        g_na_base[dev] = (unsigned char*)ptr;
    }
    *out = g_na_base[dev];
    return DC_OK;
}

}  // namespace
}  // namespace dc

using namespace dc;

extern "C" int dc_kmax_noalloc(uint32_t V, uint64_t E, const uint32_t* d_in_off, const uint32_t* d_out_off,
                               const uint32_t* d_out_nbr, int32_t* d_kmax, int32_t* kmax_max, void* stream) {
    if (V > kNaMaxV || E > kNaMaxE)
        return set_error(DC_ERR_CAPACITY,
                         "dc_kmax_noalloc: graph of %u vertices / %llu edges exceeds the fixed scratch limit of "
                         "%u vertices / %llu edges",
                         V, (unsigned long long)E, kNaMaxV, (unsigned long long)kNaMaxE);
    if (V > 0 && (!d_in_off || !d_out_off || !d_kmax || (E > 0 && !d_out_nbr)))
        return set_error(DC_ERR_INVALID, "dc_kmax_noalloc: null array");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_NO_DEVICE, "dc_kmax_noalloc: no CUDA device (%s)", cudaGetErrorString(e));
    }
    unsigned char* base = nullptr;
    if (int rc = na_scratch_base(dev, &base)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (kmax_max) *kmax_max = 0;
    if (V == 0) return DC_OK;

    NaParams p;
    p.V = V;
    p.in_off = d_in_off;
    p.out_off = d_out_off;
    p.out_nbr = d_out_nbr;
    p.kmax = d_kmax;
    p.ctl = (EngineCtl*)base;
    p.key = (int32_t*)(base + kNaKeyOff);
    p.rem0 = (uint32_t*)(base + kNaRem0Off);
    p.rem1 = (uint32_t*)(base + kNaRem1Off);
    p.q.slots = (unsigned long long*)(base + kNaRingOff);
    p.q.mask = (unsigned)(kNaRingSlots - 1);

    // the queue ring is sized for kNaMaxE adjacency entries: the edge count
    // the arrays really hold (out_off[V], in_off[V]) must be the E given
    uint32_t ends[2] = {0, 0};
    e = cudaMemcpyAsync(&ends[0], d_out_off + V, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ends[1], d_in_off + V, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "dc_kmax_noalloc: reading the edge counts failed: %s", cudaGetErrorString(e));
    }
    if (ends[0] > kNaMaxE || ends[1] > kNaMaxE)
        return set_error(DC_ERR_CAPACITY,
                         "dc_kmax_noalloc: the arrays hold %u out- / %u in-edges, beyond the fixed scratch limit of "
                         "%llu edges",
                         ends[0], ends[1], (unsigned long long)kNaMaxE);
    if ((uint64_t)ends[0] != E || (uint64_t)ends[1] != E)
        return set_error(DC_ERR_INVALID, "dc_kmax_noalloc: E = %llu but out_off[V] = %u and in_off[V] = %u",
                         (unsigned long long)E, ends[0], ends[1]);

    // the shared scratch keeps the previous call's contents: reset the
    // control block and empty the queue ring
    e = cudaMemsetAsync(base, 0, kNaCtlBytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(base + kNaRingOff, 0xFF, 8ull * kNaRingSlots, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "dc_kmax_noalloc: scratch reset failed: %s", cudaGetErrorString(e));
    }
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_kmax_noalloc, kNaThreads, 0);
    if (e != cudaSuccess || per_sm < 1 || sms < 1) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "dc_kmax_noalloc: occupancy query failed");
    }
    void* args[] = {&p};
    e = cudaLaunchCooperativeKernel((const void*)k_kmax_noalloc, dim3(sms), dim3(kNaThreads), args, 0, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "dc_kmax_noalloc: launch failed: %s", cudaGetErrorString(e));
    }
    EngineCtl hc;
    e = cudaMemcpyAsync(&hc, base, sizeof(EngineCtl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(DC_ERR_CUDA, "dc_kmax_noalloc: %s", cudaGetErrorString(e));
    }
    if (hc.error)
        return set_error(hc.error & DC_DEV_ERR_TIMEOUT ? DC_ERR_TIMEOUT : DC_ERR_CUDA,
                         "dc_kmax_noalloc: device status 0x%x (site %u)", hc.error, hc.err_where);
    if (kmax_max) *kmax_max = hc.maxv[0];
    return DC_OK;
}
