// Device-side insert-batch partition: getKmaxEdgeBatches with
// KEDGE_BATCHING (main.cu:1441-1488) on the GPU.
//
// The reference gives every edge a root -- the endpoint with the larger kmax,
// the target on ties (main.cu:1449-1452) -- buckets the edges by the root's
// kmax in ascending order and splits each bucket greedily, in input order,
// into sub-batches with pairwise distinct roots, allocating a vector<bool>(V)
// per sub-batch on the host (main.cu:1469).  The greedy pass j of a bucket
// takes the j-th remaining edge of every root, so the sub-batch of edge e is
//     base[kmax(root e)] + occ(e)
// where occ(e) counts the earlier edges (input order) with the same root and
// base[k] is the number of sub-batches of the buckets below k (a bucket has as
// many as its most frequent root has edges).  On the device:
//   1. roots and root kmax per edge;
//   2. a stable LSD radix sort of the edge indices by root (4-bit digits,
//      only the bits a vertex id of this graph uses): per-tile digit counts,
//      one scan, a scatter that ranks equal digits in input order;
//   3. occ(e) = position - start of the root's run (run starts by a scan);
//   4. passes per root kmax by atomicMax, a scan, and the numbering.
// Everything is O(B) work on the graph's stream with B-sized scratch; no
// O(V) pass per sub-batch.
#include <algorithm>
#include <atomic>
#include <cstdint>

#include "dc_engine.cuh"
#include "dc_internal.h"

namespace dc {
extern std::atomic<unsigned long long> g_launches;
}

namespace dc {
namespace {

constexpr int kPT = 256;                // threads per block
constexpr int kPItems = 16;             // elements per thread and tile
constexpr int kPTile = kPT * kPItems;   // elements per block tile
constexpr int kDigitBits = 4;
constexpr int kDigits = 1 << kDigitBits;

__device__ __forceinline__ uint32_t block_excl_scan32(uint32_t x, uint32_t* total) {
    __shared__ uint32_t s_w[kPT / 32 + 1];
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= (unsigned)o) inc += y;
    }
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int i = 0; i < kPT / 32; ++i) {
            uint32_t t = s_w[i];
            s_w[i] = run;
            run += t;
        }
        s_w[kPT / 32] = run;
    }
    __syncthreads();
    const uint32_t r = inc - x + s_w[w];
    *total = s_w[kPT / 32];
    __syncthreads();
    return r;
}

// roots: key[e] = root vertex, val[e] = e, rk[e] = kmax of the root
__global__ void k_pt_roots(uint64_t B, uint32_t V, const uint32_t* from, const uint32_t* to, const int32_t* kmax,
                           uint32_t* key, uint32_t* val, int32_t* rk, unsigned* bad) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < B; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t f = from[e], t = to[e];
        if (f >= V || t >= V) {
            atomicOr(bad, 1u);
            key[e] = 0;
            val[e] = (uint32_t)e;
            rk[e] = 0;
            continue;
        }
        const uint32_t r = kmax[f] > kmax[t] ? f : t;
        key[e] = r;
        val[e] = (uint32_t)e;
        rk[e] = kmax[r];
    }
}

// digit counts of one tile per block: cnt[d * nblk + blk]
__global__ void k_pt_digit_count(uint64_t n, const uint32_t* key, int shift, uint32_t* cnt) {
    __shared__ uint32_t s_c[kDigits];
    if (threadIdx.x < kDigits) s_c[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t t0 = (uint64_t)blockIdx.x * kPTile;
    for (int r = 0; r < kPItems; ++r) {
        const uint64_t i = t0 + (uint64_t)r * kPT + threadIdx.x;
        if (i < n) atomicAdd(&s_c[(key[i] >> shift) & (kDigits - 1)], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kDigits) cnt[(uint64_t)threadIdx.x * gridDim.x + blockIdx.x] = s_c[threadIdx.x];
}

// exclusive scan of a[0..n) in place by one block; a[n] = total
__global__ void k_pt_scan_one_block(uint32_t* a, uint64_t n) {
    uint32_t carry = 0;
    for (uint64_t b = 0; b < n; b += kPT) {
        const uint64_t i = b + threadIdx.x;
        const uint32_t x = i < n ? a[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan32(x, &tot);
        if (i < n) a[i] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) a[n] = carry;
}

// stable scatter of one digit pass: the elements of a tile are visited in
// index order, 256 at a time; equal digits are ranked inside each warp
// (match) and across the block's warps (shared counts), on top of the
// tile's base for the digit
__global__ void k_pt_digit_scatter(uint64_t n, const uint32_t* key_in, const uint32_t* val_in, uint32_t* key_out,
                                   uint32_t* val_out, int shift, const uint32_t* off) {
    __shared__ uint32_t s_base[kDigits];
    __shared__ uint32_t s_wc[kPT / 32][kDigits];
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    if (threadIdx.x < kDigits) s_base[threadIdx.x] = off[(uint64_t)threadIdx.x * gridDim.x + blockIdx.x];
    const uint64_t t0 = (uint64_t)blockIdx.x * kPTile;
    for (int r = 0; r < kPItems; ++r) {
        for (int j = threadIdx.x; j < (kPT / 32) * kDigits; j += kPT) (&s_wc[0][0])[j] = 0;
        __syncthreads();
        const uint64_t i = t0 + (uint64_t)r * kPT + threadIdx.x;
        const bool ok = i < n;
        const uint32_t k = ok ? key_in[i] : 0u;
        const uint32_t d = (k >> shift) & (kDigits - 1);
        const unsigned peers = __match_any_sync(0xFFFFFFFFu, ok ? d : (uint32_t)(kDigits + lane));
        const unsigned rank = __popc(peers & ((1u << lane) - 1u));
        if (ok && lane == (unsigned)(__ffs(peers) - 1)) s_wc[w][d] = __popc(peers);
        __syncthreads();
        if (ok) {
            uint32_t pre = 0;
            for (unsigned x = 0; x < w; ++x) pre += s_wc[x][d];
            const uint32_t pos = s_base[d] + pre + rank;
            key_out[pos] = k;
            val_out[pos] = val_in[i];
        }
        __syncthreads();
        if (threadIdx.x < kDigits) {
            uint32_t t = 0;
            for (int x = 0; x < kPT / 32; ++x) t += s_wc[x][threadIdx.x];
            s_base[threadIdx.x] += t;
        }
        __syncthreads();
    }
}

// run starts of the sorted roots: f[i] = 1 where a new root begins; per-tile
// sums into part[blk]
__global__ void k_pt_run_flags(uint64_t n, const uint32_t* key, uint32_t* f, uint32_t* part) {
    const uint64_t t0 = (uint64_t)blockIdx.x * kPTile + (uint64_t)threadIdx.x * kPItems;
    uint32_t s = 0;
    for (int j = 0; j < kPItems; ++j) {
        const uint64_t i = t0 + j;
        if (i < n) {
            const uint32_t x = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
            f[i] = x;
            s += x;
        }
    }
    uint32_t tot;
    block_excl_scan32(s, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// run index of every sorted position (exclusive scan of the flags plus the
// flag, minus one) and the start of every run
__global__ void k_pt_runs(uint64_t n, const uint32_t* f, const uint32_t* part, uint32_t* run, uint32_t* start) {
    const uint64_t t0 = (uint64_t)blockIdx.x * kPTile + (uint64_t)threadIdx.x * kPItems;
    uint32_t s = 0;
    for (int j = 0; j < kPItems; ++j)
        if (t0 + j < n) s += f[t0 + j];
    uint32_t tot;
    uint32_t ex = block_excl_scan32(s, &tot) + part[blockIdx.x];
    for (int j = 0; j < kPItems; ++j) {
        const uint64_t i = t0 + j;
        if (i < n) {
            ex += f[i];
            run[i] = ex - 1;
            if (f[i]) start[ex - 1] = (uint32_t)i;
        }
    }
}

// occurrence of the edge held at each sorted position, and the passes each
// root kmax needs
__global__ void k_pt_occ(uint64_t n, const uint32_t* val, const uint32_t* run, const uint32_t* start,
                         const int32_t* rk, uint32_t* occ, uint32_t* passes) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t e = val[i];
        const uint32_t o = (uint32_t)i - start[run[i]];
        occ[e] = o;
        atomicMax(&passes[rk[e]], o + 1);
    }
}

__global__ void k_pt_number(uint64_t B, const int32_t* rk, const uint32_t* occ, const uint32_t* base,
                            int64_t* batch_of) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < B; e += (uint64_t)gridDim.x * blockDim.x)
        batch_of[e] = (int64_t)base[rk[e]] + (int64_t)occ[e];
}

template <typename T>
int pt_alloc(cudaStream_t st, T** p, uint64_t n) {
    cudaError_t e = cudaMallocAsync((void**)p, std::max<uint64_t>(n, 1) * sizeof(T), st);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "edge-batch partition: device allocation failed: %s", cudaGetErrorString(e));
    }
    return DC_OK;
}

}  // namespace

int kmax_edge_batches_device(dc_graph* h, uint64_t B, const uint32_t* d_from, const uint32_t* d_to,
                             int64_t* d_batch_of, int64_t* n_batches) {
    *n_batches = 0;
    if (B == 0) return DC_OK;
    if (B >= (1ull << 31)) return set_error(DC_ERR_INVALID, "edge-batch partition: at most 2^31 - 1 edges per call");
    const uint32_t V = h->g.V;
    const int32_t K = h->d.kmax;
    cudaStream_t st = h->stream;
    const uint64_t nblk = (B + kPTile - 1) / kPTile;
    const int grid = (int)std::min<uint64_t>((B + kPT - 1) / kPT, (uint64_t)h->geom.sms * 8);
    uint32_t *key0 = nullptr, *val0 = nullptr, *key1 = nullptr, *val1 = nullptr, *cnt = nullptr, *f = nullptr,
             *part = nullptr, *run = nullptr, *start = nullptr, *occ = nullptr, *passes = nullptr;
    int32_t* rk = nullptr;
    unsigned* bad = nullptr;
    int rc = DC_OK;
    auto release = [&]() {
        for (void* p : {(void*)key0, (void*)val0, (void*)key1, (void*)val1, (void*)cnt, (void*)f, (void*)part,
                        (void*)run, (void*)start, (void*)occ, (void*)passes, (void*)rk, (void*)bad})
            if (p) cudaFreeAsync(p, st);
    };
    if ((rc = pt_alloc(st, &key0, B)) || (rc = pt_alloc(st, &val0, B)) || (rc = pt_alloc(st, &key1, B)) ||
        (rc = pt_alloc(st, &val1, B)) || (rc = pt_alloc(st, &cnt, kDigits * nblk + 1)) ||
        (rc = pt_alloc(st, &f, B)) || (rc = pt_alloc(st, &part, nblk + 1)) || (rc = pt_alloc(st, &run, B)) ||
        (rc = pt_alloc(st, &start, B)) || (rc = pt_alloc(st, &occ, B)) ||
        (rc = pt_alloc(st, &passes, (uint64_t)K + 2)) || (rc = pt_alloc(st, &rk, B)) || (rc = pt_alloc(st, &bad, 1))) {
        release();
        return rc;
    }
    auto launched = [&](const char* what) -> int {
        ++g_launches;
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? DC_OK
                                : set_error(DC_ERR_CUDA, "edge-batch partition: %s: %s", what, cudaGetErrorString(e));
    };
    do {
        if (cudaMemsetAsync(bad, 0, sizeof(unsigned), st) != cudaSuccess ||
            cudaMemsetAsync(passes, 0, sizeof(uint32_t) * ((uint64_t)K + 2), st) != cudaSuccess) {
            rc = set_error(DC_ERR_CUDA, "edge-batch partition: memset failed");
            break;
        }
        k_pt_roots<<<grid, kPT, 0, st>>>(B, V, d_from, d_to, h->d.kmax_v, key0, val0, rk, bad);
        if ((rc = launched("roots"))) break;
        // stable LSD radix sort of the edge indices by root
        const int bits = V > 1 ? 32 - __builtin_clz(V - 1) : 0;
        for (int shift = 0; shift < bits; shift += kDigitBits) {
            k_pt_digit_count<<<(unsigned)nblk, kPT, 0, st>>>(B, key0, shift, cnt);
            if ((rc = launched("digit count"))) break;
            k_pt_scan_one_block<<<1, kPT, 0, st>>>(cnt, kDigits * nblk);
            if ((rc = launched("digit scan"))) break;
            k_pt_digit_scatter<<<(unsigned)nblk, kPT, 0, st>>>(B, key0, val0, key1, val1, shift, cnt);
            if ((rc = launched("digit scatter"))) break;
            std::swap(key0, key1);
            std::swap(val0, val1);
        }
        if (rc) break;
        // occurrence of every edge's root so far (input order), passes per root kmax
        k_pt_run_flags<<<(unsigned)nblk, kPT, 0, st>>>(B, key0, f, part);
        if ((rc = launched("run flags"))) break;
        k_pt_scan_one_block<<<1, kPT, 0, st>>>(part, nblk);
        if ((rc = launched("run scan"))) break;
        k_pt_runs<<<(unsigned)nblk, kPT, 0, st>>>(B, f, part, run, start);
        if ((rc = launched("runs"))) break;
        k_pt_occ<<<grid, kPT, 0, st>>>(B, val0, run, start, rk, occ, passes);
        if ((rc = launched("occurrences"))) break;
        k_pt_scan_one_block<<<1, kPT, 0, st>>>(passes, (uint64_t)K + 1);
        if ((rc = launched("pass scan"))) break;
        k_pt_number<<<grid, kPT, 0, st>>>(B, rk, occ, passes, d_batch_of);
        if ((rc = launched("numbering"))) break;
        uint32_t total = 0;
        unsigned hbad = 0;
        if (cudaMemcpyAsync(&total, passes + K + 1, sizeof(total), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = set_error(DC_ERR_CUDA, "edge-batch partition: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (hbad) {
            rc = set_error(DC_ERR_INVALID, "edge-batch partition: vertex id out of range");
            break;
        }
        *n_batches = total;
    } while (0);
    release();
    if (rc == DC_OK && cudaStreamSynchronize(st) != cudaSuccess)
        rc = set_error(DC_ERR_CUDA, "edge-batch partition: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

}  // namespace dc
