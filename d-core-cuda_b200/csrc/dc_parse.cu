// GPU-side file formats: the text graph parsed on the device and the
// .decompCPU text written from the device skyline.
//
// Text graph (Graph::readFile, src/graph.cpp:146-250; host restatement in
// dc_io.cpp): the file's bytes go to the device in one copy; newlines are
// found and ranked per 4 KB tile (counts, one scan, a stable scatter of the
// line starts), one thread parses each line with the host parser's rules
// (first line = "# V" header; blank lines and lines starting with '#'
// skipped; "s t" in decimal, each at most 0xFFFFFFFE, else the file is
// malformed; self-loops dropped, duplicates kept), the edges are compacted in
// file order, and, with pruning, vertices without edges are dropped and the
// rest renumbered in increasing id order (pruneEmptyVertices,
// src/graph.cpp:110-144) -- all on the device.  Lines are at most 511 bytes
// (the host parser's line buffer).
//
// .decompCPU (writeDecompFileCPU, src/utils.h:110-124): "V\n", then per
// vertex its row values 0..kmax[v] separated by spaces, a newline after every
// vertex but the last.  Each vertex's line is formatted from its skyline
// corners (a run of equal values per corner), line lengths are scanned, the
// text is written on the device and copied to the host once.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "dc_engine.cuh"
#include "dc_internal.h"

namespace dc {
extern std::atomic<unsigned long long> g_launches;
}

namespace dc {
namespace {

constexpr int kFT = 256;                // threads per block
constexpr int kFBytes = 16;             // bytes (or items) per thread and tile
constexpr int kFTile = kFT * kFBytes;   // per block tile
constexpr int kMaxLine = 511;           // host parser's fgets buffer minus the terminator

__device__ __forceinline__ unsigned long long block_excl_scan_u64(unsigned long long x, unsigned long long* total) {
    __shared__ unsigned long long s_w[kFT / 32 + 1];
    const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    unsigned long long inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= (unsigned)o) inc += y;
    }
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long run = 0;
        for (int i = 0; i < kFT / 32; ++i) {
            unsigned long long t = s_w[i];
            s_w[i] = run;
            run += t;
        }
        s_w[kFT / 32] = run;
    }
    __syncthreads();
    const unsigned long long r = inc - x + s_w[w];
    *total = s_w[kFT / 32];
    __syncthreads();
    return r;
}

// exclusive scan of a[0..n) in place by one block; a[n] = total
__global__ void k_f_scan_one_block(unsigned long long* a, uint64_t n) {
    unsigned long long carry = 0;
    for (uint64_t b = 0; b < n; b += kFT) {
        const uint64_t i = b + threadIdx.x;
        const unsigned long long x = i < n ? a[i] : 0ull;
        unsigned long long tot;
        const unsigned long long ex = block_excl_scan_u64(x, &tot);
        if (i < n) a[i] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) a[n] = carry;
}

// per tile: number of flagged items; flag(i) given as a functor
template <typename Flag>
__global__ void k_f_tile_count(uint64_t n, Flag flag, unsigned long long* part) {
    const uint64_t t0 = (uint64_t)blockIdx.x * kFTile + (uint64_t)threadIdx.x * kFBytes;
    unsigned long long s = 0;
    for (int j = 0; j < kFBytes; ++j)
        if (t0 + j < n) s += flag(t0 + j) ? 1u : 0u;
    unsigned long long tot;
    block_excl_scan_u64(s, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// stable scatter: every flagged item i gets its rank r (items before it that
// are flagged) and emit(i, r) is called
template <typename Flag, typename Emit>
__global__ void k_f_tile_scatter(uint64_t n, Flag flag, Emit emit, const unsigned long long* part) {
    const uint64_t t0 = (uint64_t)blockIdx.x * kFTile + (uint64_t)threadIdx.x * kFBytes;
    unsigned long long s = 0;
    for (int j = 0; j < kFBytes; ++j)
        if (t0 + j < n) s += flag(t0 + j) ? 1u : 0u;
    unsigned long long tot;
    unsigned long long r = block_excl_scan_u64(s, &tot) + part[blockIdx.x];
    for (int j = 0; j < kFBytes; ++j) {
        const uint64_t i = t0 + j;
        if (i < n && flag(i)) emit(i, r++);
    }
}

struct IsNewline {
    const char* b;
    __device__ bool operator()(uint64_t i) const { return b[i] == '\n'; }
};
// line l + 1 starts after the l-th newline
struct LineStart {
    uint64_t* start;
    __device__ void operator()(uint64_t i, unsigned long long r) const { start[r + 1] = i + 1; }
};

__device__ __forceinline__ bool is_blank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// decimal number at b[*p .. e) after blanks and an optional '+'; false when
// there is no digit; *v saturates above 2^40
__device__ bool parse_u(const char* b, uint64_t* p, uint64_t e, unsigned long long* v) {
    uint64_t i = *p;
    while (i < e && is_blank(b[i])) ++i;
    if (i < e && b[i] == '+') ++i;
    unsigned long long x = 0;
    bool any = false;
    while (i < e && b[i] >= '0' && b[i] <= '9') {
        x = x * 10 + (unsigned long long)(b[i] - '0');
        if (x > (1ull << 40)) x = 1ull << 40;
        any = true;
        ++i;
    }
    *p = i;
    *v = x;
    return any;
}

// kind[l]: 0 skipped, 1 edge (src/dst), 2 malformed; line 0 is the header
__global__ void k_f_parse_lines(const char* b, uint64_t nbytes, const uint64_t* start, uint64_t nlines, uint32_t* src,
                                uint32_t* dst, uint8_t* kind, unsigned long long* bad_line, unsigned* maxid,
                                unsigned long long* header_v) {
    for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < nlines; l += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t s = start[l];
        uint64_t e = l + 1 < nlines ? start[l + 1] - 1 : nbytes;  // before the newline
        if (e > s + kMaxLine) e = s + kMaxLine;
        uint8_t k = 0;
        if (l == 0) {
            uint64_t i = s;
            while (i < e && (b[i] == '#' || b[i] == ' ' || b[i] == '\t')) ++i;
            unsigned long long v = 0;
            parse_u(b, &i, e, &v);
            *header_v = v;
        } else {
            uint64_t i = s;
            while (i < e && (b[i] == ' ' || b[i] == '\t')) ++i;
            if (i < e && b[i] != '\r' && b[i] != '#') {
                unsigned long long a = 0, c = 0;
                const bool ok1 = parse_u(b, &i, e, &a);
                const bool ok2 = ok1 && parse_u(b, &i, e, &c);
                if (!ok1 || !ok2 || a > 0xFFFFFFFEull || c > 0xFFFFFFFEull) {
                    k = 2;
                    atomicMin(bad_line, (unsigned long long)l);
                } else if (a != c) {
                    k = 1;
                    src[l] = (uint32_t)a;
                    dst[l] = (uint32_t)c;
                    atomicMax(maxid, (unsigned)max(a, c));
                }
            }
        }
        kind[l] = k;
    }
}

struct IsEdge {
    const uint8_t* kind;
    __device__ bool operator()(uint64_t l) const { return kind[l] == 1; }
};
struct PackEdge {
    const uint32_t* src_l;
    const uint32_t* dst_l;
    uint32_t* src;
    uint32_t* dst;
    __device__ void operator()(uint64_t l, unsigned long long r) const {
        src[r] = src_l[l];
        dst[r] = dst_l[l];
    }
};

__global__ void k_f_mark_used(uint64_t E, const uint32_t* src, const uint32_t* dst, uint8_t* used) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        used[src[e]] = 1;
        used[dst[e]] = 1;
    }
}
struct IsUsed {
    const uint8_t* used;
    __device__ bool operator()(uint64_t v) const { return used[v] != 0; }
};
struct MapUsed {
    uint32_t* map;
    __device__ void operator()(uint64_t v, unsigned long long r) const { map[v] = (uint32_t)r; }
};
__global__ void k_f_renumber(uint64_t E, uint32_t* src, uint32_t* dst, const uint32_t* map) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        src[e] = map[src[e]];
        dst[e] = map[dst[e]];
    }
}

// ---- .decompCPU -------------------------------------------------------------
__device__ __forceinline__ int ndigits(int32_t x) {  // x >= 0
    int n = 1;
    while (x >= 10) {
        x /= 10;
        ++n;
    }
    return n;
}

// bytes of vertex v's line (its newline included except for the last vertex)
__global__ void k_f_line_len(uint32_t V, const int32_t* kmax, const uint32_t* off, const int32_t* ks, const int32_t* ls,
                             unsigned long long* len) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t km = kmax[v];
        unsigned long long n = 0;
        if (off[v] == off[v + 1]) n = 2ull * (km + 1);  // no corner: every value 0
        for (uint32_t i = off[v]; i < off[v + 1]; ++i) {
            const int32_t k0 = ks[i];
            const int32_t k1 = i + 1 < off[v + 1] ? min(ks[i + 1], km + 1) : km + 1;
            if (k1 > k0) n += (unsigned long long)(k1 - k0) * (unsigned long long)(ndigits(ls[i]) + 1);
        }
        // values separated by spaces: one separator fewer than values; a
        // newline after every line but the last
        len[v] = n - 1 + (v + 1 < V ? 1 : 0);
    }
}

__global__ void k_f_write_lines(uint32_t V, const int32_t* kmax, const uint32_t* off, const int32_t* ks,
                                const int32_t* ls, const unsigned long long* pos, char* out) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t km = kmax[v];
        char* o = out + pos[v];
        bool firstv = true;
        if (off[v] == off[v + 1])  // no corner: every value 0
            for (int32_t k = 0; k <= km; ++k) {
                if (!firstv) *o++ = ' ';
                firstv = false;
                *o++ = '0';
            }
        for (uint32_t i = off[v]; i < off[v + 1]; ++i) {
            const int32_t k0 = ks[i];
            const int32_t k1 = i + 1 < off[v + 1] ? min(ks[i + 1], km + 1) : km + 1;
            char dig[12];
            int nd = 0;
            int32_t x = ls[i];
            do {
                dig[nd++] = (char)('0' + x % 10);
                x /= 10;
            } while (x);
            for (int32_t k = k0; k < k1; ++k) {
                if (!firstv) *o++ = ' ';
                firstv = false;
                for (int d = nd - 1; d >= 0; --d) *o++ = dig[d];
            }
        }
        if (v + 1 < V) *o = '\n';
    }
}

template <typename T>
int f_alloc(cudaStream_t st, T** p, uint64_t n) {
    cudaError_t e = cudaMallocAsync((void**)p, std::max<uint64_t>(n, 1) * sizeof(T), st);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return set_error(DC_ERR_NOMEM, "device allocation failed: %s", cudaGetErrorString(e));
    }
    return DC_OK;
}

}  // namespace

// Text graph parsed on the device into device edge arrays (allocated on
// stream st; the caller frees them).  *V, *E as dc_text_read_edges reports.
int parse_text_graph_device(const char* path, int prune, cudaStream_t st, int sms, uint32_t* V_out, uint64_t* E_out,
                            uint32_t** d_src_out, uint32_t** d_dst_out) {
    *d_src_out = *d_dst_out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(DC_ERR_IO, "cannot open graph file '%s': %s", path, strerror(errno));
    fseek(f, 0, SEEK_END);
    const long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size <= 0) {
        fclose(f);
        return set_error(DC_ERR_INVALID, "'%s': empty file (no header line)", path);
    }
    const uint64_t nb = (uint64_t)size;
    char* hbuf = nullptr;
    if (cudaMallocHost((void**)&hbuf, nb) != cudaSuccess) {
        cudaGetLastError();
        fclose(f);
        return set_error(DC_ERR_NOMEM, "pinned host buffer of %llu bytes", (unsigned long long)nb);
    }
    const bool read_ok = fread(hbuf, 1, nb, f) == nb;
    fclose(f);
    if (!read_ok) {
        cudaFreeHost(hbuf);
        return set_error(DC_ERR_IO, "short read of '%s'", path);
    }
    int rc = DC_OK;
    char* d_b = nullptr;
    uint64_t* start = nullptr;
    unsigned long long *part = nullptr, *misc = nullptr;
    uint32_t *src_l = nullptr, *dst_l = nullptr, *src = nullptr, *dst = nullptr, *map = nullptr;
    uint8_t *kind = nullptr, *used = nullptr;
    const int grid = sms * 8;
    auto launched = [&](const char* what) -> int {
        ++g_launches;
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? DC_OK : set_error(DC_ERR_CUDA, "text parse: %s: %s", what, cudaGetErrorString(e));
    };
    uint64_t nlines = 0, E = 0, V = 0;
    do {
        const uint64_t ntile = (nb + kFTile - 1) / kFTile;
        if ((rc = f_alloc(st, &d_b, nb)) || (rc = f_alloc(st, &part, ntile + 1)) || (rc = f_alloc(st, &misc, 4)))
            break;
        if (cudaMemcpyAsync(d_b, hbuf, nb, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            rc = set_error(DC_ERR_CUDA, "text parse: upload failed");
            break;
        }
        // line starts
        IsNewline isnl{d_b};
        k_f_tile_count<<<(unsigned)ntile, kFT, 0, st>>>(nb, isnl, part);
        if ((rc = launched("newline count"))) break;
        k_f_scan_one_block<<<1, kFT, 0, st>>>(part, ntile);
        if ((rc = launched("newline scan"))) break;
        unsigned long long nnl = 0;
        if (cudaMemcpyAsync(&nnl, part + ntile, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = set_error(DC_ERR_CUDA, "text parse: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        // a last line without a newline counts too
        nlines = nnl + (hbuf[nb - 1] != '\n' ? 1 : 0);
        if ((rc = f_alloc(st, &start, nlines + 1))) break;
        const uint64_t zero = 0;
        if (cudaMemcpyAsync(start, &zero, 8, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            rc = set_error(DC_ERR_CUDA, "text parse: upload failed");
            break;
        }
        k_f_tile_scatter<<<(unsigned)ntile, kFT, 0, st>>>(nb, isnl, LineStart{start}, part);
        if ((rc = launched("line starts"))) break;
        // parse every line
        if ((rc = f_alloc(st, &src_l, nlines)) || (rc = f_alloc(st, &dst_l, nlines)) || (rc = f_alloc(st, &kind, nlines)))
            break;
        const unsigned long long init[4] = {~0ull, 0ull, 0ull, 0ull};  // bad line, max id, header V, -
        if (cudaMemcpyAsync(misc, init, sizeof(init), cudaMemcpyHostToDevice, st) != cudaSuccess) {
            rc = set_error(DC_ERR_CUDA, "text parse: upload failed");
            break;
        }
        k_f_parse_lines<<<grid, kFT, 0, st>>>(d_b, nb, start, nlines, src_l, dst_l, kind, misc,
                                              (unsigned*)(misc + 1), misc + 2);
        if ((rc = launched("parse"))) break;
        // compact the edges in file order
        const uint64_t ltile = (nlines + kFTile - 1) / kFTile;
        unsigned long long* lpart = nullptr;
        if ((rc = f_alloc(st, &lpart, ltile + 1))) break;
        IsEdge ise{kind};
        k_f_tile_count<<<(unsigned)ltile, kFT, 0, st>>>(nlines, ise, lpart);
        rc = launched("edge count");
        if (!rc) {
            k_f_scan_one_block<<<1, kFT, 0, st>>>(lpart, ltile);
            rc = launched("edge scan");
        }
        unsigned long long hm[4] = {0, 0, 0, 0}, ne = 0;
        if (!rc && (cudaMemcpyAsync(hm, misc, sizeof(hm), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaMemcpyAsync(&ne, lpart + ltile, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess))
            rc = set_error(DC_ERR_CUDA, "text parse: %s", cudaGetErrorString(cudaGetLastError()));
        if (!rc && hm[0] != ~0ull)
            rc = set_error(DC_ERR_INVALID, "%s:%llu: malformed edge line", path, hm[0] + 1);
        E = ne;
        if (!rc && ((rc = f_alloc(st, &src, E)) || (rc = f_alloc(st, &dst, E)))) {
        }
        if (!rc) {
            k_f_tile_scatter<<<(unsigned)ltile, kFT, 0, st>>>(nlines, ise, PackEdge{src_l, dst_l, src, dst}, lpart);
            rc = launched("edge pack");
        }
        cudaFreeAsync(lpart, st);
        if (rc) break;
        const uint64_t maxid = (unsigned)hm[1];
        V = E ? maxid + 1 : 0;
        if (!prune) {
            V = std::max<uint64_t>(V, hm[2]);
            if (V > 0xFFFFFFFFull) {
                rc = set_error(DC_ERR_INVALID, "'%s': too many vertices", path);
                break;
            }
            break;
        }
        if (V == 0) break;
        // prune: vertices without edges dropped, the rest renumbered in id order
        const uint64_t vtile = (V + kFTile - 1) / kFTile;
        unsigned long long* vpart = nullptr;
        if ((rc = f_alloc(st, &used, V)) || (rc = f_alloc(st, &map, V)) || (rc = f_alloc(st, &vpart, vtile + 1))) {
            if (vpart) cudaFreeAsync(vpart, st);
            break;
        }
        if (cudaMemsetAsync(used, 0, V, st) != cudaSuccess) rc = set_error(DC_ERR_CUDA, "text parse: memset failed");
        if (!rc) {
            k_f_mark_used<<<grid, kFT, 0, st>>>(E, src, dst, used);
            rc = launched("mark used");
        }
        IsUsed isu{used};
        if (!rc) {
            k_f_tile_count<<<(unsigned)vtile, kFT, 0, st>>>(V, isu, vpart);
            rc = launched("used count");
        }
        if (!rc) {
            k_f_scan_one_block<<<1, kFT, 0, st>>>(vpart, vtile);
            rc = launched("used scan");
        }
        if (!rc) {
            k_f_tile_scatter<<<(unsigned)vtile, kFT, 0, st>>>(V, isu, MapUsed{map}, vpart);
            rc = launched("renumber map");
        }
        if (!rc) {
            k_f_renumber<<<grid, kFT, 0, st>>>(E, src, dst, map);
            rc = launched("renumber");
        }
        unsigned long long nv = 0;
        if (!rc && (cudaMemcpyAsync(&nv, vpart + vtile, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess))
            rc = set_error(DC_ERR_CUDA, "text parse: %s", cudaGetErrorString(cudaGetLastError()));
        cudaFreeAsync(vpart, st);
        V = nv;
    } while (0);
    for (void* p : {(void*)d_b, (void*)start, (void*)part, (void*)misc, (void*)src_l, (void*)dst_l, (void*)kind,
                    (void*)used, (void*)map})
        if (p) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaFreeHost(hbuf);
    if (rc) {
        if (src) cudaFreeAsync(src, st);
        if (dst) cudaFreeAsync(dst, st);
        cudaStreamSynchronize(st);
        return rc;
    }
    *V_out = (uint32_t)V;
    *E_out = E;
    *d_src_out = src;
    *d_dst_out = dst;
    return DC_OK;
}

// .decompCPU of the handle's decomposition, formatted on the device.
int write_decomp_cpu_device(dc_graph* h, const char* path) {
    const uint32_t V = h->g.V;
    const Decomp& d = h->d;
    cudaStream_t st = h->stream;
    char head[16];
    const int hn = snprintf(head, sizeof(head), "%u\n", V);
    int rc = DC_OK;
    unsigned long long* len = nullptr;
    char* d_out = nullptr;
    char* hbuf = nullptr;
    unsigned long long total = 0;
    const int grid = h->geom.sms * 8;
    do {
        if (V) {
            if ((rc = f_alloc(st, &len, (uint64_t)V + 1))) break;
            ++g_launches;
            k_f_line_len<<<grid, kFT, 0, st>>>(V, d.kmax_v, d.sky_off, d.sky_k, d.sky_l, len);
            ++g_launches;
            k_f_scan_one_block<<<1, kFT, 0, st>>>(len, V);
            if (cudaMemcpyAsync(&total, len + V, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                rc = set_error(DC_ERR_CUDA, "decompCPU: %s", cudaGetErrorString(cudaGetLastError()));
                break;
            }
            if ((rc = f_alloc(st, &d_out, total))) break;
            ++g_launches;
            k_f_write_lines<<<grid, kFT, 0, st>>>(V, d.kmax_v, d.sky_off, d.sky_k, d.sky_l, len, d_out);
            if (cudaMallocHost((void**)&hbuf, std::max<unsigned long long>(total, 1)) != cudaSuccess) {
                cudaGetLastError();
                rc = set_error(DC_ERR_NOMEM, "pinned host buffer of %llu bytes", total);
                break;
            }
            if (cudaMemcpyAsync(hbuf, d_out, total, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                rc = set_error(DC_ERR_CUDA, "decompCPU: %s", cudaGetErrorString(cudaGetLastError()));
                break;
            }
        }
        FILE* f = fopen(path, "wb");
        if (!f) {
            rc = set_error(DC_ERR_IO, "cannot write '%s': %s", path, strerror(errno));
            break;
        }
        bool ok = fwrite(head, 1, (size_t)hn, f) == (size_t)hn;
        if (ok && total) ok = fwrite(hbuf, 1, total, f) == total;
        if (fclose(f) != 0) ok = false;
        if (!ok) rc = set_error(DC_ERR_IO, "short write to '%s'", path);
    } while (0);
    if (len) cudaFreeAsync(len, st);
    if (d_out) cudaFreeAsync(d_out, st);
    cudaStreamSynchronize(st);
    if (hbuf) cudaFreeHost(hbuf);
    return rc;
}

}  // namespace dc
