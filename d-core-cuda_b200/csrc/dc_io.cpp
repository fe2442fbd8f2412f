// Host-side file formats of the reference, restated:
//   text graph      "# V" header line, then one "s t" edge per line
//                   (Graph::readFile, src/graph.cpp:146-250): self-loops are
//                   dropped (:167), duplicate edges kept, vertices without
//                   edges pruned and the rest renumbered in increasing id
//                   order (pruneEmptyVertices, src/graph.cpp:110-144).
//   binary graph    "<file>-binary-g=<GAP>" (Graph::writeBinary/readBinary,
//                   src/graph.cpp:261-325): V:u32, E:u32, in_deg[V]:i32,
//                   out_deg[V]:i32, in_off[V+1]:u32, out_off[V+1]:u32,
//                   in_nbr[E+GAP*V]:u32, out_nbr[E+GAP*V]:u32.
//   .decomp         kmax:i32, lmax:i32, kmaxes[V]:i32, lmaxes[kmax+1][V]:i32
//                   (writeDecompFile / readDecompFile, src/utils.h:76-109)
//   .decompCPU      text: V, then per vertex its row values 0..kmax[v]
//                   separated by spaces, one vertex per line, no newline
//                   after the last (writeDecompFileCPU, src/utils.h:110-124)
// All functions here are host-only and need no GPU.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dc_internal.h"

namespace dc {

// Parses the text format.  prune != 0 applies the reference's empty-vertex
// pruning and renumbering; prune == 0 keeps ids as they are, with
// V = max(header V, max id + 1).
int parse_text_graph(const char* path, int prune, uint32_t* V_out, std::vector<uint32_t>& src,
                     std::vector<uint32_t>& dst) {
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(DC_ERR_IO, "cannot open graph file '%s': %s", path, strerror(errno));
    src.clear();
    dst.clear();
    char line[512];
    uint64_t header_V = 0;
    bool first = true;
    uint64_t maxid = 0;
    bool any = false;
    uint64_t lineno = 0;
    while (fgets(line, sizeof(line), f)) {
        ++lineno;
        if (first) {
            first = false;
            // first line is the vertex-count header ("# V"); the reference
            // ignores its value (src/graph.cpp:156-158)
            const char* p = line;
            while (*p == '#' || *p == ' ' || *p == '\t') ++p;
            header_V = strtoull(p, nullptr, 10);
            continue;
        }
        char* p = line;
        while (*p == ' ' || *p == '\t') ++p;
        if (*p == '\0' || *p == '\n' || *p == '\r' || *p == '#') continue;
        char* e1 = nullptr;
        errno = 0;
        unsigned long long s = strtoull(p, &e1, 10);
        if (e1 == p) {
            fclose(f);
            return set_error(DC_ERR_INVALID, "%s:%llu: malformed edge line", path, (unsigned long long)lineno);
        }
        char* e2 = nullptr;
        unsigned long long t = strtoull(e1, &e2, 10);
        if (e2 == e1 || errno == ERANGE || s > 0xFFFFFFFEull || t > 0xFFFFFFFEull) {
            fclose(f);
            return set_error(DC_ERR_INVALID, "%s:%llu: malformed edge line", path, (unsigned long long)lineno);
        }
        if (s == t) continue;  // no self loops
        src.push_back((uint32_t)s);
        dst.push_back((uint32_t)t);
        maxid = std::max<uint64_t>(maxid, std::max(s, t));
        any = true;
    }
    fclose(f);
    if (first) return set_error(DC_ERR_INVALID, "'%s': empty file (no header line)", path);
    uint64_t V = any ? maxid + 1 : 0;
    if (!prune) {
        V = std::max<uint64_t>(V, header_V);
        if (V > 0xFFFFFFFFull) return set_error(DC_ERR_INVALID, "'%s': too many vertices", path);
        *V_out = (uint32_t)V;
        return DC_OK;
    }
    std::vector<uint8_t> used((size_t)V, 0);
    for (size_t i = 0; i < src.size(); ++i) used[src[i]] = used[dst[i]] = 1;
    std::vector<uint32_t> map((size_t)V, 0);
    uint32_t n = 0;
    for (uint64_t v = 0; v < V; ++v)
        if (used[v]) map[v] = n++;
    for (size_t i = 0; i < src.size(); ++i) {
        src[i] = map[src[i]];
        dst[i] = map[dst[i]];
    }
    *V_out = n;
    return DC_OK;
}

int read_binary_graph(const char* path, BinaryGraph& b) {
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(DC_ERR_IO, "cannot open binary graph '%s': %s", path, strerror(errno));
    fseek(f, 0, SEEK_END);
    long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    auto rd = [&](void* p, size_t bytes) { return fread(p, 1, bytes, f) == bytes; };
    if (size < 8 || !rd(&b.V, 4) || !rd(&b.E, 4)) {
        fclose(f);
        return set_error(DC_ERR_INVALID, "'%s': truncated binary header", path);
    }
    uint64_t V = b.V;
    uint64_t fixed = 8 + 8 * V + 8 * (V + 1);
    if ((uint64_t)size < fixed) {
        fclose(f);
        return set_error(DC_ERR_INVALID, "'%s': truncated binary graph (V=%u)", path, b.V);
    }
    b.in_deg.resize(V);
    b.out_deg.resize(V);
    b.in_off.resize(V + 1);
    b.out_off.resize(V + 1);
    bool ok = rd(b.in_deg.data(), 4 * V) && rd(b.out_deg.data(), 4 * V) && rd(b.in_off.data(), 4 * (V + 1)) &&
              rd(b.out_off.data(), 4 * (V + 1));
    if (!ok) {
        fclose(f);
        return set_error(DC_ERR_INVALID, "'%s': truncated binary graph", path);
    }
    uint64_t slots = b.in_off[V];
    if (b.out_off[V] != slots || (uint64_t)size != fixed + 8 * slots) {
        fclose(f);
        return set_error(DC_ERR_INVALID, "'%s': binary graph size does not match its offsets", path);
    }
    b.in_nbr.resize(slots);
    b.out_nbr.resize(slots);
    ok = rd(b.in_nbr.data(), 4 * slots) && rd(b.out_nbr.data(), 4 * slots);
    fclose(f);
    if (!ok) return set_error(DC_ERR_INVALID, "'%s': truncated adjacency", path);
    // validate: degrees fit their slot ranges, ids in range, sums match E
    uint64_t so = 0, si = 0;
    for (uint64_t v = 0; v < V; ++v) {
        if (b.in_off[v] > b.in_off[v + 1] || b.out_off[v] > b.out_off[v + 1] || b.in_deg[v] < 0 || b.out_deg[v] < 0 ||
            (uint64_t)b.in_deg[v] > b.in_off[v + 1] - b.in_off[v] ||
            (uint64_t)b.out_deg[v] > b.out_off[v + 1] - b.out_off[v])
            return set_error(DC_ERR_INVALID, "'%s': inconsistent degrees/offsets at vertex %llu", path,
                             (unsigned long long)v);
        for (int32_t i = 0; i < b.out_deg[v]; ++i)
            if (b.out_nbr[b.out_off[v] + i] >= V) return set_error(DC_ERR_INVALID, "'%s': neighbour id out of range", path);
        for (int32_t i = 0; i < b.in_deg[v]; ++i)
            if (b.in_nbr[b.in_off[v] + i] >= V) return set_error(DC_ERR_INVALID, "'%s': neighbour id out of range", path);
        so += b.out_deg[v];
        si += b.in_deg[v];
    }
    if (so != b.E || si != b.E)
        return set_error(DC_ERR_INVALID, "'%s': degree sums (%llu out, %llu in) differ from E=%u", path,
                         (unsigned long long)so, (unsigned long long)si, b.E);
    return DC_OK;
}

// Writes V/E + CSR/CSC in the reference binary layout.  Each list is written
// in ascending neighbour order followed by `gap` free slots filled with
// 0xCDCDCDCD, the fill the reference's files carry in their free slots.
int write_binary_graph(const char* path, uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                       uint32_t gap) {
    if (E > 0xFFFFFFFFull) return set_error(DC_ERR_INVALID, "binary format holds at most 2^32-1 edges");
    std::vector<int32_t> ideg(V, 0), odeg(V, 0);
    for (uint64_t e = 0; e < E; ++e) {
        if (src[e] >= V || dst[e] >= V) return set_error(DC_ERR_INVALID, "edge endpoint out of range");
        odeg[src[e]]++;
        ideg[dst[e]]++;
    }
    std::vector<uint32_t> ioff((size_t)V + 1), ooff((size_t)V + 1);
    uint64_t si = 0, so = 0;
    for (uint32_t v = 0; v < V; ++v) {
        ioff[v] = (uint32_t)si;
        ooff[v] = (uint32_t)so;
        si += (uint64_t)ideg[v] + gap;
        so += (uint64_t)odeg[v] + gap;
    }
    if (si > 0xFFFFFFFFull) return set_error(DC_ERR_INVALID, "binary format offsets overflow u32");
    ioff[V] = (uint32_t)si;
    ooff[V] = (uint32_t)so;
    std::vector<uint32_t> inb(si, 0xCDCDCDCDu), onb(so, 0xCDCDCDCDu);
    std::vector<uint32_t> fi(V, 0), fo(V, 0);
    for (uint64_t e = 0; e < E; ++e) {
        onb[ooff[src[e]] + fo[src[e]]++] = dst[e];
        inb[ioff[dst[e]] + fi[dst[e]]++] = src[e];
    }
    for (uint32_t v = 0; v < V; ++v) {
        std::sort(onb.begin() + ooff[v], onb.begin() + ooff[v] + odeg[v]);
        std::sort(inb.begin() + ioff[v], inb.begin() + ioff[v] + ideg[v]);
    }
    FILE* f = fopen(path, "wb");
    if (!f) return set_error(DC_ERR_IO, "cannot write '%s': %s", path, strerror(errno));
    uint32_t E32 = (uint32_t)E;
    bool ok = fwrite(&V, 4, 1, f) == 1 && fwrite(&E32, 4, 1, f) == 1 &&
              fwrite(ideg.data(), 4, V, f) == V && fwrite(odeg.data(), 4, V, f) == V &&
              fwrite(ioff.data(), 4, (size_t)V + 1, f) == (size_t)V + 1 &&
              fwrite(ooff.data(), 4, (size_t)V + 1, f) == (size_t)V + 1 && fwrite(inb.data(), 4, si, f) == si &&
              fwrite(onb.data(), 4, so, f) == so;
    ok = (fclose(f) == 0) && ok;
    if (!ok) return set_error(DC_ERR_IO, "short write to '%s'", path);
    return DC_OK;
}

}  // namespace dc

using namespace dc;

extern "C" int dc_text_read_edges(const char* path, int prune, uint32_t* V, uint64_t* E, uint32_t* src,
                                  uint32_t* dst, uint64_t capacity) {
    if (!path || !V || !E) return set_error(DC_ERR_INVALID, "dc_text_read_edges: null argument");
    std::vector<uint32_t> s, d;
    if (int rc = parse_text_graph(path, prune, V, s, d)) return rc;
    *E = s.size();
    if (!src || !dst) return DC_OK;
    if (capacity < s.size()) return set_error(DC_ERR_CAPACITY, "dc_text_read_edges: capacity %llu < %llu edges",
                                              (unsigned long long)capacity, (unsigned long long)s.size());
    std::memcpy(src, s.data(), s.size() * 4);
    std::memcpy(dst, d.data(), d.size() * 4);
    return DC_OK;
}

extern "C" int dc_binary_read_edges(const char* path, uint32_t* V, uint64_t* E, uint32_t* src, uint32_t* dst,
                                    uint64_t capacity) {
    if (!path || !V || !E) return set_error(DC_ERR_INVALID, "dc_binary_read_edges: null argument");
    BinaryGraph b;
    if (int rc = read_binary_graph(path, b)) return rc;
    *V = b.V;
    *E = b.E;
    if (!src || !dst) return DC_OK;
    if (capacity < b.E) return set_error(DC_ERR_CAPACITY, "dc_binary_read_edges: capacity too small");
    uint64_t e = 0;
    for (uint32_t v = 0; v < b.V; ++v)
        for (int32_t i = 0; i < b.out_deg[v]; ++i) {
            src[e] = v;
            dst[e] = b.out_nbr[b.out_off[v] + i];
            ++e;
        }
    return DC_OK;
}

extern "C" int dc_binary_write_edges(const char* path, uint32_t V, uint64_t E, const uint32_t* src,
                                     const uint32_t* dst, uint32_t gap) {
    if (!path || (E && (!src || !dst))) return set_error(DC_ERR_INVALID, "dc_binary_write_edges: null argument");
    return write_binary_graph(path, V, E, src, dst, gap);
}

extern "C" int dc_decomp_file_write(const char* path, uint32_t V, int32_t kmax, int32_t lmax, const int32_t* kmaxes,
                                    const int32_t* rows) {
    if (!path || (V && (!kmaxes || !rows)) || kmax < 0) return set_error(DC_ERR_INVALID, "dc_decomp_file_write: bad argument");
    FILE* f = fopen(path, "wb");
    if (!f) return set_error(DC_ERR_IO, "cannot write '%s': %s", path, strerror(errno));
    uint64_t n = (uint64_t)(kmax + 1) * V;
    bool ok = fwrite(&kmax, 4, 1, f) == 1 && fwrite(&lmax, 4, 1, f) == 1 && fwrite(kmaxes, 4, V, f) == V &&
              fwrite(rows, 4, n, f) == n;
    ok = (fclose(f) == 0) && ok;
    return ok ? DC_OK : set_error(DC_ERR_IO, "short write to '%s'", path);
}

// Reads a .decomp file.  With kmaxes or rows NULL (or rows_cap too small)
// only *kmax / *lmax are filled and DC_ERR_CAPACITY is returned when rows
// were requested but do not fit.
extern "C" int dc_decomp_file_read(const char* path, uint32_t V, int32_t* kmax, int32_t* lmax, int32_t* kmaxes,
                                   int32_t* rows, uint64_t rows_cap) {
    if (!path || !kmax || !lmax) return set_error(DC_ERR_INVALID, "dc_decomp_file_read: null argument");
    FILE* f = fopen(path, "rb");
    if (!f) return set_error(DC_ERR_IO, "cannot open '%s': %s", path, strerror(errno));
    fseek(f, 0, SEEK_END);
    long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size < 8 || fread(kmax, 4, 1, f) != 1 || fread(lmax, 4, 1, f) != 1 || *kmax < 0) {
        fclose(f);
        return set_error(DC_ERR_INVALID, "'%s': bad .decomp header", path);
    }
    uint64_t want = 8 + 4ull * V + 4ull * (uint64_t)(*kmax + 1) * V;
    if ((uint64_t)size != want) {
        fclose(f);
        return set_error(DC_ERR_INVALID, "'%s': size %lld does not match V=%u, kmax=%d", path, size, V, *kmax);
    }
    if (!kmaxes || !rows) {
        fclose(f);
        return DC_OK;
    }
    uint64_t n = (uint64_t)(*kmax + 1) * V;
    if (rows_cap < n) {
        fclose(f);
        return set_error(DC_ERR_CAPACITY, "dc_decomp_file_read: rows capacity %llu < %llu",
                         (unsigned long long)rows_cap, (unsigned long long)n);
    }
    bool ok = fread(kmaxes, 4, V, f) == V && fread(rows, 4, n, f) == n;
    fclose(f);
    return ok ? DC_OK : set_error(DC_ERR_INVALID, "'%s': truncated", path);
}

extern "C" int dc_decomp_cpu_file_write(const char* path, uint32_t V, const int32_t* kmaxes, const int32_t* rows) {
    if (!path || (V && (!kmaxes || !rows))) return set_error(DC_ERR_INVALID, "dc_decomp_cpu_file_write: bad argument");
    FILE* f = fopen(path, "wb");
    if (!f) return set_error(DC_ERR_IO, "cannot write '%s': %s", path, strerror(errno));
    fprintf(f, "%u\n", V);
    for (uint32_t v = 0; v < V; ++v) {
        int32_t end = kmaxes[v];
        for (int32_t j = 0; j <= end; ++j) {
            fprintf(f, "%d", rows[(uint64_t)j * V + v]);
            if (j < end) fputc(' ', f);
        }
        if (v != V - 1) fputc('\n', f);
    }
    return fclose(f) == 0 ? DC_OK : set_error(DC_ERR_IO, "short write to '%s'", path);
}
