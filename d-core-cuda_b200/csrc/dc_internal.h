// Internal helpers shared by the engine's translation units: error status
// plumbing for the C ABI.  Every exported function returns DC_OK (0) or a
// negative DC_ERR_* code and records a message readable via dc_last_error().
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/dcore_b200.h"

namespace dc {

int set_error(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();

void radix_sort_u64(uint64_t* keys, uint64_t* tmp, size_t n, int bits);

}  // namespace dc

#include <vector>

namespace dc {

struct BinaryGraph {
    uint32_t V = 0, E = 0;
    std::vector<int32_t> in_deg, out_deg;
    std::vector<uint32_t> in_off, out_off, in_nbr, out_nbr;
};

int parse_text_graph(const char* path, int prune, uint32_t* V_out, std::vector<uint32_t>& src,
                     std::vector<uint32_t>& dst);
int read_binary_graph(const char* path, BinaryGraph& b);
int write_binary_graph(const char* path, uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                       uint32_t gap);

}  // namespace dc
