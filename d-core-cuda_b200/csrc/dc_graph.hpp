// Host-side handle of one device-resident graph and its decomposition.
//
// HBM layout (all arrays owned by the handle, one CUDA stream per handle):
//   out_off[V+1]  u32   start of v's out-list slot range (capacity = off[v+1]-off[v])
//   out_len[V]    i32   live out-degree of v (first out_len[v] slots are edges)
//   out_nbr[cap]  u32   out-neighbour ids, slack slots after the live prefix
//   in_off / in_len / in_nbr   the same for in-neighbours (CSC)
// This is the reference's device_graph_pointers (src/common.h:81-91) with
// per-list slack generalised from OFFSET_GAP = 1 (src/common.h:36).
//
// Decomposition state:
//   kmax[V]                  in-degree core numbers (g.kmaxes in the reference)
//   sky_off[V+1], sky_k[], sky_l[]
//                            compact skyline: v's value in row k is sky_l of
//                            the last corner with sky_k <= k, for k <= kmax[v];
//                            0 above kmax[v]
//   rows[(kmax+1) * V]       optional dense rows, row-major (g.lmaxes)
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "dc_device.cuh"
#include "../../include/dcore_b200.h"

namespace dc {

struct DevGraph {
    uint32_t V = 0;
    uint64_t E = 0;  // live edges
    uint32_t* out_off = nullptr;
    int32_t* out_len = nullptr;
    uint32_t* out_nbr = nullptr;
    uint32_t* in_off = nullptr;
    int32_t* in_len = nullptr;
    uint32_t* in_nbr = nullptr;
    uint64_t out_cap = 0, in_cap = 0;
    // allocations behind out_nbr / in_nbr (the lists start at the first
    // 16-byte boundary inside them: the row kernel reads ids 16 bytes at a time)
    uint32_t* out_nbr_alloc = nullptr;
    uint32_t* in_nbr_alloc = nullptr;
    bool sorted_kmax = false;  // lists ordered by neighbour kmax of the current graph
};

// Persistent-kernel launch geometry for the current device.
struct LaunchGeom {
    int sms = 0;
    int blocks = 0;   // cooperative grid size
    int threads = 0;  // per block
};

struct Scratch;  // engine scratch buffers (dc_engine.cu)

struct Decomp {
    bool valid = false;
    int32_t kmax = 0;
    int32_t lmax = 0;
    int32_t* kmax_v = nullptr;  // [V]
    int32_t* row0 = nullptr;    // [V] row 0 (out-degree core numbers)
    uint32_t* sky_off = nullptr;
    int32_t* sky_k = nullptr;
    int32_t* sky_l = nullptr;
    uint64_t n_corners = 0;
    uint64_t corner_cap = 0;
    int32_t* rows = nullptr;  // dense rows when materialised
    uint64_t rows_cap = 0;    // elements allocated
    bool rows_valid = false;
    bool peel_valid = false;  // kmax_v and row0 match the current graph
    int32_t row_lo = 1, row_hi = -1;  // rows held besides row 0 (all: 1..kmax)
    // spare skyline buffers that maintenance rotates through (a batch's
    // partial and merged skylines), so steady-state batches allocate nothing
    uint32_t* spare_off[2] = {nullptr, nullptr};
    int32_t* spare_k[2] = {nullptr, nullptr};
    int32_t* spare_l[2] = {nullptr, nullptr};
    uint64_t spare_cap[2] = {0, 0};
    bool full() const { return valid && row_lo <= 1 && row_hi >= kmax; }
    // every row of [k0, k0 + n) is held (row 0 always is)
    bool holds(uint64_t k0, uint64_t n) const {
        if (n == 0) return true;
        const int64_t first = (int64_t)(k0 == 0 ? 1 : k0), last = (int64_t)(k0 + n - 1);
        return last < first || (first >= row_lo && last <= row_hi);
    }
};

struct MaintLogRec {
    float feat[16];
    int32_t method;
    float total_ms, core_ms, rows_ms;
};

struct MaintTimes {
    float apply_ms = 0, core_ms = 0, rows_ms = 0, total_ms = 0;
};

struct PhaseTimes {
    float build_ms = 0, kmax_ms = 0, row0_ms = 0, trans_ms = 0, sky_ms = 0, expand_ms = 0;
};

}  // namespace dc

struct dc_graph {
    int device = 0;
    cudaStream_t stream = nullptr;
    dc::DevGraph g;
    dc::Decomp d;
    dc::LaunchGeom geom;
    dc::EngineCtl* ctl = nullptr;  // device
    dc::Scratch* scratch = nullptr;
    dc::PhaseTimes times;
    dc::MaintTimes mtimes;
    struct dc_sched* sched = nullptr;      // learned maintenance scheduler (not owned)
    bool log_maint = false;                // record features and timings of each batch
    std::vector<dc::MaintLogRec> maint_log;
    cudaEvent_t ev[8] = {};
    uint32_t gap_min = 1;      // minimum free slots per list
    uint32_t gap_div = 0;      // extra slack = len / gap_div (0 = none)
    int method = 0;            // 0 = incremental rows, 1 = per-row peel
    int blocks_per_sm = 0;     // persistent-kernel blocks per SM (0 = default)
    int peel_bps = 0;          // the fused peel's blocks per SM (0 = blocks_per_sm)
    int rows_bps = 0;          // the row kernel's blocks per SM (0 = blocks_per_sm)
    unsigned peel_chunk = 64;  // adjacency entries per peel work item
    int row_repair = 1;        // deletions: repair rows locally instead of recomputing
    // full decompositions: rows cut after kmax * rows_split[i] / 1000 for
    // each nonzero entry (ascending), segments run concurrently
    int rows_split[dc::kMaxRowSegments - 1] = {};
    // corner logs of the segments after the first from the last run:
    // [seg_off[i], seg_off[i] + seg_n[i]), seg_void[i] entries voided (row k < 0)
    int nseg_extra = 0;
    uint64_t seg_off[dc::kMaxRowSegments - 1] = {}, seg_n[dc::kMaxRowSegments - 1] = {},
             seg_void[dc::kMaxRowSegments - 1] = {};
    uint64_t stat_evals = 0, stat_drops = 0, stat_entries = 0;
    uint64_t full_work = 0;  // sum over vertices of degree x kmax at the last full decomposition
    float full_rows_ms = 0;  // rows phase (rows 1..kmax) of the last full decomposition
    // limit of one bounded device wait in ns (0: the default, dc::kWaitNs)
    uint64_t wait_ns = 0;
    // failure-detection tests: block of the next persistent launch that
    // leaves at its first grid barrier without arriving (-1: none)
    int32_t barrier_fault_block = -1;
    // maintenance batches as captured CUDA graphs (dc_maint.cu)
    bool captured_batches = true;
    uint32_t* cb_host = nullptr;           // pinned: batch arrays, then the status block
    uint32_t* cb_dev = nullptr;            // device copy of the batch arrays
    dc::BatchStatus* cb_status = nullptr;  // device status block
    uint64_t cb_words = 0;                 // capacity of cb_host / cb_dev in words (status excluded)
    cudaGraphExec_t cb_exec[2] = {};       // deletion / insertion batch graphs (updated per batch)
    dc::EngineCtl ctl_init{};
    dc::EngineCtl ctl_init_seg[dc::kMaxRowSegments - 1] = {};  // the other row segments'
    // optional per-step trace of persistent kernels (diagnostics)
    unsigned long long* trace_dev = nullptr;
    unsigned long long* trace_host = nullptr;
    unsigned trace_cap = 0;
    unsigned trace_steps = 0;
    void (*trace_cb)(const char* phase, const unsigned long long* rec, unsigned steps, void* user) = nullptr;
    void* trace_user = nullptr;
};
