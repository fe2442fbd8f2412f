// Host entry points of the device engine (implemented in dc_engine.cu).
#pragma once
#include <cstdint>

#include "dc_graph.hpp"

namespace dc {

// One row segment after the first: rows split over concurrent launches,
// each segment with its own values, counters, marks, ticket ring, control
// block and stream.
struct RowSegment {
    uint32_t cap_V = 0;
    int32_t* cur = nullptr;
    int32_t* cnt_out = nullptr;
    int32_t* cnt_in = nullptr;
    uint32_t* mark = nullptr;
    int32_t* stamp = nullptr;
    uint32_t* logidx = nullptr;
    unsigned long long* tring = nullptr;
    uint64_t tring_cap = 0;
    EngineCtl* ctl = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

struct Scratch {
    uint32_t cap_V = 0;
    int32_t* key = nullptr;      // [V] peeling degree / cnt_in
    int32_t* cdeg = nullptr;     // [V] constraint degree
    int32_t* cur = nullptr;      // [V] current row values
    int32_t* row0 = nullptr;     // [V] row 0 values
    uint32_t* mark = nullptr;    // [V]
    int32_t* stamp = nullptr;    // [V]
    uint32_t* logidx = nullptr;  // [V]
    uint32_t* rem0 = nullptr;    // [V]
    uint32_t* rem1 = nullptr;    // [V]
    uint32_t* order = nullptr;   // [V] vertices by kmax descending
    uint32_t* ck = nullptr;      // [kmax+2] |C_k|
    uint32_t ck_cap = 0;
    uint32_t* ring = nullptr;    // ring queue slots
    uint32_t ring_mask = 0;
    uint32_t* log_v = nullptr;
    int32_t* log_k = nullptr;
    int32_t* log_l = nullptr;
    uint64_t log_cap = 0;
    uint64_t* tmp64 = nullptr;   // [V+1] scan scratch
    uint64_t* partial = nullptr; // [blocks] scan scratch
    uint32_t* cursor = nullptr;  // [V+1]
    // second peel instance
    int32_t* key2 = nullptr;
    int32_t* cdeg2 = nullptr;
    uint32_t* rem2 = nullptr;
    uint32_t* rem3 = nullptr;
    int32_t* cnt_out = nullptr;  // [V]
    // ticket-queue ring
    unsigned long long* tring = nullptr;
    uint64_t tring_cap = 0;
    // prunable working copies of the adjacency
    int32_t* w_out_len = nullptr;
    int32_t* w_in_len = nullptr;
    uint32_t* w_out_nbr = nullptr;
    uint32_t* w_in_nbr = nullptr;
    uint64_t w_out_cap = 0, w_in_cap = 0;
    // maintenance
    int32_t* kmax_old = nullptr;  // [V]
    int32_t* row0_old = nullptr;  // [V]
    // row segments after the first (rows split over concurrent launches)
    RowSegment seg[kMaxRowSegments - 1];
    // the graph relabeled in kmax-descending order for the row kernel:
    // new id = position in `order`; lists of new ids sorted by neighbour kmax
    uint32_t* pos = nullptr;                    // [V] new id of each vertex
    int32_t* kmax_r = nullptr;                  // [V] kmax by new id
    int32_t* row0_r = nullptr;                  // [V] row 0 by new id
    uint32_t* r_off[2] = {nullptr, nullptr};    // out / in list starts [V+1]
    int32_t* r_len[2] = {nullptr, nullptr};     // [V]
    uint32_t* r_nbr_alloc[2] = {nullptr, nullptr};
    uint32_t* r_nbr[2] = {nullptr, nullptr};    // 16-byte aligned inside r_nbr_alloc
    uint32_t r_cap_V = 0;
    uint64_t r_cap = 0;                         // list entries per side
};

// Allocation / release (all errors reported through set_error, return DC_*).
int ensure_scratch(dc_graph* h, uint32_t V);
void free_scratch(dc_graph* h);
int init_handle(dc_graph* h);
void free_graph_arrays(DevGraph& g, cudaStream_t st);
void free_decomp(Decomp& d, cudaStream_t st);
// Device bytes currently held by the handle (graph, decomposition, scratch).
uint64_t device_footprint(const dc_graph* h);

// Builds the slack CSR/CSC of h from device edge arrays (src, dst of length E).
int build_from_device_edges(dc_graph* h, uint32_t V, uint64_t E, const uint32_t* d_src, const uint32_t* d_dst);
// Builds from host CSR/CSC arrays in the reference binary layout.
int build_from_host_csr(dc_graph* h, uint32_t V, uint64_t E, const int32_t* in_deg, const int32_t* out_deg,
                        const uint32_t* in_off, const uint32_t* out_off, const uint32_t* in_nbr,
                        const uint32_t* out_nbr, uint64_t nbr_len);

// Batch maintenance (dc_maint.cu).
int maintain(dc_graph* h, const uint32_t* pairs, const uint8_t* is_del, uint64_t b, int method, dc_maint_stats* st);
// Rows 1..R repaired in place after a deletion-only batch (dc_repair.cu),
// giving up after deadline_ns (0: no limit); *applied = false when the caller
// must recompute them instead.
int rows_repair(dc_graph* h, int32_t R, const uint32_t* d_du, const uint32_t* d_dv, uint32_t n_del,
                unsigned long long deadline_ns, bool* applied);
// Deletions per batch below which maintenance splits a mixed batch to repair
// its rows in place.
uint32_t row_repair_max_deletions();
// Whether a row repair after deleting these (device) edges is expected to
// beat recomputing the rows (uses the graph before the deletions).
bool row_repair_worthwhile(dc_graph* h, const uint32_t* d_u, const uint32_t* d_v, uint32_t n);
// Rows 1..R repaired in place after an insertion-only batch (dc_repair.cu),
// giving up after deadline_ns (0: no limit); *applied = false when the caller
// must recompute them instead.
int rows_repair_ins(dc_graph* h, int32_t R, const uint32_t* d_iu, const uint32_t* d_iv, uint32_t n_ins,
                    unsigned long long deadline_ns, bool* applied, unsigned long long* scanned);
// Insertions per batch below which maintenance repairs rows in place.
uint32_t row_repair_max_insertions();
// New skyline from the current one, the updated row 0 and kmax, and the first
// nlog entries of the scratch change log (dc_repair.cu); nlog = 0 when no row
// above 0 changed.
int apply_change_log(dc_graph* h, uint64_t nlog, bool* applied);
// Captured batches (dc_repair.cu): the row maintenance of a batch with its
// decisions in a device status block, enqueued without waiting.
int repair_prepare(dc_graph* h);
int decide_enqueue(dc_graph* h, BatchStatus* st, const int* dbuf, int rmode, uint32_t n_edges, bool insertions);
// Releases a handle's captured-batch graphs and staging buffers (dc_maint.cu).
void free_captured_batches(dc_graph* h);
int repair_enqueue(dc_graph* h, bool insertions, const uint32_t* d_u, const uint32_t* d_v, uint32_t n,
                   uint64_t log_cap, BatchStatus* st);
int merge_enqueue(dc_graph* h, BatchStatus* st, uint32_t* coff, int32_t* ck, int32_t* cl, uint32_t* noff,
                  int32_t* nk, int32_t* nl);
// Change-log capacity of a repair (at least 2^20 entries).
int ensure_change_log(dc_graph* h, uint64_t* cap_out);
// Maintenance method for a batch (rule of thumb or the learned scheduler).
int choose_method(dc_graph* h, uint64_t n_ins, uint64_t n_del);

// KEDGE_BATCHING partition of a device edge batch by the graph's current
// kmax (dc_partition.cu).
int kmax_edge_batches_device(dc_graph* h, uint64_t B, const uint32_t* d_from, const uint32_t* d_to,
                             int64_t* d_batch_of, int64_t* n_batches);

// Text graph parsed on the device into device edge arrays allocated on st
// (dc_parse.cu); .decompCPU formatted on the device.
int parse_text_graph_device(const char* path, int prune, cudaStream_t st, int sms, uint32_t* V_out, uint64_t* E_out,
                            uint32_t** d_src_out, uint32_t** d_dst_out);
int write_decomp_cpu_device(dc_graph* h, const char* path);

// Full decomposition; method 0 = incremental rows, 1 = per-row peel.
int decompose(dc_graph* h, int method, int materialize_rows);
// Rows K0..Kstop from row 0 (in the scratch row0) and kmax; corners left in
// the scratch log.  K0 > 1 jumps from row 0 straight to row K0: the first
// step is the fixpoint of row K0 below row 0, so the corners it logs at K0
// are relative to row 0 and rows 1..K0-1 of the resulting skyline are not
// meaningful.
// allow_relabel: with sorting allowed, run on the graph relabeled in kmax
// order (whole decompositions and row ranges); else sort the handle's lists
// in place (maintenance recomputations, whose graph changes every batch).
int rows_from_row0(dc_graph* h, int32_t K, int32_t Kstop, bool allow_sort, uint64_t* nlog_out, int32_t K0 = 1,
                   bool allow_relabel = true);
// kmax and row 0 (fused peel) when k_first <= 0 or not current, then rows
// max(k_first, 1)..min(k_last, kmax) only; the decomposition then holds row 0
// and that range.
int decompose_range(dc_graph* h, int32_t k_first, int32_t k_last);
// Sum over vertices of (in + out degree) x kmax (a deterministic measure of
// the row work of a graph).
int degree_kmax_sum(dc_graph* h, uint64_t* out);
// out[k] = total in + out degree of C_k (vertices with kmax >= k), k = 0..kmax.
int row_weights(dc_graph* h, uint64_t* out);
// Dense rows [k0, k0+n) into dst (device pointer, row-major, V per row).
int expand_rows(dc_graph* h, uint32_t k0, uint32_t n, int32_t* d_dst);

// Peel of one pass into d_val (device); returns the largest value via *maxval.
int run_peel(dc_graph* h, int which, const int32_t* member, int32_t k, int32_t* d_val, int32_t* maxval, int sync);

// Cooperative launch helper.
int coop_launch(dc_graph* h, const void* fn, void** args, int threads, const char* name);

// Shared host helpers of the engine (dc_engine.cu).
int ensure_tring(dc_graph* h, uint64_t need);
// Device status of a control block (copied back on stream st, which is
// synchronised) converted to DC_* codes.
int check_ctl_on(EngineCtl* ctl, cudaStream_t st, EngineCtl* hc, const char* what);
// bps: blocks per SM for this kernel (0 = the handle's blocks_per_sm, else 2).
int run_persistent(dc_graph* h, const void* fn, void** args, const char* name, EngineCtl* out, int bps = 0);
// Capture-safe forms (no host memory, no waiting): a control block reset by a
// kernel, and a persistent launch after such a reset.
int ctl_init_enqueue(dc_graph* h, EngineCtl* ctl, cudaStream_t st);
int persistent_enqueue(dc_graph* h, const void* fn, void** args, const char* name, EngineCtl* ctl, cudaStream_t st,
                       int bps = 0);
int check_ctl(dc_graph* h, EngineCtl* hc, const char* what);
int scan_tmp64(dc_graph* h, uint64_t n);
// Skyline from row 0 and the corner log: entries [0, nlog) and, when a second
// row segment ran, [off2, off2 + n2).
int build_skyline_from_log(dc_graph* h, uint64_t nlog);
int prepare_row_segments(dc_graph* h);
// Spare skyline buffers (slot 0 or 1): take hands over the slot's buffers with
// room for at least n corners and V + 1 offsets (allocated or grown with a
// quarter of headroom; the slot is left empty); put returns buffers to a slot
// (freeing what it held).
int sky_take_spare(dc_graph* h, int slot, uint64_t n, uint32_t** off, int32_t** k, int32_t** l, uint64_t* cap);
void sky_put_spare(dc_graph* h, int slot, uint32_t* off, int32_t* k, int32_t* l, uint64_t cap);
// kmax (in-degree peel) and row 0 (out-degree peel) of the current graph into
// d.kmax_v and the scratch row 0; reports the largest values.
int peel_kmax_row0(dc_graph* h, int32_t* kmax, int32_t* lmax);

}  // namespace dc
