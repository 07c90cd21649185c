// dvg_internal.h -- host-side structures shared by the translation units of
// libdvg.so.  Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <tuple>
#include <mutex>
#include <unordered_map>
#include <stdexcept>
#include <string>
#include <vector>

#include "dvg.h"

struct dvg_matrix {
  uint32_t nrows = 0;
  uint32_t ncols = 0;
  uint64_t nentries = 0;
  uint64_t nnz = 0;
  uint64_t* rowmap = nullptr;   // device, nrows + 1
  uint32_t* entries = nullptr;  // device, nentries (allocation padded to 16 B)
  bool owned = true;
  bool canonical = true;  // rows sorted, disjoint and non-adjacent (as SpGEMM emits them)
  int device = 0;
};

// Device control block: counters that kernels accumulate into and read back.
struct DeviceControl {
  unsigned long long nnz;        // sum of run lengths of the last product
  unsigned long long range_ops;  // B ranges visited by the last product
  unsigned long long invalid;    // query pairs out of range / validation bits
  unsigned long long status;     // nonzero: a kernel detected an internal error
  unsigned long long total;      // entries of the last fused product
  unsigned long long overflow;   // nonzero: the fused product exceeded its capacity
  unsigned long long timeout;    // nonzero: a bounded device wait gave up
  unsigned long long tiles_direct;  // tiles that took the direct (unstaged) path
  unsigned long long slow_rows;     // row-mode rows that missed the shared window
};

// DeviceControl::status bit of a query that met row pointers outside its
// index's entries (the pair is answered 0, nothing past the entries is read).
constexpr unsigned long long kQueryCorrupt = 128ull;

// A row-kernel shape chosen by the autotuner.
struct TuneChoice {
  int slot_variant;    // run-list entries per thread: 0 -> 16, 1 -> 24, 2 -> 32
  int64_t chunk_rows;  // 0: automatic
};

struct dvg_context {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;      // the stream all work is issued on
  cudaStream_t own_stream = nullptr;  // created by dvg_init
  std::recursive_mutex mu;
  dvg_stats stats{};
  DeviceControl* d_ctl = nullptr;     // device control block
  DeviceControl* h_ctl = nullptr;     // pinned host mirror
  uint64_t* d_tile_sums = nullptr;    // scan scratch
  size_t tile_sums_cap = 0;
  void* d_tile_desc = nullptr;        // fused SpGEMM look-back descriptors
  size_t tile_desc_cap = 0;           // bytes
  unsigned* d_ticket = nullptr;       // fused SpGEMM tile ticket
  uint32_t* d_pairs = nullptr;        // staging for host-buffer queries
  uint8_t* d_answers = nullptr;
  uint64_t pairs_cap = 0;
  int64_t opt_chunk_rows = 0;         // fused SpGEMM look-back chunk rows (0: automatic)
  int64_t opt_spgemm_mode = 0;        // fused SpGEMM: 0 automatic, 1 tiled, 2 light
  int64_t opt_dindex_schedule = 0;    // 0: sum of powers, 1: the reference's squaring
  int64_t opt_row_stage = 1;          // row kernel defers write-out through staging buffers
  uint32_t* d_row_stage = nullptr;    // staging for single products
  size_t row_stage_cap = 0;           // bytes
  int64_t opt_row_slot = 1;           // row kernel run-list width variant (0: 16, 1: 24, 2: 32 entries)
  int64_t opt_levels = 1;             // products with long A ranges read union levels of B (row kernel)
  int64_t opt_spadd_single = 1;       // SpAdd: 1 = one pass with a chunk look-back, 0 = count, scan, fill
  uint32_t row_resident[3] = {0, 0, 0};  // resident CTAs of the row kernel per variant
  int64_t opt_planned = 1;            // 1: index builds run planned (no host round trips)
  double plan_growth = 3.0;           // planned builds: entry capacity per step / input entries
  uint64_t max_product_entries = 0;   // largest product output since the last reset (read-back path)
  int64_t opt_autotune = 1;           // batches: tune the row kernel per (window, size class)
  std::map<std::tuple<unsigned, unsigned, int>, TuneChoice> tuned;
  void* h_stage = nullptr;            // pinned host staging for read-backs
  size_t h_stage_cap = 0;
  std::vector<void*> h_retired;       // outgrown pinned buffers, freed at shutdown
  bool opt_timing = false;
  // event pairs bracketing timed kernels, resolved at the next stream sync
  struct TimedSpan {
    cudaEvent_t begin, end;
    int kind;
  };
  std::vector<TimedSpan> timed;
  std::vector<cudaEvent_t> event_pool;
  // caching allocator: blocks freed by the context are kept (stream order
  // makes their reuse on the context's stream safe) and handed out again
  std::multimap<size_t, void*> free_blocks;      // bytes -> block
  std::unordered_map<void*, size_t> live_blocks;  // block -> bytes
  size_t cached_bytes = 0;
  size_t owned_bytes = 0;   // device memory this context holds (live + cached)
  // the last cudaMemGetInfo answer, when it was taken, and owned_bytes then
  size_t mi_free = 0, mi_owned = 0;
  uint64_t mi_ns = 0;
};

namespace dvg {

// Internal failure; converted to a dvg_status at the C ABI.
struct Error : std::runtime_error {
  dvg_status status;
  Error(dvg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void cuda_check(cudaError_t e, const char* what);
// Throws DVG_ERR_INVALID_ARG with `msg` unless `ok`.
void require(bool ok, const char* msg);
// Sets the message dvg_last_error() returns on the calling thread.
void record_error(const std::string& msg);
#define DVG_CUDA(call) ::dvg::cuda_check((call), #call)

void* dalloc(dvg_context* ctx, size_t bytes);
void dfree(dvg_context* ctx, void* p);
size_t device_free_bytes(dvg_context* ctx);  // free device memory for planning (cached query)
// The range-CRS adjacency of nodes [lower, upper) of a sequence graph
// (dvg_adjacency.cu; arguments as dvg_adjacency_from_graph, host arrays).
dvg_matrix* adjacency_from_graph(dvg_context* ctx, uint32_t nnodes, const uint32_t* node_len,
                                 uint64_t nedges, const uint32_t* edges, uint32_t lower, uint32_t upper);

// A device matrix owned by the context's allocator.
dvg_matrix* new_matrix(dvg_context* ctx, uint32_t nrows, uint32_t ncols, uint64_t nentries);
void free_matrix(dvg_context* ctx, dvg_matrix* m);

// Kernel timing with CUDA events on ctx->stream (active with the "timing"
// option): span_begin records a start event, span_end its end and the kind.
// kProduct: a single-pass SpGEMM kernel; kLevels: building union levels of B
enum TimedKind { kProduct = 0, kLevels = 1, kScan = 2, kSpadd = 3, kQuery = 4 };
cudaEvent_t span_begin(dvg_context* ctx);
void span_end(dvg_context* ctx, cudaEvent_t begin, TimedKind kind);

// The failed checks of a validation word (bits 1, 2, 4, 8 of the validation
// kernels), as "; "-separated text.
std::string validation_message(unsigned long long bits);

// Reads the control block back (synchronises the stream).
DeviceControl read_control(dvg_context* ctx);
void reset_control(dvg_context* ctx);

// Kernels (launch wrappers).  All run on ctx->stream.
void launch_identity(dvg_context* ctx, dvg_matrix* out);
void launch_validate(dvg_context* ctx, const uint64_t* rowmap, uint32_t nrows, const uint32_t* entries,
                     uint64_t nentries, uint32_t ncols);
void launch_widen_rowmap(dvg_context* ctx, const uint32_t* src, uint64_t* dst, uint64_t n);
void launch_narrow_rowmap(dvg_context* ctx, const uint64_t* src, uint32_t* dst, uint64_t n);
// In-place inclusive scan of rowmap[1..n]; rowmap[0] must be 0.
void launch_rowmap_scan(dvg_context* ctx, uint64_t* rowmap, uint64_t n);
void launch_spadd(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, bool b_identity, uint64_t* c_rowmap,
                  uint32_t* c_entries, bool fill);
// C = A + B (B the identity when b_identity) in one pass: c_rowmap written
// fully, c_entries up to `cap` entries (a.nentries + b's entries always
// suffice); the control block receives the total entries, the nnz and a
// timeout flag.  `scratch`: spadd_single_pass_scratch(a->nrows) bytes.
uint64_t spadd_single_pass_scratch(uint32_t nrows);
void launch_spadd_single_pass(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, bool b_identity,
                              uint64_t* c_rowmap, uint32_t* c_entries, uint64_t cap, void* scratch);
// Out-of-range pairs are counted into ctl->invalid (ctx->d_ctl when null).
void launch_query(dvg_context* ctx, const dvg_matrix* idx, const uint32_t* d_pairs, uint64_t npairs, uint8_t* d_out,
                  DeviceControl* ctl = nullptr);

// Fused single-pass SpGEMM (dvg_spgemm_fused.cu): writes c_rowmap fully and
// c_entries up to `cap` entries; the control block receives the total entry
// count, the nnz and an overflow flag when total > cap.
// C = A B, or C = D + A B when d is not null (row kernel only)
// `levels` (row kernel only): union levels of b, level k + 1 at index k.
void launch_spgemm_fused(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b,
                         const dvg_matrix* d, uint64_t* c_rowmap, uint32_t* c_entries, uint64_t cap,
                         const std::vector<dvg_matrix*>* levels = nullptr);
// C = U + S U with S the identity shifted by `shift` rows (row j of C is the
// union of U's rows j and j + shift): one union level from the previous one.
// The warp-per-row SpGEMM for rows that name many B ranges (dvg_spgemm_wide.cu):
// desc holds spgemm_wide_desc_bytes(a->nrows) zeroed bytes, ticket a zeroed word.
size_t spgemm_wide_desc_bytes(uint32_t nrows);
void launch_spgemm_wide(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, const dvg_matrix* d,
                        uint64_t* c_rowmap, uint32_t* c_entries, uint64_t cap, void* desc, unsigned* ticket);
// Range operations a second the warp-per-row kernel's inner work sustains on
// this device (measured; synchronises the context's stream).
double calibrate_range_ops(dvg_context* ctx);
// Random 8-byte reads a second over a buffer of `bytes` (dvg_misc.cu).
double calibrate_random_reads(dvg_context* ctx, uint64_t bytes);
void launch_row_shifted_sum(dvg_context* ctx, const dvg_matrix* u, uint32_t shift, uint64_t* c_rowmap,
                            uint32_t* c_entries, uint64_t cap);

// Thread-per-row single-pass product (dvg_spgemm_rows.cu) on raw arrays:
// C = A B, C = D + A B, or C = I + A B (d_identity); A may be the identity.
// The caller provides zeroed chunk descriptors (desc_bytes of the shape), a
// zeroed ticket and the control block the kernel reports into; `abort`, when
// not null, is checked before any work and set when C is unusable.
struct RowLaunch {
  const uint64_t* a_rowmap = nullptr;
  const uint32_t* a_entries = nullptr;
  bool a_identity = false;
  const uint64_t* b_rowmap = nullptr;
  const uint32_t* b_entries = nullptr;
  const uint64_t* d_rowmap = nullptr;
  const uint32_t* d_entries = nullptr;
  bool d_identity = false;
  uint64_t* c_rowmap = nullptr;
  uint32_t* c_entries = nullptr;
  uint64_t cap = 0;
  uint32_t nrows = 0;
  void* desc = nullptr;
  unsigned* ticket = nullptr;
  DeviceControl* ctl = nullptr;
  unsigned long long* abort = nullptr;
  int slot_variant = 1;  // run-list entries per thread: 0 -> 16, 1 -> 24, 2 -> 32
  uint32_t a_shift = 0;  // with a_identity: A's row r is column r + a_shift (empty past b_nrows)
  uint32_t b_nrows = 0;
  // union levels of B (level k: rows j .. j + 2^k - 1 of B), at most 12
  uint32_t nlevels = 0;
  const uint64_t* lv_rowmap[12] = {};
  const uint32_t* lv_entries[12] = {};
  // staging for deferred write-out, RowLaunchShape::stage_bytes (null: off)
  uint32_t* stage_buf = nullptr;
};
struct RowLaunchShape {
  uint32_t resident, chunk_rows, nchunks, grid;
  size_t desc_bytes;
  size_t stage_bytes;  // staging buffers of the whole grid
};
RowLaunchShape row_launch_shape(dvg_context* ctx, uint32_t nrows, int64_t chunk_rows_opt, int slot_variant);
void launch_rowmode(dvg_context* ctx, const RowLaunch& L, const RowLaunchShape& shape);

int row_slot_entries(int variant);
// Runs the row kernel's look-back on descriptors nothing publishes, its wait
// bounded by spin_limit polls (the kernel records a timeout in the control
// block and returns).
void selftest_bounded_wait(dvg_context* ctx, uint32_t spin_limit);

// Host orchestration (dvg_api.cu).
dvg_matrix* range_spgemm(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b);
dvg_matrix* range_spadd(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, bool b_identity);
dvg_matrix* range_power(dvg_context* ctx, const dvg_matrix* a, unsigned k);
dvg_matrix* create_distance_index(dvg_context* ctx, const dvg_matrix* a, unsigned dlo, unsigned dup);
// Host range-CRS -> device (H2D, validation with one read-back).
dvg_matrix* upload_matrix(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint64_t* rowmap,
                          const uint32_t* entries, uint64_t nnz);
// Device bytes a planned build of an n x n input with `nentries` entries is
// expected to hold at its peak (input, every live step's buffers at `growth`
// times the input's entries, scratch).
uint64_t predict_build_bytes(double growth, uint32_t n, uint64_t nentries, unsigned dlo, unsigned dup);

inline uint64_t matrix_bytes(const dvg_matrix* m) {
  return 8ull * (uint64_t(m->nrows) + 1) + 4ull * m->nentries;
}

// Bytes allocated for `nentries` entries: padded to 16 bytes so vector loads
// of the last range stay inside.
inline size_t entries_alloc_bytes(uint64_t nentries) { return size_t((nentries * 4 + 15) / 16 * 16 + 16); }

uint64_t now_ns();
// Folds the completed event spans into the statistics (after a stream sync).
void resolve_spans(dvg_context* ctx);
// Pinned host staging of at least `bytes` (grown on demand).
void* host_stage(dvg_context* ctx, size_t bytes);

// ---- planned builds (dvg_engine.cu) -----------------------------------------
// The index schedule as a fixed sequence of thread-per-row products whose
// buffers are all allocated before the first launch, so the whole build runs
// without a host round trip (and can be captured in a CUDA graph).  Output
// capacities are estimated; a step whose output overflows sets a device word
// that makes every later step return at once, and the host then re-runs the
// build on the synchronised path.
struct PlanStep {
  int c, a, b, d;      // slots: output, left factor, right factor, addend (-1: none)
  bool a_id, d_id;     // left factor / addend is the identity
};
struct IndexPlan {
  std::vector<PlanStep> steps;
  int nslots = 1;      // slot 0 is the adjacency matrix
  int out = -1;        // slot of the index
};
IndexPlan plan_index(unsigned dlo, unsigned dup);

struct PlannedBuild {
  IndexPlan plan;
  const dvg_matrix* input = nullptr;
  uint32_t n = 0;
  std::vector<uint64_t*> rowmap;    // per slot, as the launches use them (slot 0: the input's)
  std::vector<uint32_t*> entries;
  std::vector<char> live;           // the slot still owns its buffers (not yet handed back)
  std::vector<uint64_t> cap;        // entry capacity per slot
  std::vector<int> owner_step;      // producing step per slot (-1: input)
  RowLaunchShape shape{};
  int slot_variant = 1;
  void* scratch = nullptr;          // chunk descriptors | tickets | controls | abort word
  size_t scratch_bytes = 0;
  size_t desc_stride = 0;
  unsigned* tickets = nullptr;
  DeviceControl* ctls = nullptr;
  unsigned long long* abort = nullptr;
  uint32_t* stage = nullptr;        // row kernel staging (shape.stage_bytes), shared by the steps
};
// Allocates every buffer of the plan for input `a` (no device work beyond
// stream-ordered allocation).
PlannedBuild prepare_build(dvg_context* ctx, const IndexPlan& plan, const dvg_matrix* a);
// The same with the row kernel's run-list width variant and chunk rows given.
PlannedBuild prepare_build(dvg_context* ctx, const IndexPlan& plan, const dvg_matrix* a, int slot_variant,
                           int64_t chunk_rows);
// Issues the build: one memset and one kernel per step, no host round trip.
void launch_build(dvg_context* ctx, PlannedBuild& pb, bool timed);
// Reads the step controls back (one synchronisation), releases the
// intermediates and returns the index, or nullptr after an overflow (all
// buffers released).
dvg_matrix* finish_build(dvg_context* ctx, PlannedBuild& pb);
void release_build(dvg_context* ctx, PlannedBuild& pb);

// ---- batches (dvg_batch.cu) ----------------------------------------------------
// Fastest row-kernel shape for planned builds of `a`'s size class and window,
// timed once per context and kept.
TuneChoice autotune_build(dvg_context* ctx, const dvg_matrix* a, unsigned dlo, unsigned dup);
void batch_distance_index(dvg_context* ctx, uint32_t ngraphs, const dvg_matrix* const* graphs, const unsigned* dmin,
                          const unsigned* dmax, dvg_matrix** out);

}  // namespace dvg
