// dvg_internal.h -- host-side structures shared by the translation units of
// libdvg.so.  Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
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
  int64_t opt_group_lanes = 0;
  int64_t opt_window_words = 0;
  int64_t opt_algo = 0;               // 0: fused tiled SpGEMM, 1: two-pass direct
  int64_t opt_chunk_rows = 0;         // fused SpGEMM look-back chunk rows (0: automatic)
  int64_t opt_spgemm_mode = 0;        // fused SpGEMM: 0 automatic, 1 tiled, 2 light
  int64_t opt_dindex_schedule = 0;    // 0: sum of powers, 1: the reference's squaring
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
};

namespace dvg {

// Internal failure; converted to a dvg_status at the C ABI.
struct Error : std::runtime_error {
  dvg_status status;
  Error(dvg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void cuda_check(cudaError_t e, const char* what);
// Sets the message dvg_last_error() returns on the calling thread.
void record_error(const std::string& msg);
#define DVG_CUDA(call) ::dvg::cuda_check((call), #call)

void* dalloc(dvg_context* ctx, size_t bytes);
void dfree(dvg_context* ctx, void* p);

// A device matrix owned by the context's allocator.
dvg_matrix* new_matrix(dvg_context* ctx, uint32_t nrows, uint32_t ncols, uint64_t nentries);
void free_matrix(dvg_context* ctx, dvg_matrix* m);

// Kernel timing with CUDA events on ctx->stream (active with the "timing"
// option): span_begin records a start event, span_end its end and the kind.
enum TimedKind { kSymbolic = 0, kNumeric = 1, kScan = 2, kSpadd = 3 };
cudaEvent_t span_begin(dvg_context* ctx);
void span_end(dvg_context* ctx, cudaEvent_t begin, TimedKind kind);

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
void launch_query(dvg_context* ctx, const dvg_matrix* idx, const uint32_t* d_pairs, uint64_t npairs, uint8_t* d_out);

struct SpgemmPlan {
  int group_lanes;   // lanes per output row: 4, 8, 16 or 32
  int window_words;  // 32-bit accumulator words per group
};
SpgemmPlan plan_spgemm(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b);
// Symbolic (fill = false: c_rowmap[r+1] = entries of row r, nnz and range_ops
// accumulate in the control block) or numeric (fill = true: rows written at
// c_rowmap offsets) pass of C = A*B.  a_identity: A is the identity of order
// b->nrows and `a` is ignored.
void launch_spgemm(dvg_context* ctx, const SpgemmPlan& plan, const dvg_matrix* a, bool a_identity,
                   const dvg_matrix* b, uint64_t* c_rowmap, uint32_t* c_entries, bool fill);

// Fused single-pass SpGEMM (dvg_spgemm_fused.cu): writes c_rowmap fully and
// c_entries up to `cap` entries; the control block receives the total entry
// count, the nnz and an overflow flag when total > cap.
// C = A B, or C = D + A B when d is not null (row kernel only)
void launch_spgemm_fused(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b,
                         const dvg_matrix* d, uint64_t* c_rowmap, uint32_t* c_entries, uint64_t cap);

// Host orchestration (dvg_api.cu).
dvg_matrix* range_spgemm(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b);
dvg_matrix* range_spadd(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, bool b_identity);
dvg_matrix* range_power(dvg_context* ctx, const dvg_matrix* a, unsigned k);
dvg_matrix* create_distance_index(dvg_context* ctx, const dvg_matrix* a, unsigned dlo, unsigned dup);

inline uint64_t matrix_bytes(const dvg_matrix* m) {
  return 8ull * (uint64_t(m->nrows) + 1) + 4ull * m->nentries;
}

}  // namespace dvg
