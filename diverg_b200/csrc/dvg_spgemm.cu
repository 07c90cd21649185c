// dvg_spgemm.cu -- range-CRS Boolean SpGEMM C = A*B on sm_100a.
//
// Follows the semantics of the reference's TeamSequential / HBitVector
// SpGEMM (include/diverg/range_sparse.hpp:1132-1442 in cartoonist/diverg):
// row r of C is the union, over every range [s,f] of A's row r, of all
// ranges of B rows s..f (one contiguous slice of B.entries), emitted as
// sorted maximal runs.  The output is canonical, so it is bit-identical to
// every accumulator and partition of the reference.
//
// B200 design:
//  * a group of G lanes (G = 4..32, chosen per product from the work per row)
//    owns one output row; a CTA holds 256/G groups; rows are interleaved over
//    the whole grid so concurrently running groups read neighbouring B rows
//    and reuse them from L1/L2;
//  * the accumulator is a per-group window of W 32-bit words in shared memory
//    plus a "reach" word per bitset: a B range [s,e] costs at most three
//    shared-memory atomics however long it is (its two edge words are ORed,
//    the full words in between are recorded as one max at the first of them);
//    a prefix max over `reach` while gathering turns them into full words.
//    This replaces the reference's per-word range set (hbitvector.hpp:
//    1155-1233) whose cost grows with the range length;
//  * rows whose column band exceeds the window are processed in consecutive
//    column chunks carrying the boundary state across (the reference instead
//    spills to a full-width L2 bitvector in global memory per team);
//  * the gather maps every word x with carry c = msb(previous word) to run
//    starts (x ^ (x<<1|c)) & x and run ends ((x<<1|c) & ~x), as the
//    reference's map01/map10 (hbitvector.hpp:568-597), counts them with popc,
//    places them with a group prefix sum (instead of the reference's quadratic
//    recount, range_sparse.hpp:1411-1421) and extracts them with ffs; a zero
//    word is kept after the band so every run closes inside it and the
//    reference's last-word fix-up (range_sparse.hpp:1435-1440) is not needed.
#include <algorithm>

#include "dvg_device.cuh"
#include "dvg_internal.h"

namespace dvg {
namespace {

constexpr int kThreads = 256;

struct SpgemmArgs {
  const uint64_t* __restrict__ a_rowmap;
  const uint32_t* __restrict__ a_entries;
  const uint64_t* __restrict__ b_rowmap;
  const uint32_t* __restrict__ b_entries;
  uint64_t* __restrict__ c_rowmap;
  uint32_t* __restrict__ c_entries;
  DeviceControl* ctl;
  uint32_t nrows;  // rows of A and C
  uint32_t ww;     // accumulator window words per group
};

// One A range [s, f] as the slice of B range indices [b0, b1).
struct Slice {
  uint64_t b0, b1;
};

template <bool A_IDENTITY>
__device__ __forceinline__ Slice a_slice(const SpgemmArgs& p, uint64_t row, uint64_t ai) {
  uint32_t s, f;
  if constexpr (A_IDENTITY) {
    s = f = uint32_t(row);
  } else {
    uint2 r = load_range(p.a_entries, ai >> 1);
    s = r.x;
    f = r.y;
  }
  if (f < s) return {0, 0};
  return {__ldg(p.b_rowmap + s) >> 1, __ldg(p.b_rowmap + uint64_t(f) + 1) >> 1};
}

template <int G, bool A_IDENTITY, bool FILL>
__global__ void __launch_bounds__(kThreads) k_spgemm_rows(SpgemmArgs p) {
  extern __shared__ uint32_t smem[];
  __shared__ unsigned long long cta_nnz, cta_ops;
  const int lg = lane_id() & (G - 1);
  const unsigned gm = group_mask<G>();
  const int gid = threadIdx.x / G;
  constexpr int kGroups = kThreads / G;
  uint32_t* bits = smem + size_t(gid) * 2 * p.ww;
  uint32_t* reach = bits + p.ww;
  if (threadIdx.x == 0) {
    cta_nnz = 0;
    cta_ops = 0;
  }
  __syncthreads();
  unsigned long long my_nnz = 0, my_ops = 0;

  for (uint64_t row = uint64_t(blockIdx.x) * kGroups + gid; row < p.nrows;
       row += uint64_t(gridDim.x) * kGroups) {
    uint64_t a0, a1;
    if constexpr (A_IDENTITY) {
      a0 = 0;
      a1 = 2;
    } else {
      a0 = __ldg(p.a_rowmap + row);
      a1 = __ldg(p.a_rowmap + row + 1);
    }

    // Pass 1: column band [mn, mx] of the row and the number of B ranges.
    uint32_t mn = 0xffffffffu, mx = 0;
    uint64_t nranges = 0;
    for (uint64_t ai = a0; ai < a1; ai += 2) {
      Slice sl = a_slice<A_IDENTITY>(p, row, ai);
      if (sl.b1 > sl.b0) nranges += sl.b1 - sl.b0;
      for (uint64_t t = sl.b0 + lg; t < sl.b1; t += G) {
        uint2 r = load_range(p.b_entries, t);
        mn = min(mn, r.x);
        mx = max(mx, r.y);
      }
    }
    mn = group_min<G>(gm, mn);
    mx = group_max<G>(gm, mx);
    my_ops += nranges;

    uint64_t out_pos = 0, out_end = 0;
    if constexpr (FILL) {
      out_pos = p.c_rowmap[row];
      out_end = p.c_rowmap[row + 1];
    }
    uint64_t count = 0;  // entries emitted for this row (group-uniform)
    if (mn <= mx) {
      const uint64_t base = mn & ~31u;
      // one extra word after the band stays zero, so every run closes inside
      const uint64_t nw_total = ((uint64_t(mx) - base) >> 5) + 2;
      uint32_t carry = 0;  // msb of the previous word
      for (uint64_t w0 = 0; w0 < nw_total; w0 += p.ww) {
        const uint32_t nwc = uint32_t(min(uint64_t(p.ww), nw_total - w0));
        const uint64_t cb = base + 32 * w0;          // first column of the chunk
        const uint64_t ce = cb + 32ull * nwc - 1;    // last column of the chunk
        for (uint32_t w = lg; w < nwc; w += G) {
          bits[w] = 0;
          reach[w] = 0;
        }
        __syncwarp(gm);
        // Pass 2: accumulate the clipped B ranges.
        for (uint64_t ai = a0; ai < a1; ai += 2) {
          Slice sl = a_slice<A_IDENTITY>(p, row, ai);
          for (uint64_t t = sl.b0 + lg; t < sl.b1; t += G) {
            uint2 r = load_range(p.b_entries, t);
            uint64_t cs = max(uint64_t(r.x), cb);
            uint64_t cf = min(uint64_t(r.y), ce);
            if (cs > cf || r.y < r.x) continue;
            uint32_t ws = uint32_t((cs - cb) >> 5), we = uint32_t((cf - cb) >> 5);
            uint32_t lo = ~0u << (cs & 31);
            uint32_t hi = ~0u >> (31 - (cf & 31));
            if (ws == we) {
              atomicOr(bits + ws, lo & hi);
            } else {
              atomicOr(bits + ws, lo);
              atomicOr(bits + we, hi);
              if (we > ws + 1) atomicMax(reach + ws + 1, we);
            }
          }
        }
        __syncwarp(gm);
        // Pass 3: gather runs.
        uint32_t run_reach = 0;
        for (uint32_t wb = 0; wb < nwc; wb += G) {
          const uint32_t w = wb + lg;
          const bool valid = w < nwc;
          uint32_t x = 0, rr = 0;
          if (valid) {
            x = bits[w];
            rr = reach[w];
          }
          rr = group_incl_max<G>(gm, rr, lg);
          rr = max(rr, run_reach);
          if (valid && rr > w) x = ~0u;
          run_reach = group_bcast<G>(gm, rr, G - 1);
          uint32_t prev = __shfl_up_sync(gm, x, 1, G);
          uint32_t c = lg == 0 ? carry : (prev >> 31);
          uint32_t sh = (x << 1) | c;
          // lanes past the chunk's last word emit nothing: a run open there
          // continues into the next chunk (the final chunk ends on a zero word)
          uint32_t bnd = valid ? (((x ^ sh) & x) | (sh & ~x)) : 0u;
          uint32_t cnt = __popc(bnd);
          my_nnz += __popc(x);
          uint32_t incl = group_incl_sum<G>(gm, cnt, lg);
          if constexpr (FILL) {
            uint64_t k = count + incl - cnt;  // row-local index of the first boundary
            const uint64_t col0 = cb + 32ull * w;
            while (bnd) {
              int b = __ffs(bnd) - 1;
              bnd &= bnd - 1;
              uint64_t pos = out_pos + k;
              if (pos < out_end) {
                p.c_entries[pos] = uint32_t(col0 + b - (k & 1));
              } else {
                atomicOr(&p.ctl->status, 1ull);
              }
              ++k;
            }
          }
          count += group_bcast<G>(gm, incl, G - 1);
          carry = group_bcast<G>(gm, x, int(min(uint32_t(G - 1), nwc - 1 - wb))) >> 31;
        }
        __syncwarp(gm);
      }
    }
    if constexpr (!FILL) {
      if (lg == 0) p.c_rowmap[row + 1] = count;
    } else {
      if (lg == 0 && out_pos + count != out_end) atomicOr(&p.ctl->status, 2ull);
    }
  }
  if constexpr (!FILL) {
    // nnz was counted by every lane over its own words; ops once per group
    if (lg != 0) my_ops = 0;
    atomicAdd(&cta_nnz, my_nnz);
    atomicAdd(&cta_ops, my_ops);
    __syncthreads();
    if (threadIdx.x == 0) {
      atomicAdd(&p.ctl->nnz, cta_nnz);
      atomicAdd(&p.ctl->range_ops, cta_ops);
    }
  }
}

template <int G, bool A_IDENTITY, bool FILL>
void launch_t(dvg_context* ctx, const SpgemmArgs& args) {
  auto kern = k_spgemm_rows<G, A_IDENTITY, FILL>;
  const size_t smem = size_t(kThreads / G) * 2 * args.ww * sizeof(uint32_t);
  if (smem > 48 * 1024) DVG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int per_sm = 0;
  DVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
  if (per_sm < 1) throw Error(DVG_ERR_INVALID_ARG, "spgemm: accumulator window too large for shared memory");
  const uint64_t groups = kThreads / G;
  uint64_t want = (uint64_t(args.nrows) + groups - 1) / groups;
  uint64_t cap = uint64_t(per_sm) * ctx->num_sms;
  unsigned grid = unsigned(std::max<uint64_t>(1, std::min(want, cap)));
  kern<<<grid, kThreads, smem, ctx->stream>>>(args);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

template <bool A_IDENTITY, bool FILL>
void launch_g(dvg_context* ctx, int g, const SpgemmArgs& args) {
  switch (g) {
    case 4: launch_t<4, A_IDENTITY, FILL>(ctx, args); break;
    case 8: launch_t<8, A_IDENTITY, FILL>(ctx, args); break;
    case 16: launch_t<16, A_IDENTITY, FILL>(ctx, args); break;
    default: launch_t<32, A_IDENTITY, FILL>(ctx, args); break;
  }
}

}  // namespace

SpgemmPlan plan_spgemm(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b) {
  SpgemmPlan plan{};
  int g = int(ctx->opt_group_lanes);
  if (g != 4 && g != 8 && g != 16 && g != 32) {
    // B ranges visited per output row, estimated from the operands' densities:
    // (rows of B named per A row) x (ranges per B row).
    double a_rows_per_row = 1.0;
    if (!a_identity && a->nrows) a_rows_per_row = double(a->nnz) / double(a->nrows);
    double b_ranges_per_row = b->nrows ? double(b->nentries / 2) / double(b->nrows) : 0.0;
    double work = a_rows_per_row * b_ranges_per_row;
    g = work <= 6 ? 4 : work <= 20 ? 8 : work <= 64 ? 16 : 32;
  }
  plan.group_lanes = g;
  int ww = int(ctx->opt_window_words);
  plan.window_words = ww > 0 ? ww : 8 * g;
  return plan;
}

void launch_spgemm(dvg_context* ctx, const SpgemmPlan& plan, const dvg_matrix* a, bool a_identity,
                   const dvg_matrix* b, uint64_t* c_rowmap, uint32_t* c_entries, bool fill) {
  SpgemmArgs args{};
  args.a_rowmap = a_identity ? nullptr : a->rowmap;
  args.a_entries = a_identity ? nullptr : a->entries;
  args.b_rowmap = b->rowmap;
  args.b_entries = b->entries;
  args.c_rowmap = c_rowmap;
  args.c_entries = c_entries;
  args.ctl = ctx->d_ctl;
  args.nrows = a_identity ? b->nrows : a->nrows;
  args.ww = uint32_t(plan.window_words);
  if (args.nrows == 0) return;
  if (a_identity) {
    if (fill) launch_g<true, true>(ctx, plan.group_lanes, args);
    else launch_g<true, false>(ctx, plan.group_lanes, args);
  } else {
    if (fill) launch_g<false, true>(ctx, plan.group_lanes, args);
    else launch_g<false, false>(ctx, plan.group_lanes, args);
  }
}

}  // namespace dvg
