// dvg_spgemm_fused.cu -- single-pass, tile-staged range SpGEMM C = A*B.
//
// Same result as the reference's symbolic + numeric SpGEMM
// (include/diverg/range_sparse.hpp:1132-1442 in cartoonist/diverg, the
// TeamSequential / HBitVector pair, dispatched by range_spgemm :2215-2281):
// row r of C is the union of all ranges of B rows s..f for every range
// [s,f] of A's row r, emitted as sorted maximal runs.
//
// The kernel is persistent.  Each CTA takes chunks of consecutive C rows from
// an atomic ticket (so chunks start in order) and walks a chunk in sub-tiles
// of kSubRows rows.  For every sub-tile it
//  1. stages the sub-tile's A ranges and the slice of B rows they name (one
//     contiguous rowmap window and one contiguous entries window) in shared
//     memory;
//  2. builds, over the staged B rows, union bitmaps on the sub-tile's column
//     window: for blocks of `sb` rows the prefix union PRE[j] (block start ..
//     j), the suffix union SUF[j] (j .. block end) and the block union BU[b].
//     A range [s,f] of A then costs SUF[s] | BU[..] | PRE[f] -- a few word
//     ORs per column word -- instead of one visit per B row, which is what
//     dominates products of wide-range matrices (powers of A+I);
//  3. gathers every C row from those words with the boundary masks of the
//     reference's HBitVector gather (map01 / map10, hbitvector.hpp:568-597):
//     popc counts, a lane-group prefix sum places, ffs extracts;
//  4. appends the rows' runs, in row order, to a shared-memory staging area.
// At the end of the chunk a warp-parallel decoupled look-back over the chunk
// order yields the chunk's output offset (no separate symbolic pass or scan
// kernel); c_rowmap and the staged entries are then written with coalesced
// stores.  Sub-tiles whose A ranges, B slice or column window exceed the
// staging buffers take the direct path (a warp per row accumulates the B
// ranges in a shared bitvector window, in column chunks when the band is
// wider); rows that no longer fit the staging area are recomputed by the
// direct path straight into global memory after the look-back.  Look-back
// waits are bounded: on expiry the kernel records a timeout.
#include <algorithm>
#include <mutex>

#include "dvg_device.cuh"
#include "dvg_internal.h"

namespace dvg {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSubRows = 32;      // rows per staged sub-tile
constexpr int kChunkMax = 2048;   // rows per look-back chunk (upper bound)
constexpr int kAMax = 256;        // A ranges staged per sub-tile
constexpr int kSpanMax = 512;     // B rows staged per sub-tile
constexpr int kBMax = 1024;       // B ranges staged per sub-tile
constexpr int kBitWords = 7168;   // union bitmaps (PRE, SUF, BU) or direct windows
constexpr int kStageMax = 6144;   // output entries staged per chunk
constexpr int kDirectWW = kBitWords / (2 * kWarps);  // direct path window words per warp
constexpr unsigned long long kFlag = 1ull << 63;
constexpr uint32_t kSpinLimit = 1u << 22;

enum TileMode : int { kTiled = 0, kDirect = 1, kEmpty = 2 };

struct ChunkDesc {
  unsigned long long agg;       // kFlag | entries of the chunk
  unsigned long long agg_nnz;
  unsigned long long incl;      // kFlag | entries of chunks 0..t
  unsigned long long incl_nnz;
};

struct FusedArgs {
  const uint64_t* __restrict__ a_rowmap;
  const uint32_t* __restrict__ a_entries;
  const uint64_t* __restrict__ b_rowmap;
  const uint32_t* __restrict__ b_entries;
  uint64_t* __restrict__ c_rowmap;
  uint32_t* __restrict__ c_entries;
  uint64_t cap;
  ChunkDesc* desc;
  unsigned* ticket;
  DeviceControl* ctl;
  uint32_t nrows;
  uint32_t chunk_rows;  // multiple of kSubRows, <= kChunkMax
  uint32_t nchunks;
};

struct Smem {
  uint64_t arow[kSubRows + 1];
  uint64_t brow[kSpanMax + 1];
  uint2 a[kAMax];
  uint2 b[kBMax];
  uint32_t bits[kBitWords];
  uint32_t stage[kStageMax];
  uint32_t incl[kChunkMax];       // row entry counts, then their inclusive prefix
  uint32_t sub_off[kSubRows];     // stage offset of each row of the sub-tile
  unsigned long long red[kWarps];
  uint32_t redu[2 * kWarps];
  unsigned long long prefix;
  uint32_t chunk;
  uint32_t stage_used;   // staged entries of the chunk
  uint32_t staged_rows;  // leading rows of the chunk whose runs are staged
  uint32_t stage_open;   // 0 once a row did not fit
  uint32_t sub_fit;      // rows of the current sub-tile that were staged
};

// ---- small helpers -----------------------------------------------------------

// Bits of the 32-column word starting at column c0 covered by [rs, re].
__device__ __forceinline__ uint32_t word_mask(uint32_t rs, uint32_t re, uint64_t c0) {
  uint64_t lo = max(uint64_t(rs), c0), hi = min(uint64_t(re), c0 + 31);
  if (rs > re || lo > hi) return 0u;
  return (~0u << uint32_t(lo - c0)) & (~0u >> uint32_t(31 - (hi - c0)));
}

// Union of staged B row j on the word starting at c0.
__device__ __forceinline__ uint32_t row_mask(const Smem& S, uint64_t b_base, uint32_t j, uint64_t c0) {
  uint32_t k0 = uint32_t((S.brow[j] - b_base) >> 1), k1 = uint32_t((S.brow[j + 1] - b_base) >> 1);
  uint32_t m = 0;
  for (uint32_t k = k0; k < k1; ++k) m |= word_mask(S.b[k].x, S.b[k].y, c0);
  return m;
}

__device__ __forceinline__ unsigned runtime_group_mask(int g) {
  return g == 32 ? kFullMask : (((1u << g) - 1u) << (lane_id() & ~(g - 1)));
}

// Block-wide min and max of a uint32 pair (all threads receive both).
__device__ void block_minmax(Smem& S, uint32_t& mn, uint32_t& mx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(kFullMask, mn, o));
    mx = max(mx, __shfl_xor_sync(kFullMask, mx, o));
  }
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    S.redu[w] = mn;
    S.redu[kWarps + w] = mx;
  }
  __syncthreads();
  mn = S.redu[0];
  mx = S.redu[kWarps];
#pragma unroll
  for (int i = 1; i < kWarps; ++i) {
    mn = min(mn, S.redu[i]);
    mx = max(mx, S.redu[kWarps + i]);
  }
  __syncthreads();
}

__device__ unsigned long long block_sum(Smem& S, unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = v;
  __syncthreads();
  unsigned long long s = 0;
#pragma unroll
  for (int i = 0; i < kWarps; ++i) s += S.red[i];
  __syncthreads();
  return s;
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ---- tiled path ----------------------------------------------------------------

struct TileGeom {
  uint64_t a_base, b_base;
  uint32_t bs;    // first staged B row
  uint32_t span;  // staged B rows
  uint64_t base;  // first column of the window (32-aligned)
  uint32_t nwt;   // window words (the last one is always zero)
  uint32_t sb_shift;  // union block rows = 1 << sb_shift
};

// OR of the union bitmaps covering A row r (sub-tile local) on window word w.
__device__ __forceinline__ uint32_t tiled_acc(const Smem& S, const TileGeom& T, uint32_t r, uint32_t w) {
  const uint32_t* PRE = S.bits;
  const uint32_t* SUF = PRE + size_t(T.span) * T.nwt;
  const uint32_t* BU = SUF + size_t(T.span) * T.nwt;
  const uint64_t c0 = T.base + 32ull * w;
  const uint32_t k0 = uint32_t((S.arow[r] - T.a_base) >> 1), k1 = uint32_t((S.arow[r + 1] - T.a_base) >> 1);
  uint32_t acc = 0;
  for (uint32_t k = k0; k < k1; ++k) {
    const uint2 ar = S.a[k];
    if (ar.y < ar.x) continue;
    const uint32_t s = ar.x - T.bs, f = ar.y - T.bs;
    const uint32_t bS = s >> T.sb_shift, bF = f >> T.sb_shift;
    if (bS == bF) {
      for (uint32_t j = s; j <= f; ++j) acc |= row_mask(S, T.b_base, j, c0);
    } else {
      acc |= SUF[size_t(s) * T.nwt + w] | PRE[size_t(f) * T.nwt + w];
      for (uint32_t bb = bS + 1; bb < bF; ++bb) acc |= BU[size_t(bb) * T.nwt + w];
    }
  }
  return acc;
}

// Gathers the runs of one window chunk held by the group (word w per lane).
// Emits through `emit(row_local_index, value)`; returns the chunk's boundary
// count (group-uniform) and updates `carry` (msb of the chunk's last word).
template <class Emit>
__device__ __forceinline__ uint32_t gather_chunk(uint32_t x, bool valid, uint64_t c0, int g, int lg, unsigned gm,
                                                 uint32_t& carry, uint64_t count, uint32_t last_lane, Emit&& emit) {
  uint32_t prev = __shfl_up_sync(gm, x, 1, g);
  uint32_t c = lg == 0 ? carry : (prev >> 31);
  uint32_t sh = (x << 1) | c;
  uint32_t bnd = valid ? (((x ^ sh) & x) | (sh & ~x)) : 0u;
  uint32_t cnt = __popc(bnd);
  uint32_t incl = cnt;
  for (int o = 1; o < g; o <<= 1) {
    uint32_t u = __shfl_up_sync(gm, incl, o, g);
    if (lg >= o) incl += u;
  }
  uint64_t k = count + incl - cnt;
  while (bnd) {
    int bit = __ffs(bnd) - 1;
    bnd &= bnd - 1;
    emit(k, uint32_t(c0 + bit - (k & 1)));
    ++k;
  }
  uint32_t total = __shfl_sync(gm, incl, g - 1, g);
  carry = __shfl_sync(gm, x, int(last_lane), g) >> 31;
  return total;
}

// C row r of a tiled sub-tile, window chunk by window chunk.  Returns the
// entry count; adds the row's nnz into *nnz_acc (per lane) when given.
template <class Emit>
__device__ uint32_t tiled_row(const Smem& S, const TileGeom& T, uint32_t r, int g, int lg, unsigned gm,
                              unsigned long long* nnz_acc, Emit&& emit) {
  uint32_t carry = 0;
  uint64_t count = 0;
  for (uint32_t wb = 0; wb < T.nwt; wb += g) {
    const uint32_t w = wb + lg;
    const bool valid = w < T.nwt;
    const uint32_t x = valid ? tiled_acc(S, T, r, w) : 0u;
    if (nnz_acc) *nnz_acc += __popc(x);
    const uint32_t last = min(uint32_t(g - 1), T.nwt - 1 - wb);
    count += gather_chunk(x, valid, T.base + 32ull * w, g, lg, gm, carry, count, last, emit);
  }
  return uint32_t(count);
}

// ---- direct path: one C row by a warp, bitvector window in shared memory ----

template <class Emit>
__device__ uint64_t direct_row(const FusedArgs& p, bool a_identity, uint64_t row, uint32_t* bits, uint32_t* reach,
                               unsigned long long* nnz_acc, Emit&& emit) {
  const int lg = lane_id();
  uint64_t a0, a1;
  if (a_identity) {
    a0 = 0;
    a1 = 2;
  } else {
    a0 = p.a_rowmap[row];
    a1 = p.a_rowmap[row + 1];
  }
  auto slice = [&](uint64_t ai, uint64_t& b0, uint64_t& b1) {
    uint32_t s, f;
    if (a_identity) {
      s = f = uint32_t(row);
    } else {
      uint2 r = load_range(p.a_entries, ai >> 1);
      s = r.x;
      f = r.y;
    }
    if (f < s) {
      b0 = b1 = 0;
      return;
    }
    b0 = p.b_rowmap[s] >> 1;
    b1 = p.b_rowmap[uint64_t(f) + 1] >> 1;
  };
  uint32_t mn = 0xffffffffu, mx = 0;
  for (uint64_t ai = a0; ai < a1; ai += 2) {
    uint64_t b0, b1;
    slice(ai, b0, b1);
    for (uint64_t t = b0 + lg; t < b1; t += 32) {
      uint2 r = load_range(p.b_entries, t);
      if (r.y < r.x) continue;
      mn = min(mn, r.x);
      mx = max(mx, r.y);
    }
  }
  mn = group_min<32>(kFullMask, mn);
  mx = group_max<32>(kFullMask, mx);
  uint64_t count = 0;
  if (mn > mx) return 0;
  const uint64_t base = mn & ~31u;
  const uint64_t nw_total = ((uint64_t(mx) - base) >> 5) + 2;
  uint32_t carry = 0;
  for (uint64_t w0 = 0; w0 < nw_total; w0 += kDirectWW) {
    const uint32_t nwc = uint32_t(min(uint64_t(kDirectWW), nw_total - w0));
    const uint64_t cb = base + 32 * w0;
    const uint64_t ce = cb + 32ull * nwc - 1;
    for (uint32_t w = lg; w < nwc; w += 32) {
      bits[w] = 0;
      reach[w] = 0;
    }
    __syncwarp();
    for (uint64_t ai = a0; ai < a1; ai += 2) {
      uint64_t b0, b1;
      slice(ai, b0, b1);
      for (uint64_t t = b0 + lg; t < b1; t += 32) {
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
    __syncwarp();
    uint32_t run_reach = 0;
    for (uint32_t wb = 0; wb < nwc; wb += 32) {
      const uint32_t w = wb + lg;
      const bool valid = w < nwc;
      uint32_t x = 0, rr = 0;
      if (valid) {
        x = bits[w];
        rr = reach[w];
      }
      rr = group_incl_max<32>(kFullMask, rr, lg);
      rr = max(rr, run_reach);
      if (valid && rr > w) x = ~0u;
      run_reach = __shfl_sync(kFullMask, rr, 31);
      if (nnz_acc) *nnz_acc += __popc(x);
      const uint32_t last = min(31u, nwc - 1 - wb);
      count += gather_chunk(x, valid, cb + 32ull * w, 32, lg, kFullMask, carry, count, last, emit);
    }
    __syncwarp();
  }
  return count;
}

// ---- warp-parallel decoupled look-back over the chunk order -----------------
// Called by one full warp; every lane returns the chunk's exclusive prefix.
__device__ void lookback_warp(const FusedArgs& p, uint32_t t, unsigned long long cnt, unsigned long long nnz,
                              unsigned long long& prefix, unsigned long long& prefix_nnz) {
  const int lane = lane_id();
  ChunkDesc* d = p.desc;
  unsigned long long pre = 0, pre_nnz = 0;
  if (t != 0) {
    if (lane == 0) {
      d[t].agg_nnz = nnz;
      st_release(&d[t].agg, kFlag | cnt);
    }
    int64_t j = int64_t(t) - 1;
    uint32_t spins = 0;
    while (true) {
      const int64_t idx = j - lane;
      int st = 2;  // 2: inclusive prefix (or before chunk 0), 1: aggregate, 0: not yet
      unsigned long long v = 0, vn = 0;
      if (idx >= 0) {
        unsigned long long vi = ld_acquire(&d[idx].incl);
        if (vi & kFlag) {
          v = vi & ~kFlag;
          vn = *reinterpret_cast<volatile unsigned long long*>(&d[idx].incl_nnz);
        } else {
          unsigned long long va = ld_acquire(&d[idx].agg);
          if (va & kFlag) {
            st = 1;
            v = va & ~kFlag;
            vn = *reinterpret_cast<volatile unsigned long long*>(&d[idx].agg_nnz);
          } else {
            st = 0;
          }
        }
      }
      const unsigned incl_mask = __ballot_sync(kFullMask, st == 2);
      const unsigned wait_mask = __ballot_sync(kFullMask, st == 0);
      const int first = incl_mask ? __ffs(incl_mask) - 1 : 32;
      const unsigned before = first == 32 ? kFullMask : ((1u << first) - 1u);
      if (wait_mask & before) {
        if (++spins > kSpinLimit) {
          if (lane == 0) atomicOr(&p.ctl->timeout, 1ull);
          break;
        }
        __nanosleep(32);
        continue;
      }
      unsigned long long sv = lane <= first ? v : 0ull, sn = lane <= first ? vn : 0ull;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sv += __shfl_xor_sync(kFullMask, sv, o);
        sn += __shfl_xor_sync(kFullMask, sn, o);
      }
      pre += sv;
      pre_nnz += sn;
      if (first < 32) break;
      j -= 32;
    }
  }
  if (lane == 0) {
    d[t].incl_nnz = pre_nnz + nnz;
    st_release(&d[t].incl, kFlag | (pre + cnt));
  }
  prefix = pre;
  prefix_nnz = pre_nnz;
}

// Warp 0: stage offsets for the sub-tile's rows [r0, r0 + rows) whose counts
// are in S.incl; rows that fit are a prefix of the sub-tile.
__device__ void stage_rows(Smem& S, uint32_t r0, uint32_t rows) {
  const int lane = lane_id();
  const uint32_t v = lane < int(rows) ? S.incl[r0 + lane] : 0u;
  uint32_t incl = group_incl_sum<32>(kFullMask, v, lane);
  const uint32_t used = S.stage_used;
  const bool open = S.stage_open != 0;
  const bool fits = open && lane < int(rows) && uint64_t(used) + incl <= uint64_t(kStageMax);
  const unsigned fit_mask = __ballot_sync(kFullMask, fits);
  const uint32_t nfit = __popc(fit_mask);  // a prefix: incl grows with the lane
  if (lane < int(rows)) S.sub_off[lane] = used + incl - v;
  const uint32_t fit_total = nfit ? __shfl_sync(kFullMask, incl, int(nfit) - 1) : 0u;
  __syncwarp();
  if (lane == 0) {
    S.sub_fit = nfit;
    S.stage_used = used + fit_total;
    if (nfit < rows) S.stage_open = 0;
    S.staged_rows += nfit;
  }
}

template <bool A_ID>
__global__ void __launch_bounds__(kThreads) k_spgemm_fused(FusedArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  while (true) {
    if (tid == 0) {
      S.chunk = atomicAdd(p.ticket, 1u);
      S.stage_used = 0;
      S.staged_rows = 0;
      S.stage_open = 1;
    }
    __syncthreads();
    const uint32_t t = S.chunk;
    if (t >= p.nchunks) break;
    const uint32_t c0row = t * p.chunk_rows;
    const uint32_t crows = min(p.chunk_rows, p.nrows - c0row);
    unsigned long long nnz_acc = 0;
    bool any_direct = false;

    for (uint32_t r0 = 0; r0 < crows; r0 += kSubRows) {
      const uint32_t i0 = c0row + r0;
      const uint32_t rows = min(uint32_t(kSubRows), crows - r0);
      int mode = kTiled;
      TileGeom T{};

      // 1. A sub-tile
      uint64_t a_cnt;
      if (A_ID) {
        if (tid <= int(rows)) S.arow[tid] = 2ull * tid;
        if (tid < int(rows)) S.a[tid] = make_uint2(i0 + tid, i0 + tid);
        T.a_base = 0;
        a_cnt = rows;
        __syncthreads();
      } else {
        if (tid <= int(rows)) S.arow[tid] = p.a_rowmap[i0 + tid];
        __syncthreads();
        T.a_base = S.arow[0];
        a_cnt = (S.arow[rows] - T.a_base) >> 1;
        if (a_cnt > kAMax) {
          mode = kDirect;
        } else {
          for (uint32_t k = tid; k < a_cnt; k += kThreads) S.a[k] = load_range(p.a_entries, (T.a_base >> 1) + k);
        }
        __syncthreads();
      }

      // 2. B rows named by the sub-tile, and its column window
      if (mode == kTiled) {
        uint32_t mn = 0xffffffffu, mx = 0;
        for (uint32_t k = tid; k < a_cnt; k += kThreads) {
          uint2 r = S.a[k];
          if (r.y >= r.x) {
            mn = min(mn, r.x);
            mx = max(mx, r.y);
          }
        }
        block_minmax(S, mn, mx);
        if (mn > mx) {
          mode = kEmpty;
        } else {
          T.bs = mn;
          T.span = mx - mn + 1;
          if (T.span > kSpanMax) mode = kDirect;
        }
      }
      if (mode == kTiled) {
        for (uint32_t k = tid; k <= T.span; k += kThreads) S.brow[k] = p.b_rowmap[uint64_t(T.bs) + k];
        __syncthreads();
        T.b_base = S.brow[0];
        const uint64_t b_cnt = (S.brow[T.span] - T.b_base) >> 1;
        if (b_cnt > kBMax) {
          mode = kDirect;
        } else {
          for (uint32_t k = tid; k < b_cnt; k += kThreads) S.b[k] = load_range(p.b_entries, (T.b_base >> 1) + k);
        }
        __syncthreads();
        if (mode == kTiled) {
          uint32_t mn = 0xffffffffu, mx = 0;
          for (uint32_t k = tid; k < b_cnt; k += kThreads) {
            uint2 r = S.b[k];
            if (r.y >= r.x) {
              mn = min(mn, r.x);
              mx = max(mx, r.y);
            }
          }
          uint32_t wmax = 0;  // widest A range (rows)
          for (uint32_t k = tid; k < a_cnt; k += kThreads) {
            uint2 r = S.a[k];
            if (r.y >= r.x) wmax = max(wmax, r.y - r.x + 1);
          }
          block_minmax(S, mn, mx);
          uint32_t zero = 0;
          block_minmax(S, zero, wmax);
          if (mn > mx) {
            mode = kEmpty;
          } else {
            T.base = mn & ~31u;
            T.nwt = uint32_t(((uint64_t(mx) - T.base) >> 5) + 2);
            // union block: about a quarter of the widest A range, 2..64 rows
            uint32_t sb = 2;
            while (sb < 64 && sb * 4 <= wmax) sb <<= 1;
            T.sb_shift = __ffs(sb) - 1;
            const uint64_t nblk = (T.span + sb - 1) >> T.sb_shift;
            if ((2ull * T.span + nblk) * T.nwt > kBitWords) mode = kDirect;
          }
        }
      }

      if (mode == kTiled) {
        // 3. union bitmaps: R_j into PRE, then SUF (from R) and PRE (in place)
        uint32_t* PRE = S.bits;
        uint32_t* SUF = PRE + size_t(T.span) * T.nwt;
        uint32_t* BU = SUF + size_t(T.span) * T.nwt;
        const uint32_t items = T.span * T.nwt;
        for (uint32_t it = tid; it < items; it += kThreads) {
          const uint32_t j = it / T.nwt, w = it - j * T.nwt;
          PRE[it] = row_mask(S, T.b_base, j, T.base + 32ull * w);
        }
        __syncthreads();
        const uint32_t sb = 1u << T.sb_shift;
        const uint32_t nblk = (T.span + sb - 1) >> T.sb_shift;
        for (uint32_t it = tid; it < nblk * T.nwt; it += kThreads) {
          const uint32_t bb = it / T.nwt, w = it - bb * T.nwt;
          const uint32_t j0 = bb << T.sb_shift, j1 = min(T.span, j0 + sb);
          uint32_t acc = 0;
          for (uint32_t j = j1; j-- > j0;) {
            acc |= PRE[size_t(j) * T.nwt + w];
            SUF[size_t(j) * T.nwt + w] = acc;
          }
          acc = 0;
          for (uint32_t j = j0; j < j1; ++j) {
            acc |= PRE[size_t(j) * T.nwt + w];
            PRE[size_t(j) * T.nwt + w] = acc;
          }
          BU[size_t(bb) * T.nwt + w] = acc;
        }
        __syncthreads();

        // 4. rows: groups of g lanes, one window word per lane and chunk.
        // A group holds at most 4 rows (g >= 4 lanes -> >= 8 groups).
        const int g = T.nwt <= 4 ? 4 : T.nwt <= 8 ? 8 : T.nwt <= 16 ? 16 : 32;
        const int lg = tid & (g - 1);
        const unsigned gm = runtime_group_mask(g);
        const uint32_t gid = tid / g, ngroups = kThreads / g;
        const bool one_chunk = T.nwt <= uint32_t(g);
        uint32_t xs[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t r = gid + q * ngroups;
          xs[q] = 0;
          if (r < rows) {
            uint32_t cnt;
            if (one_chunk) {
              const bool valid = uint32_t(lg) < T.nwt;
              const uint32_t x = valid ? tiled_acc(S, T, r, lg) : 0u;
              xs[q] = x;
              nnz_acc += __popc(x);
              uint32_t carry = 0;
              cnt = gather_chunk(x, valid, 0, g, lg, gm, carry, 0, T.nwt - 1, [](uint64_t, uint32_t) {});
            } else {
              cnt = tiled_row(S, T, r, g, lg, gm, &nnz_acc, [](uint64_t, uint32_t) {});
            }
            if (lg == 0) S.incl[r0 + r] = cnt;
          }
        }
        __syncthreads();
        if (warp == 0) stage_rows(S, r0, rows);
        __syncthreads();
        const uint32_t fit = S.sub_fit;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t r = gid + q * ngroups;
          if (r < fit) {
            uint32_t* st = S.stage + S.sub_off[r];
            if (one_chunk) {
              const bool valid = uint32_t(lg) < T.nwt;
              uint32_t carry = 0;
              gather_chunk(xs[q], valid, T.base + 32ull * lg, g, lg, gm, carry, 0, T.nwt - 1,
                           [&](uint64_t k, uint32_t v) { st[k] = v; });
            } else {
              tiled_row(S, T, r, g, lg, gm, nullptr, [&](uint64_t k, uint32_t v) { st[k] = v; });
            }
          }
        }
        __syncthreads();
      } else if (mode == kDirect) {
        any_direct = true;
        uint32_t* bits = S.bits + size_t(warp) * 2 * kDirectWW;
        uint32_t* reach = bits + kDirectWW;
        for (uint32_t r = warp; r < rows; r += kWarps) {
          uint64_t c = direct_row(p, A_ID, uint64_t(i0) + r, bits, reach, &nnz_acc, [](uint64_t, uint32_t) {});
          if (lane == 0) S.incl[r0 + r] = uint32_t(min(c, uint64_t(0xffffffffu)));
        }
        __syncthreads();
        if (warp == 0) stage_rows(S, r0, rows);
        __syncthreads();
        const uint32_t fit = S.sub_fit;
        for (uint32_t r = warp; r < fit; r += kWarps) {
          uint32_t* st = S.stage + S.sub_off[r];
          direct_row(p, A_ID, uint64_t(i0) + r, bits, reach, nullptr, [&](uint64_t k, uint32_t v) { st[k] = v; });
        }
        __syncthreads();
      } else {
        if (tid < int(rows)) S.incl[r0 + tid] = 0;
        __syncthreads();
        if (warp == 0) stage_rows(S, r0, rows);
        __syncthreads();
      }
    }

    // 5. chunk prefix over the row counts (8 consecutive rows per thread)
    {
      uint32_t loc[8];
      uint64_t s = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t r = tid * 8 + k;
        s += r < crows ? S.incl[r] : 0u;
        loc[k] = uint32_t(s);
      }
      // block exclusive scan of the per-thread sums
      uint64_t inc = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint64_t u = __shfl_up_sync(kFullMask, inc, o);
        if (lane >= o) inc += u;
      }
      if (lane == 31) S.red[warp] = inc;
      __syncthreads();
      uint64_t wpre = 0;
      for (int i = 0; i < warp; ++i) wpre += S.red[i];
      const uint64_t excl = wpre + inc - s;
      if (excl + s > 0xffffffffull) atomicOr(&p.ctl->status, 16ull);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t r = tid * 8 + k;
        if (r < crows) S.incl[r] = uint32_t(excl) + loc[k];
      }
      __syncthreads();
    }
    const unsigned long long chunk_nnz = block_sum(S, nnz_acc);
    if (warp == 0) {
      const unsigned long long chunk_cnt = S.incl[crows - 1];
      unsigned long long pre, pre_nnz;
      lookback_warp(p, t, chunk_cnt, chunk_nnz, pre, pre_nnz);
      if (lane == 0) {
        S.prefix = pre;
        if (t == p.nchunks - 1) {
          p.ctl->total = pre + chunk_cnt;
          p.ctl->nnz = pre_nnz + chunk_nnz;
          if (pre + chunk_cnt > p.cap) p.ctl->overflow = pre + chunk_cnt;
        }
      }
    }
    if (tid == 0 && any_direct) atomicAdd(&p.ctl->tiles_direct, 1ull);
    __syncthreads();
    const unsigned long long prefix = S.prefix;

    // 6. rowmap, staged entries, and the rows that did not fit the stage
    for (uint32_t r = tid; r < crows; r += kThreads) p.c_rowmap[uint64_t(c0row) + r + 1] = prefix + S.incl[r];
    if (t == 0 && tid == 0) p.c_rowmap[0] = 0;
    const uint32_t staged = S.stage_used;
    if (prefix + staged <= p.cap) {
      for (uint32_t k = tid; k < staged; k += kThreads) p.c_entries[prefix + k] = S.stage[k];
    } else if (tid == 0) {
      atomicOr(&p.ctl->overflow, 1ull);
    }
    const uint32_t srows = S.staged_rows;
    if (srows < crows) {
      uint32_t* bits = S.bits + size_t(warp) * 2 * kDirectWW;
      uint32_t* reach = bits + kDirectWW;
      for (uint32_t r = srows + warp; r < crows; r += kWarps) {
        const unsigned long long dst = prefix + (r ? S.incl[r - 1] : 0u);
        const uint32_t n = S.incl[r] - (r ? S.incl[r - 1] : 0u);
        if (n == 0) continue;
        if (dst + n > p.cap) {
          if (lane == 0) atomicOr(&p.ctl->overflow, 1ull);
          continue;
        }
        uint32_t* out = p.c_entries + dst;
        bool bad = false;
        uint64_t c = direct_row(p, A_ID, uint64_t(c0row) + r, bits, reach, nullptr, [&](uint64_t k, uint32_t v) {
          if (k < n) out[k] = v;
          else bad = true;
        });
        if (bad || c != n) atomicOr(&p.ctl->status, 8ull);
      }
    }
    __syncthreads();
  }
}

}  // namespace

void launch_spgemm_fused(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b,
                         uint64_t* c_rowmap, uint32_t* c_entries, uint64_t cap) {
  const uint32_t n = a_identity ? b->nrows : a->nrows;
  if (n == 0) return;
  auto kern = a_identity ? k_spgemm_fused<true> : k_spgemm_fused<false>;
  const int smem = int(sizeof(Smem));
  DVG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int per_sm = 0;
  DVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
  if (per_sm < 1) throw Error(DVG_ERR_DEVICE, "fused spgemm: shared memory layout does not fit");
  const uint64_t resident = uint64_t(per_sm) * ctx->num_sms;
  // chunk rows: as large as possible (fewer look-back steps) while keeping
  // about four chunks per resident CTA
  uint32_t chunk_rows = kChunkMax;
  while (chunk_rows > kSubRows && (uint64_t(n) + chunk_rows - 1) / chunk_rows < 4 * resident) chunk_rows >>= 1;
  if (ctx->opt_chunk_rows > 0) chunk_rows = uint32_t(ctx->opt_chunk_rows);
  const uint32_t nchunks = uint32_t((uint64_t(n) + chunk_rows - 1) / chunk_rows);
  const size_t desc_bytes = size_t(nchunks) * sizeof(ChunkDesc);
  if (desc_bytes > ctx->tile_desc_cap) {
    if (ctx->d_tile_desc) dfree(ctx, ctx->d_tile_desc);
    ctx->d_tile_desc = nullptr;
    ctx->tile_desc_cap = 0;
    size_t want = std::max(desc_bytes, size_t(1) << 20);
    ctx->d_tile_desc = dalloc(ctx, want);
    ctx->tile_desc_cap = want;
  }
  if (!ctx->d_ticket) ctx->d_ticket = static_cast<unsigned*>(dalloc(ctx, 256));
  DVG_CUDA(cudaMemsetAsync(ctx->d_tile_desc, 0, desc_bytes, ctx->stream));
  DVG_CUDA(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(unsigned), ctx->stream));
  FusedArgs p{};
  p.a_rowmap = a_identity ? nullptr : a->rowmap;
  p.a_entries = a_identity ? nullptr : a->entries;
  p.b_rowmap = b->rowmap;
  p.b_entries = b->entries;
  p.c_rowmap = c_rowmap;
  p.c_entries = c_entries;
  p.cap = cap;
  p.desc = static_cast<ChunkDesc*>(ctx->d_tile_desc);
  p.ticket = ctx->d_ticket;
  p.ctl = ctx->d_ctl;
  p.nrows = n;
  p.chunk_rows = chunk_rows;
  p.nchunks = nchunks;
  const unsigned grid = unsigned(std::min<uint64_t>(nchunks, resident));
  kern<<<grid, kThreads, smem, ctx->stream>>>(p);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

}  // namespace dvg

// ---- the no-allocation entry point -------------------------------------------
//
// dvg_range_spgemm_noalloc runs the fused kernel above for callers that may
// not allocate device memory.  Its chunk descriptors, tile ticket and control
// block live in one file-scope device array, sized for kNoAllocMaxChunks
// chunks of at most kChunkMax rows, i.e. products with up to
// kNoAllocMaxChunks * kChunkMax = 67,108,864 output rows.  Every GPU that
// loads the library holds this array (about 1 MiB) until the process exits.
// All calls share it and it keeps the last call's contents, so each call
// clears the part it uses before its kernels run; calls whose work overlaps
// on the GPU (from several streams or threads) race on it and must be
// serialised by the caller.
namespace dvg {
namespace {

constexpr uint32_t kNoAllocMaxChunks = 32768;
constexpr size_t kNoAllocDescBytes = size_t(kNoAllocMaxChunks) * sizeof(ChunkDesc);
constexpr size_t kNoAllocCtlOffset = kNoAllocDescBytes;                 // DeviceControl
constexpr size_t kNoAllocTicketOffset = kNoAllocCtlOffset + 256;       // tile ticket
constexpr size_t kNoAllocBytes = kNoAllocTicketOffset + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device ordinal.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device (with that device current) and cached here.
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Sets bit 1 of *bad when a range-CRS matrix violates the memory-safety
// preconditions of the fused kernel (rowmap[0] = 0, non-decreasing, even row
// lengths, rowmap[n] = nentries, columns < ncols).
__global__ void k_noalloc_validate(const uint64_t* __restrict__ rowmap, uint32_t nrows,
                                   const uint32_t* __restrict__ entries, uint64_t nentries, uint32_t ncols,
                                   unsigned long long* bad) {
  unsigned long long b = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  for (uint64_t i = tid; i < nrows; i += stride) {
    const uint64_t lo = rowmap[i], hi = rowmap[i + 1];
    if (hi < lo || ((hi - lo) & 1)) b = 1;
  }
  if (tid == 0 && (rowmap[0] != 0 || rowmap[nrows] != nentries)) b = 1;
  for (uint64_t i = tid; i < nentries; i += stride)
    if (entries[i] >= ncols) b = 1;
  if (b) atomicOr(bad, 1ull);
}

dvg_status dvg_noalloc_fail(dvg_status s, const std::string& msg) {
  record_error(msg);
  return s;
}

}  // namespace
}  // namespace dvg

extern "C" dvg_status dvg_range_spgemm_noalloc(uint32_t a_nrows, uint32_t a_ncols, const uint64_t* d_a_rowmap,
                                               const uint32_t* d_a_entries, uint64_t a_nentries, uint32_t b_nrows,
                                               uint32_t b_ncols, const uint64_t* d_b_rowmap,
                                               const uint32_t* d_b_entries, uint64_t b_nentries,
                                               uint64_t* d_c_rowmap, uint32_t* d_c_entries, uint64_t c_capacity,
                                               uint64_t* c_nentries, uint64_t* c_nnz, void* cuda_stream) {
  using namespace dvg;
  // Argument checks come first and touch no pointer, so an oversized request
  // is rejected before any device work.
  if (!c_nentries || !c_nnz) return dvg_noalloc_fail(DVG_ERR_INVALID_ARG, "null output pointer");
  *c_nentries = 0;
  *c_nnz = 0;
  if (uint64_t(a_nrows) > uint64_t(kNoAllocMaxChunks) * kChunkMax)
    return dvg_noalloc_fail(DVG_ERR_INVALID_ARG,
                            "dvg_range_spgemm_noalloc: more than 67108864 output rows (its scratch limit); "
                            "use dvg_range_spgemm");
  if (a_ncols != b_nrows) return dvg_noalloc_fail(DVG_ERR_INVALID_ARG, "a.numCols() != b.numRows()");
  if (a_ncols > 0xFFFFFFFEu || b_ncols > 0xFFFFFFFEu)
    return dvg_noalloc_fail(DVG_ERR_INVALID_ARG, "ncols must be below 2^32 - 1");
  if (!d_a_rowmap || !d_b_rowmap || !d_c_rowmap || (a_nentries && !d_a_entries) || (b_nentries && !d_b_entries) ||
      (c_capacity && !d_c_entries))
    return dvg_noalloc_fail(DVG_ERR_INVALID_ARG, "null device pointer");
  if ((reinterpret_cast<uintptr_t>(d_a_entries) | reinterpret_cast<uintptr_t>(d_b_entries)) & 7)
    return dvg_noalloc_fail(DVG_ERR_INVALID_ARG, "entries must be 8-byte aligned");
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  try {
    int dev = 0;
    DVG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) throw Error(DVG_ERR_DEVICE, "device ordinal out of range");
    unsigned char* scratch = nullptr;
    {
      std::lock_guard<std::mutex> lk(g_noalloc_mu);
      if (!g_noalloc_ptr[dev]) {
        void* ptr = nullptr;
        DVG_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_noalloc_ptr[dev] = ptr;
      }
      scratch = static_cast<unsigned char*>(g_noalloc_ptr[dev]);
    }
    ChunkDesc* desc = reinterpret_cast<ChunkDesc*>(scratch);
    DeviceControl* ctl = reinterpret_cast<DeviceControl*>(scratch + kNoAllocCtlOffset);
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kNoAllocTicketOffset);
    DeviceControl h{};
    if (a_nrows == 0) {
      DVG_CUDA(cudaMemsetAsync(d_c_rowmap, 0, sizeof(uint64_t), stream));
      DVG_CUDA(cudaStreamSynchronize(stream));
      return DVG_OK;
    }
    // 1. inputs must be well formed before the product may index through them
    int nsm = 0;
    DVG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DVG_CUDA(cudaMemsetAsync(ctl, 0, sizeof(DeviceControl), stream));
    const unsigned vgrid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(
        (std::max<uint64_t>(std::max<uint64_t>(a_nrows, a_nentries), std::max<uint64_t>(b_nrows, b_nentries)) +
         255) / 256, uint64_t(nsm) * 8)));
    k_noalloc_validate<<<vgrid, 256, 0, stream>>>(d_a_rowmap, a_nrows, d_a_entries, a_nentries, a_ncols,
                                                  &ctl->invalid);
    k_noalloc_validate<<<vgrid, 256, 0, stream>>>(d_b_rowmap, b_nrows, d_b_entries, b_nentries, b_ncols,
                                                  &ctl->invalid);
    DVG_CUDA(cudaGetLastError());
    DVG_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(DeviceControl), cudaMemcpyDeviceToHost, stream));
    DVG_CUDA(cudaStreamSynchronize(stream));
    if (h.invalid) throw Error(DVG_ERR_INVALID_ARG, "malformed range-CRS input matrix");
    // 2. the fused product with this file's scratch
    auto kern = k_spgemm_fused<false>;
    const int smem = int(sizeof(Smem));
    DVG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    DVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
    if (per_sm < 1) throw Error(DVG_ERR_DEVICE, "fused spgemm: shared memory layout does not fit");
    const uint64_t resident = uint64_t(per_sm) * nsm;
    uint32_t chunk_rows = kChunkMax;
    while (chunk_rows > kSubRows && (uint64_t(a_nrows) + chunk_rows - 1) / chunk_rows < 4 * resident)
      chunk_rows >>= 1;
    const uint32_t nchunks = uint32_t((uint64_t(a_nrows) + chunk_rows - 1) / chunk_rows);
    if (nchunks > kNoAllocMaxChunks) throw Error(DVG_ERR_INVALID_ARG, "too many output chunks for the scratch");
    DVG_CUDA(cudaMemsetAsync(desc, 0, size_t(nchunks) * sizeof(ChunkDesc), stream));
    DVG_CUDA(cudaMemsetAsync(ctl, 0, sizeof(DeviceControl), stream));
    DVG_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), stream));
    FusedArgs p{};
    p.a_rowmap = d_a_rowmap;
    p.a_entries = d_a_entries;
    p.b_rowmap = d_b_rowmap;
    p.b_entries = d_b_entries;
    p.c_rowmap = d_c_rowmap;
    p.c_entries = d_c_entries;
    p.cap = c_capacity;
    p.desc = desc;
    p.ticket = ticket;
    p.ctl = ctl;
    p.nrows = a_nrows;
    p.chunk_rows = chunk_rows;
    p.nchunks = nchunks;
    const unsigned grid = unsigned(std::min<uint64_t>(nchunks, resident));
    kern<<<grid, kThreads, smem, stream>>>(p);
    DVG_CUDA(cudaGetLastError());
    DVG_CUDA(cudaMemcpyAsync(&h, ctl, sizeof(DeviceControl), cudaMemcpyDeviceToHost, stream));
    DVG_CUDA(cudaStreamSynchronize(stream));
    *c_nentries = h.total;
    *c_nnz = h.nnz;
    if (h.timeout) throw Error(DVG_ERR_TIMEOUT, "range_spgemm: chunk look-back wait expired");
    if (h.status) throw Error(DVG_ERR_DEVICE, "internal consistency check failed on the device");
    if (h.overflow)
      throw Error(DVG_ERR_OVERFLOW, "c_capacity is smaller than the product's " + std::to_string(h.total) +
                                        " entries (c_rowmap is complete; call again with a larger buffer)");
  } catch (const Error& e) {
    return dvg_noalloc_fail(e.status, e.what());
  }
  return DVG_OK;
}
