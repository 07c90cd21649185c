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

#include "dvg_spgemm_common.cuh"

namespace dvg {
namespace {

enum TileMode : uint32_t { kTiled = 0, kDirect = 1, kEmpty = 2 };

// One staged B window: rows [bs, bf] and their ranges.
struct BBuf {
  uint64_t brow[kSpanMax + 1];
  uint2 b[kBMax];
};

// A sub-tile's plan, made when its chunk starts.
struct SubDesc {
  uint32_t bs, bf;    // B rows named by the sub-tile's A ranges
  uint32_t wmax;      // widest A range (rows)
  uint32_t mode;      // TileMode
  uint64_t b0, b1;    // B entries of rows bs..bf
};

struct TileBufs {
  BBuf bb[2];                     // double-buffered B windows
  uint32_t bits[kBitWords];
  uint32_t stage[kStageMax];
};

struct Smem {
  uint32_t crow[kChunkMax + 1];   // chunk A row map, relative to its first entry
  uint2 achunk[kAChunk];          // chunk A ranges
  SubDesc sub[kSubMax];
  union {
    TileBufs t;
  } u;
  uint32_t incl[kChunkMax];       // row entry counts, then their inclusive prefix
  uint32_t sub_off[kSubRows];     // stage offset of each row of the sub-tile
  unsigned long long red[kWarps];
  uint32_t redu[2][3 * kWarps];  // double-buffered block reductions
  unsigned long long prefix;
  uint32_t chunk;
  uint32_t stage_used;   // staged entries of the chunk
  uint32_t staged_rows;  // leading rows of the chunk whose runs are staged
  uint32_t stage_open;   // 0 once a row did not fit
  uint32_t sub_fit;      // rows of the current sub-tile that were staged
  uint32_t a_staged;     // the chunk's A ranges are in achunk
};

// two CTAs per SM: 2 x (layout + 1 KB reserved) within the SM's 228 KB
static_assert(2 * (sizeof(Smem) + 1024) <= 228 * 1024, "shared layout exceeds two CTAs per SM");

// ---- small helpers -----------------------------------------------------------

// Bits of the 32-column word starting at column c0 covered by [rs, re].
__device__ __forceinline__ uint32_t word_mask(uint32_t rs, uint32_t re, uint64_t c0) {
  uint64_t lo = max(uint64_t(rs), c0), hi = min(uint64_t(re), c0 + 31);
  if (rs > re || lo > hi) return 0u;
  return (~0u << uint32_t(lo - c0)) & (~0u >> uint32_t(31 - (hi - c0)));
}

// Union of staged B row j (window-relative) on the word starting at c0.
__device__ __forceinline__ uint32_t row_mask(const BBuf& B, uint64_t b_base, uint32_t j, uint64_t c0) {
  uint32_t k0 = uint32_t((B.brow[j] - b_base) >> 1), k1 = uint32_t((B.brow[j + 1] - b_base) >> 1);
  uint32_t m = 0;
  for (uint32_t k = k0; k < k1; ++k) m |= word_mask(B.b[k].x, B.b[k].y, c0);
  return m;
}

// (cp_async8 and cp_async_commit: dvg_spgemm_common.cuh)
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ unsigned runtime_group_mask(int g) {
  return g == 32 ? kFullMask : (((1u << g) - 1u) << (lane_id() & ~(g - 1)));
}

// Block-wide (min a, max b, max c) with one barrier: warp partials go to one
// of two buffers, alternating, so the next reduction cannot overwrite a
// buffer that a slow warp is still reading.  All threads receive the result.
__device__ void block_min_max_max(Smem& S, uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& phase) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = min(a, __shfl_xor_sync(kFullMask, a, o));
    b = max(b, __shfl_xor_sync(kFullMask, b, o));
    c = max(c, __shfl_xor_sync(kFullMask, c, o));
  }
  uint32_t* buf = S.redu[phase & 1];
  phase ^= 1;
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    buf[w] = a;
    buf[kWarps + w] = b;
    buf[2 * kWarps + w] = c;
  }
  __syncthreads();
  a = buf[0];
  b = buf[kWarps];
  c = buf[2 * kWarps];
#pragma unroll
  for (int i = 1; i < kWarps; ++i) {
    a = min(a, buf[i]);
    b = max(b, buf[kWarps + i]);
    c = max(c, buf[2 * kWarps + i]);
  }
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

// ---- tiled path ----------------------------------------------------------------

struct TileGeom {
  const BBuf* B;      // the staged B window
  uint32_t r0;        // first chunk row of the sub-tile
  uint64_t b_base;
  uint32_t bs;        // first staged B row
  uint32_t span;      // staged B rows
  uint64_t base;      // first column of the window (32-aligned)
  uint32_t nwt;       // window words (the last one is always zero)
  uint32_t sb_shift;  // union block rows = 1 << sb_shift
  uint32_t pitch;     // words between two window words of PRE / SUF (odd)
  uint32_t bpitch;    // the same for BU (odd)
};

// Union bitmaps are stored word-major -- PRE[w * pitch + j] -- with an odd
// pitch, so lanes reading consecutive words of one row, or consecutive rows
// of one word, hit distinct banks.

// OR of the union bitmaps covering A row r (sub-tile local) on window word w.
__device__ __forceinline__ uint32_t tiled_acc(const Smem& S, const TileGeom& T, uint32_t r, uint32_t w) {
  const uint32_t* PRE = S.u.t.bits + size_t(w) * T.pitch;
  const uint32_t* SUF = S.u.t.bits + size_t(T.nwt) * T.pitch + size_t(w) * T.pitch;
  const uint32_t* BU = S.u.t.bits + 2 * size_t(T.nwt) * T.pitch + size_t(w) * T.bpitch;
  const uint64_t c0 = T.base + 32ull * w;
  const uint32_t k0 = S.crow[T.r0 + r] >> 1, k1 = S.crow[T.r0 + r + 1] >> 1;
  uint32_t acc = 0;
  for (uint32_t k = k0; k < k1; ++k) {
    const uint2 ar = S.achunk[k];
    if (ar.y < ar.x) continue;
    const uint32_t s = ar.x - T.bs, f = ar.y - T.bs;
    const uint32_t bS = s >> T.sb_shift, bF = f >> T.sb_shift;
    if (bS == bF) {
      for (uint32_t j = s; j <= f; ++j) acc |= row_mask(*T.B, T.b_base, j, c0);
    } else {
      acc |= SUF[s] | PRE[f];
      for (uint32_t bb = bS + 1; bb < bF; ++bb) acc |= BU[bb];
    }
  }
  return acc;
}

// Gathers the runs of one window chunk held by the group (word w per lane).
// Emits through `emit(row_local_index, value)`; returns the chunk's boundary
// count (group-uniform) and updates `carry` (msb of the chunk's last word).
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

// Warp 0: stage offsets for the sub-tile's rows [r0, r0 + rows) (rows <= 64,
// two consecutive rows per lane) whose counts are in S.incl; rows that fit
// the staging area are a prefix of the sub-tile.
__device__ void stage_rows(Smem& S, uint32_t r0, uint32_t rows) {
  const int lane = lane_id();
  const uint32_t ra = 2 * lane, rb = ra + 1;
  const uint64_t va = ra < rows ? S.incl[r0 + ra] : 0u, vb = rb < rows ? S.incl[r0 + rb] : 0u;
  const uint64_t pair = va + vb;
  uint64_t inc = pair;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(kFullMask, inc, o);
    if (lane >= o) inc += u;
  }
  const uint64_t ea = inc - pair, eb = ea + va;
  const uint64_t used = S.stage_used;
  const bool open = S.stage_open != 0;
  const bool fa = open && ra < rows && used + ea + va <= uint64_t(kStageMax);
  const bool fb = open && rb < rows && used + eb + vb <= uint64_t(kStageMax);
  // the fitting rows are a prefix: their inclusive sums grow with the row
  const uint32_t nfit = __popc(__ballot_sync(kFullMask, fa)) + __popc(__ballot_sync(kFullMask, fb));
  if (ra < rows) S.sub_off[ra] = uint32_t(used + ea);
  if (rb < rows) S.sub_off[rb] = uint32_t(used + eb);
  uint64_t fit_end = fb ? eb + vb : (fa ? ea + va : 0u);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t u = __shfl_xor_sync(kFullMask, fit_end, o);
    fit_end = u > fit_end ? u : fit_end;
  }
  __syncwarp();
  if (lane == 0) {
    S.sub_fit = nfit;
    S.stage_used = uint32_t(used + fit_end);
    if (nfit < rows) S.stage_open = 0;
    S.staged_rows += nfit;
  }
}

// Issues the asynchronous copies of sub-tile q's B window into its buffer
// and commits them as one group (an empty group when q stages nothing).
__device__ __forceinline__ void prefetch_window(Smem& S, const FusedArgs& p, uint32_t q, uint32_t nsub) {
  if (q < nsub && S.sub[q].mode == kTiled) {
    const SubDesc d = S.sub[q];
    BBuf& B = S.u.t.bb[q & 1];
    const uint32_t span = d.bf - d.bs + 1;
    for (uint32_t k = threadIdx.x; k <= span; k += kThreads) cp_async8(&B.brow[k], p.b_rowmap + d.bs + k);
    const uint64_t r0 = d.b0 >> 1;
    const uint32_t nr = uint32_t((d.b1 - d.b0) >> 1);
    for (uint32_t k = threadIdx.x; k < nr; k += kThreads)
      cp_async8(&B.b[k], reinterpret_cast<const uint2*>(p.b_entries) + r0 + k);
  }
  cp_async_commit();
}

template <bool A_ID>
__global__ void __launch_bounds__(kThreads, 2) k_spgemm_fused(FusedArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t phase = 0;  // reduction buffer parity (uniform over the CTA)

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
    const uint32_t nsub = (crows + kSubRows - 1) / kSubRows;
    unsigned long long nnz_acc = 0;
    bool any_direct = false;

    // ---- chunk plan: A row map and ranges once, then every sub-tile's B
    // rows and B entry window, so sub-tile staging needs no further lookups
    if (A_ID) {
      for (uint32_t k = tid; k <= crows; k += kThreads) S.crow[k] = 2 * k;
      if (tid == 0) S.a_staged = 1;
    } else {
      const uint64_t abase = p.a_rowmap[c0row];
      const uint64_t aend = p.a_rowmap[c0row + crows];
      const bool fits = ((aend - abase) >> 1) <= kAChunk;
      if (fits)
        for (uint32_t k = tid; k <= crows; k += kThreads) S.crow[k] = uint32_t(p.a_rowmap[c0row + k] - abase);
      if (tid == 0) S.a_staged = fits ? 1u : 0u;
    }
    __syncthreads();
    const bool a_staged = S.a_staged != 0;
    if (a_staged) {
      const uint64_t abase = A_ID ? 0 : p.a_rowmap[c0row];
      for (uint32_t q = warp; q < nsub; q += kWarps) {
        const uint32_t rq0 = q * kSubRows, rq1 = min(crows, rq0 + kSubRows);
        const uint32_t k0 = S.crow[rq0] >> 1, k1 = S.crow[rq1] >> 1;
        uint32_t mn = 0xffffffffu, mx = 0, wmax = 0;
        for (uint32_t k = k0 + lane; k < k1; k += 32) {
          uint2 r;
          if (A_ID) {
            r = make_uint2(c0row + k, c0row + k);
          } else {
            r = load_range(p.a_entries, (abase >> 1) + k);
          }
          S.achunk[k] = r;
          if (r.y >= r.x) {
            mn = min(mn, r.x);
            mx = max(mx, r.y);
            wmax = max(wmax, r.y - r.x + 1);
          }
        }
        mn = group_min<32>(kFullMask, mn);
        mx = group_max<32>(kFullMask, mx);
        wmax = group_max<32>(kFullMask, wmax);
        if (lane == 0) {
          SubDesc d{};
          d.bs = mn;
          d.bf = mx;
          d.wmax = wmax;
          d.mode = mn > mx ? kEmpty : (mx - mn + 1 > uint32_t(kSpanMax) ? kDirect : kTiled);
          S.sub[q] = d;
        }
      }
    } else {
      for (uint32_t q = tid; q < nsub; q += kThreads) S.sub[q].mode = kDirect;
    }
    __syncthreads();
    for (uint32_t q = tid; q < nsub; q += kThreads) {
      SubDesc& d = S.sub[q];
      if (d.mode == kTiled) {
        d.b0 = p.b_rowmap[d.bs];
        d.b1 = p.b_rowmap[uint64_t(d.bf) + 1];
        if (d.b1 < d.b0 || ((d.b1 - d.b0) >> 1) > uint64_t(kBMax)) d.mode = kDirect;
      }
    }
    __syncthreads();
    prefetch_window(S, p, 0, nsub);

    for (uint32_t q = 0; q < nsub; ++q) {
      const uint32_t r0 = q * kSubRows;
      const uint32_t i0 = c0row + r0;
      const uint32_t rows = min(uint32_t(kSubRows), crows - r0);
      prefetch_window(S, p, q + 1, nsub);  // overlaps this sub-tile's work
      cp_async_wait_prev();                 // this sub-tile's window has landed
      __syncthreads();
      const SubDesc d = S.sub[q];
      uint32_t mode = d.mode;
      TileGeom T{};

      if (mode == kTiled) {
        // the sub-tile's column window over its staged B ranges
        const BBuf& B = S.u.t.bb[q & 1];
        T.B = &B;
        T.r0 = r0;
        T.bs = d.bs;
        T.span = d.bf - d.bs + 1;
        T.b_base = d.b0;
        const uint32_t nb = uint32_t((d.b1 - d.b0) >> 1);
        uint32_t mn = 0xffffffffu, mx = 0, unused = 0;
        for (uint32_t k = tid; k < nb; k += kThreads) {
          const uint2 r = B.b[k];
          if (r.y >= r.x) {
            mn = min(mn, r.x);
            mx = max(mx, r.y);
          }
        }
        block_min_max_max(S, mn, mx, unused, phase);
        if (mn > mx) {
          mode = kEmpty;
        } else {
          uint32_t sb = 2;
          while (sb < kMaxBlock && sb * 4 <= d.wmax) sb <<= 1;
          T.sb_shift = __ffs(sb) - 1;
          T.base = mn & ~31u;
          T.nwt = uint32_t(((uint64_t(mx) - T.base) >> 5) + 2);
          T.pitch = T.span | 1u;
          const uint32_t nblk = (T.span + sb - 1) >> T.sb_shift;
          T.bpitch = nblk | 1u;
          if ((2ull * T.pitch + T.bpitch) * T.nwt > kBitWords) mode = kDirect;
        }
      }

      if (mode == kTiled) {
        // union bitmaps, one warp per (word, 32 staged rows): lane l holds
        // R_j (j = 32 u + l) on word w; segmented OR-scans of width sb give
        // the prefix (PRE) and suffix (SUF) unions inside each block; the
        // block's last lane holds the block union (BU).
        const BBuf& B = *T.B;
        uint32_t* PRE = S.u.t.bits;
        uint32_t* SUF = S.u.t.bits + size_t(T.nwt) * T.pitch;
        uint32_t* BU = S.u.t.bits + 2 * size_t(T.nwt) * T.pitch;
        const int sb = 1 << T.sb_shift;
        const int ls = lane & (sb - 1);
        const uint32_t nq = (T.span + 31) >> 5;
        for (uint32_t task = warp; task < nq * T.nwt; task += kWarps) {
          const uint32_t w = task / nq, u = task - w * nq;
          const uint32_t j = (u << 5) + lane;
          const uint32_t x = j < T.span ? row_mask(B, T.b_base, j, T.base + 32ull * w) : 0u;
          uint32_t pre = x, suf = x;
#pragma unroll
          for (int o = 1; o < kMaxBlock; o <<= 1) {
            if (o < sb) {
              uint32_t pu = __shfl_up_sync(kFullMask, pre, o, sb);
              if (ls >= o) pre |= pu;
              uint32_t sv = __shfl_down_sync(kFullMask, suf, o, sb);
              if (ls + o < sb) suf |= sv;
            }
          }
          if (j < T.span) {
            PRE[size_t(w) * T.pitch + j] = pre;
            SUF[size_t(w) * T.pitch + j] = suf;
          }
          if (ls == sb - 1 && (j >> T.sb_shift) < T.bpitch) BU[size_t(w) * T.bpitch + (j >> T.sb_shift)] = pre;
        }
        __syncthreads();

        // rows: groups of g lanes, one window word per lane and chunk; a
        // group holds at most 4 rows (64 rows, >= 16 groups)
        const int g = T.nwt <= 4 ? 4 : T.nwt <= 8 ? 8 : T.nwt <= 16 ? 16 : 32;
        const int lg = tid & (g - 1);
        const unsigned gm = runtime_group_mask(g);
        const uint32_t gid = tid / g, ngroups = kThreads / g;
        const bool one_chunk = T.nwt <= uint32_t(g);
        uint32_t xs[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const uint32_t r = gid + u * ngroups;
          xs[u] = 0;
          if (r < rows) {
            uint32_t cnt;
            if (one_chunk) {
              const bool valid = uint32_t(lg) < T.nwt;
              const uint32_t x = valid ? tiled_acc(S, T, r, lg) : 0u;
              xs[u] = x;
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
        for (int u = 0; u < 4; ++u) {
          const uint32_t r = gid + u * ngroups;
          if (r < fit) {
            uint32_t* st = S.u.t.stage + S.sub_off[r];
            if (one_chunk) {
              const bool valid = uint32_t(lg) < T.nwt;
              uint32_t carry = 0;
              gather_chunk(xs[u], valid, T.base + 32ull * lg, g, lg, gm, carry, 0, T.nwt - 1,
                           [&](uint64_t k, uint32_t v) { st[k] = v; });
            } else {
              tiled_row(S, T, r, g, lg, gm, nullptr, [&](uint64_t k, uint32_t v) { st[k] = v; });
            }
          }
        }
      } else if (mode == kDirect) {
        any_direct = true;
        uint32_t* bits = S.u.t.bits + size_t(warp) * 2 * kDirectWW;
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
          uint32_t* st = S.u.t.stage + S.sub_off[r];
          direct_row(p, A_ID, uint64_t(i0) + r, bits, reach, nullptr, [&](uint64_t k, uint32_t v) { st[k] = v; });
        }
      } else {
        if (tid < int(rows)) S.incl[r0 + tid] = 0;
        __syncthreads();
        if (warp == 0) stage_rows(S, r0, rows);
      }
      __syncthreads();
    }

    // ---- chunk prefix over the row counts (4 consecutive rows per thread)
    {
      constexpr int kPer = kChunkMax / kThreads;
      uint32_t loc[kPer];
      uint64_t s = 0;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        const uint32_t r = tid * kPer + k;
        s += r < crows ? S.incl[r] : 0u;
        loc[k] = uint32_t(s);
      }
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
      for (int k = 0; k < kPer; ++k) {
        const uint32_t r = tid * kPer + k;
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

    // ---- rowmap, staged entries, and the rows that did not fit the stage
    for (uint32_t r = tid; r < crows; r += kThreads) p.c_rowmap[uint64_t(c0row) + r + 1] = prefix + S.incl[r];
    if (t == 0 && tid == 0) p.c_rowmap[0] = 0;
    const uint32_t staged = S.stage_used;
    if (prefix + staged <= p.cap) {
      for (uint32_t k = tid; k < staged; k += kThreads) p.c_entries[prefix + k] = S.u.t.stage[k];
    } else if (tid == 0) {
      atomicOr(&p.ctl->overflow, 1ull);
    }
    const uint32_t srows = S.staged_rows;
    if (srows < crows) {
      uint32_t* bits = S.u.t.bits + size_t(warp) * 2 * kDirectWW;
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

// Mean A range length above which the automatic mode stages tiles.
constexpr double kWideRangeMean = 8.0;

// Scratch for one single-pass product on the context: the chunk descriptors
// (zeroed) and the ticket (zeroed).
static void* chunk_scratch(dvg_context* ctx, size_t desc_bytes) {
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
  return ctx->d_tile_desc;
}

// Staging for one single-pass row product on the context (null when the
// deferred write-out is off).
static uint32_t* stage_scratch(dvg_context* ctx, size_t bytes) {
  if (!ctx->opt_row_stage || bytes == 0) return nullptr;
  if (bytes > ctx->row_stage_cap) {
    if (ctx->d_row_stage) dfree(ctx, ctx->d_row_stage);
    ctx->d_row_stage = nullptr;
    ctx->row_stage_cap = 0;
    ctx->d_row_stage = static_cast<uint32_t*>(dalloc(ctx, bytes));
    ctx->row_stage_cap = bytes;
  }
  return ctx->d_row_stage;
}

void launch_row_shifted_sum(dvg_context* ctx, const dvg_matrix* u, uint32_t shift, uint64_t* c_rowmap,
                            uint32_t* c_entries, uint64_t cap) {
  if (u->nrows == 0) return;
  // level rows gather many runs: unless set, a row per thread and the widest run list
  const int64_t chunk_rows = ctx->opt_chunk_rows ? ctx->opt_chunk_rows : 512;
  const int slot = ctx->opt_row_slot == 1 ? 2 : int(ctx->opt_row_slot);
  const RowLaunchShape shape = row_launch_shape(ctx, u->nrows, chunk_rows, slot);
  RowLaunch L{};
  L.a_identity = true;
  L.a_shift = shift;
  L.b_rowmap = u->rowmap;
  L.b_entries = u->entries;
  L.b_nrows = u->nrows;
  L.d_rowmap = u->rowmap;
  L.d_entries = u->entries;
  L.c_rowmap = c_rowmap;
  L.c_entries = c_entries;
  L.cap = cap;
  L.nrows = u->nrows;
  L.desc = chunk_scratch(ctx, shape.desc_bytes);
  L.ticket = ctx->d_ticket;
  L.ctl = ctx->d_ctl;
  L.stage_buf = stage_scratch(ctx, shape.stage_bytes);
  L.slot_variant = slot;
  launch_rowmode(ctx, L, shape);
}

void launch_spgemm_fused(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b,
                         const dvg_matrix* d, uint64_t* c_rowmap, uint32_t* c_entries, uint64_t cap,
                         const std::vector<dvg_matrix*>* levels) {
  const uint32_t n = a_identity ? b->nrows : a->nrows;
  if (n == 0) return;
  // mode 1 forces the tile-staged kernel, mode 2 the row kernel, mode 3 the
  // warp-per-row kernel; automatic (0) takes the warp-per-row kernel when A's
  // ranges are long on average (a row then names many B ranges) and the row
  // kernel otherwise.  An addend needs the row or the warp-per-row kernel.
  const bool long_ranges = !a_identity && !(levels && !levels->empty()) && a->nentries > 0 &&
                           double(a->nnz) > kWideRangeMean * double(a->nentries / 2);
  if ((ctx->opt_spgemm_mode == 3 || (ctx->opt_spgemm_mode == 0 && long_ranges)) && !a_identity &&
      !(levels && !levels->empty())) {
    void* desc = chunk_scratch(ctx, spgemm_wide_desc_bytes(n));
    launch_spgemm_wide(ctx, a, b, d, c_rowmap, c_entries, cap, desc, ctx->d_ticket);
    return;
  }
  bool row_mode = ctx->opt_spgemm_mode != 1;
  if (d && !row_mode) throw Error(DVG_ERR_INVALID_ARG, "fused spgemm: an addend needs the row kernel");
  if (row_mode) {
    // products that read union levels (long A ranges) have rows of many runs:
    // unless set, a row per thread and the widest run list
    const bool wide = levels && !levels->empty();
    const int64_t chunk_rows = ctx->opt_chunk_rows ? ctx->opt_chunk_rows : (wide ? 512 : 0);
    const int slot = wide && ctx->opt_row_slot == 1 ? 2 : int(ctx->opt_row_slot);
    const RowLaunchShape shape = row_launch_shape(ctx, n, chunk_rows, slot);
    RowLaunch L{};
    L.a_rowmap = a_identity ? nullptr : a->rowmap;
    L.a_entries = a_identity ? nullptr : a->entries;
    L.a_identity = a_identity;
    L.b_rowmap = b->rowmap;
    L.b_entries = b->entries;
    L.b_nrows = b->nrows;
    if (levels) {
      L.nlevels = uint32_t(std::min<size_t>(levels->size(), 12));
      for (uint32_t k = 0; k < L.nlevels; ++k) {
        L.lv_rowmap[k] = (*levels)[k]->rowmap;
        L.lv_entries[k] = (*levels)[k]->entries;
      }
    }
    L.d_rowmap = d ? d->rowmap : nullptr;
    L.d_entries = d ? d->entries : nullptr;
    L.c_rowmap = c_rowmap;
    L.c_entries = c_entries;
    L.cap = cap;
    L.nrows = n;
    L.desc = chunk_scratch(ctx, shape.desc_bytes);
    L.ticket = ctx->d_ticket;
    L.ctl = ctx->d_ctl;
    L.stage_buf = stage_scratch(ctx, shape.stage_bytes);
    L.slot_variant = slot;
    launch_rowmode(ctx, L, shape);
    return;
  }
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
  FusedArgs p{};
  p.a_rowmap = a_identity ? nullptr : a->rowmap;
  p.a_entries = a_identity ? nullptr : a->entries;
  p.b_rowmap = b->rowmap;
  p.b_entries = b->entries;
  p.c_rowmap = c_rowmap;
  p.c_entries = c_entries;
  p.cap = cap;
  p.desc = static_cast<ChunkDesc*>(chunk_scratch(ctx, size_t(nchunks) * sizeof(ChunkDesc)));
  p.ticket = ctx->d_ticket;
  p.ctl = ctx->d_ctl;
  p.nrows = n;
  p.chunk_rows = chunk_rows;
  p.nchunks = nchunks;
  p.row_mode = 0;
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
constexpr size_t kNoAllocCheckOffset = kNoAllocTicketOffset + 256;     // validation words of A and B
constexpr size_t kNoAllocBytes = kNoAllocCheckOffset + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Records in *bad the memory-safety preconditions of the fused kernel that a
// range-CRS matrix violates, with the bits of the upload check (1: rowmap[0]
// != 0, 2: a decreasing rowmap or an odd row length, 4: rowmap[n] !=
// nentries, 8: a column >= ncols).
__global__ void k_noalloc_validate(const uint64_t* __restrict__ rowmap, uint32_t nrows,
                                   const uint32_t* __restrict__ entries, uint64_t nentries, uint32_t ncols,
                                   unsigned long long* bad) {
  unsigned long long b = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  for (uint64_t i = tid; i < nrows; i += stride) {
    const uint64_t lo = rowmap[i], hi = rowmap[i + 1];
    if (hi < lo || ((hi - lo) & 1)) b |= 2;
  }
  if (tid == 0) {
    if (rowmap[0] != 0) b |= 1;
    if (rowmap[nrows] != nentries) b |= 4;
  }
  for (uint64_t i = tid; i < nentries; i += stride)
    if (entries[i] >= ncols) b |= 8;
  if (b) atomicOr(bad, b);
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
    // In host code g_noalloc_scratch names a host-side stand-in, not device
    // memory: the array's address on the current device comes from the
    // runtime.  It is looked up on every call (a host-side table lookup)
    // rather than kept, because a device reset or a new primary context
    // reloads the module and may move the array.
    void* scratch_ptr = nullptr;
    DVG_CUDA(cudaGetSymbolAddress(&scratch_ptr, g_noalloc_scratch));
    unsigned char* scratch = static_cast<unsigned char*>(scratch_ptr);
    ChunkDesc* desc = reinterpret_cast<ChunkDesc*>(scratch);
    DeviceControl* ctl = reinterpret_cast<DeviceControl*>(scratch + kNoAllocCtlOffset);
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kNoAllocTicketOffset);
    unsigned long long* check = reinterpret_cast<unsigned long long*>(scratch + kNoAllocCheckOffset);
    DeviceControl h{};
    if (a_nrows == 0) {
      DVG_CUDA(cudaMemsetAsync(d_c_rowmap, 0, sizeof(uint64_t), stream));
      DVG_CUDA(cudaStreamSynchronize(stream));
      return DVG_OK;
    }
    // 1. inputs must be well formed before the product may index through them
    int nsm = 0;
    DVG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DVG_CUDA(cudaMemsetAsync(check, 0, 2 * sizeof(unsigned long long), stream));
    const unsigned vgrid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(
        (std::max<uint64_t>(std::max<uint64_t>(a_nrows, a_nentries), std::max<uint64_t>(b_nrows, b_nentries)) +
         255) / 256, uint64_t(nsm) * 8)));
    k_noalloc_validate<<<vgrid, 256, 0, stream>>>(d_a_rowmap, a_nrows, d_a_entries, a_nentries, a_ncols, check);
    k_noalloc_validate<<<vgrid, 256, 0, stream>>>(d_b_rowmap, b_nrows, d_b_entries, b_nentries, b_ncols, check + 1);
    DVG_CUDA(cudaGetLastError());
    unsigned long long bad[2] = {0, 0};
    DVG_CUDA(cudaMemcpyAsync(bad, check, sizeof(bad), cudaMemcpyDeviceToHost, stream));
    DVG_CUDA(cudaStreamSynchronize(stream));
    if (bad[0] || bad[1]) {
      std::string why;
      if (bad[0]) why += " A:" + validation_message(bad[0]);
      if (bad[1]) why += " B:" + validation_message(bad[1]);
      throw Error(DVG_ERR_INVALID_ARG, "malformed range-CRS input matrix;" + why);
    }
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
    p.row_mode = 0;
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
