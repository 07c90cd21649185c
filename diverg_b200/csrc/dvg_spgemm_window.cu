// dvg_spgemm_window.cu -- the thread-per-row range SpGEMM with its operands'
// windows staged in shared memory: C = A B or C = D + A B (D a matrix of C's
// shape, or the identity).
//
// Same result as the reference's symbolic + numeric SpGEMM
// (include/diverg/range_sparse.hpp:1132-1442 in cartoonist/diverg, dispatched
// by range_spgemm :2215-2281) followed, for the sums, by range_spadd
// (:112-357) on canonical operands: row r of C is the union of D's row r and
// of all ranges of B rows s..f for every range [s,f] of A's row r, emitted as
// sorted maximal runs (merge on start <= hi + 1, as the reference's
// accumulators merge).
//
// Why a second row kernel.  k_spgemm_rowmode walks every row straight from
// HBM: per row a chain of dependent loads (addend row pointers -> addend
// ranges; A range -> B row pointers -> B ranges), four rows per thread one
// after the other.  With 32 warps per SM that keeps too few bytes in flight
// (latency-bound at 30 % of HBM bandwidth).  Here a chunk's operands are
// copied into shared memory before its rows are walked: the chunk's A and
// addend row pointers and ranges (contiguous in HBM) and the window of B rows
// its A ranges name (contiguous too: the rows of an index product reach a
// band of columns near their own), each copy issued by every thread at once
// with cp.async -- kilobytes in flight per CTA, no registers held.  The copies
// of chunk t+1 are issued while chunk t's predecessor is written out (its
// look-back and image copy), so their latency overlaps that work.  A range
// outside a staged window, or a chunk whose ranges exceed a stage's capacity,
// falls back to reading HBM for the missing part; results are identical.
//
// Each row is walked once, from shared memory.  A row of one run keeps it in
// shared memory (frun), a row of more runs writes them to a per-CTA scratch
// in global memory (L2-resident, 8 entries a row); rows whose runs overflow
// the walk's 4-run list are recomputed from HBM by the warp-cooperative path.
// So once a chunk is counted its stages are dead, and the next chunk's
// operands are requested at once: their latency overlaps the counted chunk's
// prefix and image and the write-out of the chunk before it.  Output order,
// deferred write-out through per-CTA staging buffers, the CTA-wide decoupled
// look-back, bounded waits, the abort word of planned builds and every
// self-check are those of k_spgemm_rowmode.
#include <algorithm>

#include "dvg_spgemm_common.cuh"

namespace dvg {
namespace {

constexpr int kWRows = kChunkMax;          // rows per chunk (upper bound)
constexpr int kWRpt = kWRows / kThreads;   // rows per thread at the largest chunk
// stage capacities: a little above a chunk's rows, as index products average
// slightly more than one range a row (a chunk that holds more reads the rest
// from HBM)
constexpr int kWAEnt = 2304;               // A ranges staged per chunk
constexpr int kWDEnt = 2304;               // addend ranges staged per chunk
constexpr int kWBRows = 2559;              // B rows in the staged window (at most)
constexpr int kWBEnt = 2688;               // B ranges staged per chunk
constexpr int kWList = 8;                  // run-list entries per walking thread (four closed runs)
constexpr int kWGenThreads = 256;          // threads that walk the general rows
constexpr int kWRowScratch = kRowScratchPerRow;  // scratch entries a row (four runs)
constexpr int kWDirectWarps = 2;           // warps that run the warp path
constexpr int kWDirectWW = 192;            // warp path: 32-bit window words per warp
constexpr int kWRowStagePerRow = 16;       // image entries per chunk row, as the staging buffers are sized

// Shared memory of one CTA.  The next chunk's 64-bit A row pointers land in
// `bent` and its addend row pointers in `dent` before they are compacted to
// 16 bits, and the B window's row pointers land in `bent` before the B
// ranges do: those arrays are free while a chunk is being staged.
struct WinSmem {
  uint2 aent[kWAEnt];     // the chunk's A ranges (from abase on)
  uint2 dent[kWDEnt];     // the chunk's addend ranges (from dbase on)
  uint2 bent[kWBEnt];     // the B window's ranges (from bbase on)
  uint2 frun[kWRows];     // the counted chunk's rows: the run of a one-run row, or a kFrun* marker
  uint32_t list[kWList * kWGenThreads];  // closed runs of the row in hand: entry k of thread t at [k * kWGenThreads + t]
  // range offsets (rowmap / 2) relative to the stage's first range, in 16 bits:
  // A and addend rows c0 .. c0 + crows, B rows wlo .. wlo + wn; row r spans
  // [x[r], x[r + 1]) of its stage (a chunk's rows are used only while it holds
  // < 2^16 ranges)
  uint16_t arow[kWRows + 1];
  uint16_t drow[kWRows + 1];
  uint16_t brow[kWBRows + 1];
  uint32_t incl[kWRows];      // the counted chunk's (then chunk-local inclusive) row counts
  uint32_t slow[kSlowMax];    // rows of the counted chunk left to the warp path
  uint16_t gen[kWRows];       // rows of the counted chunk left to the general walk (kinds marked)
  uint32_t direct[2 * kWDirectWW * kWDirectWarps];  // warp path: bits + reach per warp
  unsigned long long red[kWarps];
  unsigned long long red_nnz[kWarps];
  unsigned long long lb_sum[2][kWarps];  // look-back records by round parity, per warp
  uint32_t lb_flag[2][kWarps];
  uint32_t phase[kWarps];                // iterations per warp, checked at every iteration's end
  uint32_t wmin[kWarps], wmax[kWarps];   // per-warp bounds of the chunk's A ranges
  unsigned long long abase, dbase, bbase;  // 64-bit range offset of each stage's first range
  // the staged chunk waiting in image buffer k, kept per buffer: its readers
  // (the next iteration) and the writer of the next one (that iteration's
  // end, which a look-back of no rounds may not separate from them by a
  // barrier) never meet on one slot
  unsigned long long pend_cnt[2];
  uint32_t na, nd, nb;                   // ranges staged
  uint32_t rows_ok;                      // bit 0: arow usable, bit 1: drow usable (< 2^16 ranges)
  uint32_t wlo, wn;                      // staged B rows [wlo, wlo + wn)
  uint32_t wn_req;                       // B rows whose row pointers were requested (from wlo)
  uint32_t pend_t[2], pend_crows[2];
  uint32_t next;                         // the chunk taken for the next iteration
  uint32_t nslow;
  uint32_t ngen;
};
static_assert(sizeof(WinSmem) <= 115712, "two CTAs per SM must fit");
static_assert(sizeof(uint2) * kWBEnt >= 8 * (kWRows + 1) && sizeof(uint2) * kWDEnt >= 8 * (kWRows + 1),
              "the next chunk's row pointers fit bent and dent");
static_assert(sizeof(uint2) * kWBEnt >= 8 * (kWBRows + 1), "the B window's row pointers fit bent");

// frun markers (x > y, so no run): the row's runs are in the CTA's scratch,
// or are recomputed by the warp path, or by the per-thread bit-window walk.
constexpr uint32_t kFrunScratch = 0xffffffffu, kFrunWarp = 0xfffffffeu, kFrunLight = 0xfffffffdu;

// Offset of row k's first range in its stage.
__device__ __forceinline__ uint32_t rel(const uint16_t* x, uint32_t k) { return x[k]; }

// ---- staging ------------------------------------------------------------------
// Four phases, each ended by the next one's wait: (1) request the chunk's A
// and addend row pointers; (2) compact them, request the A and addend ranges;
// (3) bound the B rows the staged A ranges name, request their row pointers;
// (4) clip the window to the B-range capacity, compact, request the B ranges.
// Every phase is called by the whole CTA (uniform branches).

template <bool A_ID>
__device__ void stage_req_rows(WinSmem& S, const FusedArgs& p, uint32_t c0row, uint32_t crows) {
  uint64_t* rawA = reinterpret_cast<uint64_t*>(S.bent);
  uint64_t* rawD = reinterpret_cast<uint64_t*>(S.dent);
  for (uint32_t k = threadIdx.x; k <= crows; k += kThreads) {
    if (!A_ID) cp_async8(rawA + k, p.a_rowmap + uint64_t(c0row) + k);
    if (p.d_rowmap) cp_async8(rawD + k, p.d_rowmap + uint64_t(c0row) + k);
  }
  cp_async_commit();
}

template <bool A_ID>
__device__ void stage_rows_req_ranges(WinSmem& S, const FusedArgs& p, uint32_t crows) {
  const uint64_t* rawA = reinterpret_cast<const uint64_t*>(S.bent);
  const uint64_t* rawD = reinterpret_cast<const uint64_t*>(S.dent);
  cp_async_wait();
  cta_sync();
  // every thread reads the same words: the stage sizes are uniform
  uint64_t abase = 0, na64 = 0, dbase = 0, nd64 = 0;
  if (!A_ID) {
    abase = rawA[0] >> 1;
    na64 = (rawA[crows] >> 1) - abase;
  }
  if (p.d_rowmap) {
    dbase = rawD[0] >> 1;
    nd64 = (rawD[crows] >> 1) - dbase;
  }
  for (uint32_t k = threadIdx.x; k <= crows; k += kThreads) {
    if (!A_ID) S.arow[k] = uint16_t((rawA[k] >> 1) - abase);
    if (p.d_rowmap) S.drow[k] = uint16_t((rawD[k] >> 1) - dbase);
  }
  const uint32_t na = uint32_t(min(na64, uint64_t(kWAEnt)));
  const uint32_t nd = uint32_t(min(nd64, uint64_t(kWDEnt)));
  if (threadIdx.x == 0) {
    S.abase = abase;
    S.dbase = dbase;
    S.na = na;
    S.nd = nd;
    // 16-bit row offsets hold while a chunk's ranges stay below 2^16
    S.rows_ok = (na64 < (1ull << 16) ? 1u : 0u) | (nd64 < (1ull << 16) ? 2u : 0u);
  }
  cta_sync();  // the raw words are dead from here on
  for (uint32_t k = threadIdx.x; k < na; k += kThreads) cp_async8(&S.aent[k], p.a_entries + 2 * (abase + k));
  for (uint32_t k = threadIdx.x; k < nd; k += kThreads) cp_async8(&S.dent[k], p.d_entries + 2 * (dbase + k));
  cp_async_commit();
}

template <bool A_ID>
__device__ void stage_window_req_brows(WinSmem& S, const FusedArgs& p, uint32_t c0row, uint32_t crows) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  cp_async_wait();
  cta_sync();
  uint32_t mn = 0xffffffffu, mx = 0;
  if (A_ID) {
    const uint64_t lo = uint64_t(c0row) + p.a_shift, hi = lo + crows - 1;
    if (lo < p.b_nrows) {
      mn = uint32_t(lo);
      mx = uint32_t(min(hi, uint64_t(p.b_nrows) - 1));
    }
  } else {
    const uint32_t na = S.na;
    for (uint32_t k = tid; k < na; k += kThreads) {
      const uint2 r = S.aent[k];
      if (r.y < r.x) continue;
      mn = min(mn, r.x);
      mx = max(mx, r.y);
    }
    mn = group_min<32>(kFullMask, mn);
    mx = group_max<32>(kFullMask, mx);
    if (lane == 0) {
      S.wmin[warp] = mn;
      S.wmax[warp] = mx;
    }
    cta_sync();
    mn = 0xffffffffu;
    mx = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      mn = min(mn, S.wmin[w]);
      mx = max(mx, S.wmax[w]);
    }
  }
  // A's columns index B's rows (< b_nrows); the window is clipped to the stage
  uint32_t wn = 0;
  if (mn <= mx && mn < p.b_nrows) {
    const uint64_t hi = min(uint64_t(mx), uint64_t(p.b_nrows) - 1);
    wn = uint32_t(min(hi - mn + 1, uint64_t(kWBRows)));
  }
  if (tid == 0) {
    S.wlo = mn;
    S.wn_req = wn;
  }
  uint64_t* raw = reinterpret_cast<uint64_t*>(S.bent);
  if (wn)
    for (uint32_t k = tid; k <= wn; k += kThreads) cp_async8(raw + k, p.b_rowmap + uint64_t(mn) + k);
  cp_async_commit();
}

__device__ void stage_brows_req_branges(WinSmem& S, const FusedArgs& p) {
  const int tid = threadIdx.x;
  cp_async_wait();
  cta_sync();
  const uint64_t* raw = reinterpret_cast<const uint64_t*>(S.bent);
  uint32_t wn = S.wn_req;
  uint64_t bbase = 0, nb64 = 0;
  if (wn) {
    bbase = raw[0] >> 1;
    // the longest run of whole rows from wlo whose ranges fit the stage
    // (the same search in every thread: uniform result)
    if ((raw[wn] >> 1) - bbase > uint64_t(kWBEnt)) {
      uint32_t lo = 0, hi = wn;  // rows [0, lo) fit; rows [0, hi] do not
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((raw[mid] >> 1) - bbase <= uint64_t(kWBEnt)) lo = mid;
        else hi = mid;
      }
      wn = lo;
    }
    nb64 = (raw[wn] >> 1) - bbase;
  }
  for (uint32_t k = tid; k <= wn && wn; k += kThreads) S.brow[k] = uint16_t((raw[k] >> 1) - bbase);
  if (tid == 0) {
    S.wn = wn;
    S.bbase = bbase;
    S.nb = uint32_t(nb64);
  }
  cta_sync();  // the raw words are dead from here on
  for (uint32_t k = tid; k < uint32_t(nb64); k += kThreads) cp_async8(&S.bent[k], p.b_entries + 2 * (bbase + k));
  cp_async_commit();
}

// All four phases at once, complete on return.
template <bool A_ID>
__device__ void stage_chunk(WinSmem& S, const FusedArgs& p, uint32_t t) {
  const uint32_t c0row = t * p.chunk_rows;
  const uint32_t crows = min(p.chunk_rows, p.nrows - c0row);
  stage_req_rows<A_ID>(S, p, c0row, crows);
  stage_rows_req_ranges<A_ID>(S, p, crows);
  stage_window_req_brows<A_ID>(S, p, c0row, crows);
  stage_brows_req_branges(S, p);
  cp_async_wait();
  cta_sync();
}

// ---- one row ---------------------------------------------------------------------
//
// Nearly every row of an index product is the union of at most two ranges:
// its addend range and the one range of the B row its single A range names
// (measured on the products of a synthetic chromosome graph: 97-99.8 % of
// rows).  fast_row does such a row on a short straight path from the stages
// and returns true, with count = its entries, its nnz accumulated and its
// runs kept (a run in frun[r]; two runs in the row's scratch slot `scr`);
// any other row (more ranges, unstaged data, union levels) returns false and
// is listed for the general walk, which the CTA spreads over kWGenThreads
// threads of all warps -- a handful of general rows per chunk, so no warp
// waits on a warp that met one.
template <bool A_ID>
__device__ __forceinline__ bool fast_row(WinSmem& S, const FusedArgs& p, uint32_t row, uint32_t r, uint32_t& count,
                                         unsigned long long& nnz, uint32_t* scr) {
  // the caller checked that the chunk's stages have usable row offsets and
  // that no union levels are in play
  uint2 u = make_uint2(1u, 0u), v = make_uint2(1u, 0u);  // the row's (at most) two input ranges
  bool ok = true;
  if (p.d_identity) {
    u = make_uint2(row, row);
  } else if (p.d_rowmap) {
    const uint32_t d0 = S.drow[r], d1 = S.drow[r + 1];
    ok = d1 - d0 <= 1u && d1 <= S.nd;
    if (ok && d1 > d0) u = S.dent[d0];
  }
  uint2 ar = make_uint2(1u, 0u);
  if (A_ID) {
    ar = id_range(p, row);
  } else {
    const uint32_t a0 = S.arow[r], a1 = S.arow[r + 1];
    ok = ok && a1 - a0 == 1u && a1 <= S.na;
    if (ok) ar = S.aent[a0];
  }
  if (ok && ar.x <= ar.y) {
    // B rows s..f in the window: f - wlo < wn and s >= wlo (s - wlo <= f - wlo)
    const uint32_t x = ar.x - S.wlo, y = ar.y - S.wlo;
    ok = y < S.wn && x <= y;
    if (ok) {
      const uint32_t t0 = S.brow[x], t1 = S.brow[y + 1];
      ok = t1 - t0 <= 1u;
      if (ok && t1 > t0) v = S.bent[t0];
    }
  }
  if (!ok) return false;
  const bool hu = u.x <= u.y, hv = v.x <= v.y;
  if (hu && hv && v.x < u.x) {
    const uint2 w = u;
    u = v;
    v = w;
  }
  uint32_t nr;
  uint2 r0 = hu ? u : v, r1 = v;
  if (hu && hv) {
    if (v.x <= u.y || v.x - u.y == 1u) {  // overlapping or adjacent: one run
      r0 = make_uint2(u.x, max(u.y, v.y));
      nr = 1;
    } else {
      nr = 2;
    }
  } else {
    nr = (hu || hv) ? 1u : 0u;
  }
  if (nr == 2) {
    *reinterpret_cast<uint4*>(scr) = make_uint4(r0.x, r0.y, r1.x, r1.y);
    S.frun[r] = make_uint2(kFrunScratch, 0u);
    nnz += uint64_t(r0.y - r0.x) + uint64_t(r1.y - r1.x) + 2;
  } else {
    S.frun[r] = r0;
    if (nr) nnz += uint64_t(r0.y - r0.x) + 1;
  }
  count = 2 * nr;
  return true;
}

// The general walk of C row `row` (chunk row r) from the stages (HBM for what
// is not staged) into run list `slot` (< kWGenThreads) of the walking thread.
// Returns true with count = the row's entries, its nnz accumulated and its
// runs kept as fast_row keeps them (more than one run: in its scratch slot
// `scr`); false, leaving no trace, when the runs overflow the list.
template <bool A_ID>
__device__ bool general_row(WinSmem& S, const FusedArgs& p, uint64_t row, uint32_t r, uint32_t& count,
                            unsigned long long& nnz, uint32_t* scr, uint32_t slot) {
  constexpr uint32_t kT = kWGenThreads;
  uint32_t* L = S.list + slot;  // run k: lo at L[2k*kT], hi at L[(2k+1)*kT]
  constexpr uint32_t max_runs = kWList / 2;
  uint32_t nr = 0;
  // merges [x, y] into the list; false when it needs more runs than fit
  auto merge = [&](uint32_t x, uint32_t y) -> bool {
    uint32_t k = 0;
    while (k < nr && uint64_t(L[(2 * k + 1) * kT]) + 1 < x) ++k;
    if (k == nr || uint64_t(y) + 1 < L[2 * k * kT]) {
      if (nr == max_runs) return false;
      for (uint32_t m = nr; m > k; --m) {
        L[2 * m * kT] = L[2 * (m - 1) * kT];
        L[(2 * m + 1) * kT] = L[(2 * m - 1) * kT];
      }
      L[2 * k * kT] = x;
      L[(2 * k + 1) * kT] = y;
      ++nr;
      return true;
    }
    uint32_t lo = min(L[2 * k * kT], x), hi = max(L[(2 * k + 1) * kT], y);
    uint32_t m = k + 1;
    while (m < nr && uint64_t(hi) + 1 >= L[2 * m * kT]) {
      hi = max(hi, L[(2 * m + 1) * kT]);
      ++m;
    }
    L[2 * k * kT] = lo;
    L[(2 * k + 1) * kT] = hi;
    const uint32_t gone = m - k - 1;
    if (gone) {
      for (uint32_t q = m; q < nr; ++q) {
        L[2 * (q - gone) * kT] = L[2 * q * kT];
        L[(2 * (q - gone) + 1) * kT] = L[(2 * q + 1) * kT];
      }
      nr -= gone;
    }
    return true;
  };
  bool any = false;
  uint32_t run_lo = 0, run_hi = 0;
  // one input range: extend the open run, or merge the open run and open anew
  auto take = [&](uint2 b) -> bool {
    if (b.y < b.x) return true;
    if (!any) {
      any = true;
      run_lo = b.x;
      run_hi = b.y;
      return true;
    }
    if (uint64_t(b.x) <= uint64_t(run_hi) + 1 && uint64_t(b.y) + 1 >= run_lo) {
      run_lo = min(run_lo, b.x);
      run_hi = max(run_hi, b.y);
      return true;
    }
    if (!merge(run_lo, run_hi)) return false;
    run_lo = b.x;
    run_hi = b.y;
    return true;
  };
  const uint32_t rows_ok = S.rows_ok;
  // the addend
  if (p.d_identity) {
    take(make_uint2(uint32_t(row), uint32_t(row)));
  } else if (p.d_rowmap) {
    uint64_t d0, d1;
    if (rows_ok & 2u) {
      d0 = rel(S.drow, r);
      d1 = rel(S.drow, r + 1);
    } else {
      d0 = (__ldg(p.d_rowmap + row) >> 1) - S.dbase;
      d1 = (__ldg(p.d_rowmap + row + 1) >> 1) - S.dbase;
    }
    const uint32_t nd = S.nd;
    for (uint64_t t = d0; t < d1; ++t)
      if (!take(t < nd ? S.dent[t] : load_range(p.d_entries, S.dbase + t))) return false;
  }
  // A's ranges and the B rows they name
  uint64_t a0 = 0, a1 = 1;
  if (!A_ID) {
    if (rows_ok & 1u) {
      a0 = rel(S.arow, r);
      a1 = rel(S.arow, r + 1);
    } else {
      a0 = (__ldg(p.a_rowmap + row) >> 1) - S.abase;
      a1 = (__ldg(p.a_rowmap + row + 1) >> 1) - S.abase;
    }
  }
  const uint32_t na = S.na, wlo = S.wlo, wn = S.wn;
  for (uint64_t k = a0; k < a1; ++k) {
    uint2 ar;
    if (A_ID) ar = id_range(p, row);
    else ar = k < na ? S.aent[k] : load_range(p.a_entries, S.abase + k);
    if (ar.y < ar.x) continue;
    if (p.nlevels && ar.y - ar.x >= 3u) {
      // blocks of 2^lv rows from s, the last one ending at f (they may overlap)
      const uint32_t len = ar.y - ar.x + 1;
      const uint32_t lv = min(uint32_t(31 - __clz(len)), p.nlevels);
      const uint32_t step = 1u << lv, last = ar.y - step + 1;
      const uint64_t* __restrict__ lr = p.lv_rowmap[lv - 1];
      const uint32_t* __restrict__ le = p.lv_entries[lv - 1];
      for (uint32_t blk0 = ar.x;; blk0 += step) {
        const uint32_t blk = min(blk0, last);
        const uint64_t u0 = __ldg(lr + blk) >> 1, u1 = __ldg(lr + uint64_t(blk) + 1) >> 1;
        for (uint64_t t = u0; t < u1; ++t)
          if (!take(load_range(le, t))) return false;
        if (blk == last) break;
      }
      continue;
    }
    if (ar.x >= wlo && uint64_t(ar.y) < uint64_t(wlo) + wn) {
      // every B range of rows s..f is staged (the window's ranges are whole rows)
      const uint32_t t0 = rel(S.brow, ar.x - wlo), t1 = rel(S.brow, ar.y + 1 - wlo);
      for (uint32_t t = t0; t < t1; ++t)
        if (!take(S.bent[t])) return false;
    } else {
      const uint64_t t0 = __ldg(p.b_rowmap + ar.x) >> 1, t1 = __ldg(p.b_rowmap + uint64_t(ar.y) + 1) >> 1;
      for (uint64_t t = t0; t < t1; ++t)
        if (!take(load_range(p.b_entries, t))) return false;
    }
  }
  if (any && !merge(run_lo, run_hi)) return false;
  uint64_t n = 0;
  for (uint32_t k = 0; k < nr; ++k) {
    const uint32_t lo = L[2 * k * kT], hi = L[(2 * k + 1) * kT];
    n += uint64_t(hi - lo) + 1;
    if (nr > 1) {
      scr[2 * k] = lo;
      scr[2 * k + 1] = hi;
    }
  }
  if (nr == 1) S.frun[r] = make_uint2(L[0], L[kT]);
  else if (nr > 1) S.frun[r] = make_uint2(kFrunScratch, 0u);
  count = 2 * nr;
  nnz += n;
  return true;
}

// ---- the kernel --------------------------------------------------------------------
// With rpt = ceil(chunk_rows / kThreads) rows per thread, thread (warp, lane)
// owns chunk rows (warp * rpt + u) * 32 + lane, u < rpt: the lanes of a warp
// take consecutive rows.  An iteration counts chunk t from its stages, then
// -- with the stages dead -- requests chunk t+1's operands phase by phase
// between its remaining steps: the warp path, the chunk's prefix, its image
// in staging buffer b (or, when it does not fit, its write-out in place) and
// the write-out of the chunk staged one iteration before (look-back, row
// map, one coalesced copy).
//
// Rows of a chunk: fast rows (fast_row) by their own thread; the rest, listed
// in S.gen, by the general walk spread over kWGenThreads threads; rows whose
// runs overflow the general walk's list by the warp path (S.slow, kSlowMax a
// chunk) or, past that list, by the per-thread bit-window walk (light_row),
// both recomputing from HBM when the runs are written.
template <bool A_ID>
__global__ void __launch_bounds__(kThreads, 2) k_spgemm_window(FusedArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WinSmem& S = *reinterpret_cast<WinSmem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* dbits = S.direct + size_t(warp < kWDirectWarps ? warp : 0) * 2 * kWDirectWW;
  uint32_t* dreach = dbits + kWDirectWW;
  const uint32_t rpt = (p.chunk_rows + kThreads - 1) / kThreads;  // 1..kWRpt
  // per CTA two buffers: a chunk's image (stage_cap entries), then its
  // chunk-local inclusive row counts (chunk_rows words); after every CTA's
  // buffers, per CTA kWRowScratch entries a chunk row for rows of several runs
  uint32_t* const stage = p.stage_buf + size_t(blockIdx.x) * 2 * (p.stage_cap + p.chunk_rows);
  uint32_t* const scratch = p.stage_buf + size_t(gridDim.x) * 2 * (p.stage_cap + p.chunk_rows) +
                            size_t(blockIdx.x) * kWRowScratch * p.chunk_rows;
  // a planned build stops at the first step whose output is unusable
  auto stopped = [&]() { return p.abort && *reinterpret_cast<volatile unsigned long long*>(p.abort) != 0; };
  if (tid == 0) {
    S.next = stopped() ? 0xffffffffu : atomicAdd(p.ticket, 1u);
    S.nslow = 0;
    S.ngen = 0;
  }
  cta_sync();
  uint32_t t = S.next, b = 0, par = 0;
  bool pend = false;  // a staged chunk waits in buffer b ^ 1 (described in S.pend_*)
  if (t < p.nchunks) stage_chunk<A_ID>(S, p, t);
  uint32_t iter = 0;
  // writes the runs of every row of the counted chunk at base + its
  // chunk-local offset (base: the image, or C at the chunk's prefix); a row
  // past `cap` entries of base is not written (an overflow is raised)
  auto write_rows = [&](uint32_t c0row, uint32_t crows, uint32_t nslow, uint32_t* base, unsigned long long cap) {
    const uint32_t* incl = S.incl;
#pragma unroll 1
    for (int u = 0; u < kWRpt; ++u) {
      if (uint32_t(u) >= rpt) break;
      const uint32_t r = (warp * rpt + u) * 32 + lane;
      if (r >= crows) continue;
      const uint32_t o = r ? incl[r - 1] : 0u;
      const uint32_t n = incl[r] - o;
      if (n == 0) continue;
      const uint2 f = S.frun[r];
      if (f.x == kFrunWarp) continue;  // the warp path below
      if (uint64_t(o) + n > cap) {     // only a chunk written in place can meet the end of C
        raise_flag(p, &p.ctl->overflow, 1ull);
        continue;
      }
      uint32_t* out = base + o;
      if (f.x <= f.y) {
        if (n != 2) raise_flag(p, &p.ctl->status, 8ull);
        out[0] = f.x;
        out[1] = f.y;
      } else if (f.x == kFrunScratch) {
        const uint32_t* scr = scratch + size_t(r) * kWRowScratch;
        if (n > uint32_t(kWRowScratch)) raise_flag(p, &p.ctl->status, 8ull);
        else
          for (uint32_t k = 0; k < n; ++k) out[k] = __ldcg(scr + k);
      } else {
        const uint32_t c = light_row<A_ID>(nullptr, nullptr, p, c0row, r, false, nullptr,
                                           [&](uint64_t k, uint32_t v) {
                                             if (k < n) out[k] = v;
                                           });
        if (c != n) raise_flag(p, &p.ctl->status, 8ull);
      }
    }
    if (warp < kWDirectWarps) {
      for (uint32_t i = warp; i < nslow; i += kWDirectWarps) {
        const uint32_t r = S.slow[i];
        const uint32_t o = r ? incl[r - 1] : 0u;
        const uint32_t n = incl[r] - o;
        if (n == 0) continue;
        if (uint64_t(o) + n > cap) {
          if (lane == 0) raise_flag(p, &p.ctl->overflow, 1ull);
          continue;
        }
        uint32_t* out = base + o;
        bool bad = false;
        const uint64_t c = direct_row(p, A_ID, uint64_t(c0row) + r, dbits, dreach, nullptr,
                                      [&](uint64_t k, uint32_t v) {
                                        if (k < n) out[k] = v;
                                        else bad = true;
                                      },
                                      kWDirectWW);
        if (bad || c != n) raise_flag(p, &p.ctl->status, 8ull);
      }
    }
  };
  while (t < p.nchunks || pend) {
    const bool have = t < p.nchunks;
    // the stage of chunk t may still be landing (requested last iteration)
    cp_async_wait();
    cta_sync();
    const uint32_t c0row = have ? t * p.chunk_rows : 0u;
    const uint32_t crows = have ? min(p.chunk_rows, p.nrows - c0row) : 0u;
    uint32_t* const incl = S.incl;
    unsigned long long nnz_acc = 0, cnt = 0, cnnz = 0;
    uint32_t nslow = 0;
    bool staged = false;
    uint32_t next = 0xffffffffu;
    if (have) {
      // the next chunk, taken while this one is counted (the ticket's
      // latency hides behind the rows; it is stored after them)
      if (tid == 0 && !stopped()) next = atomicAdd(p.ticket, 1u);
      // count: fast rows by their threads, the rest listed
      const bool try_fast = S.rows_ok == 3u && p.nlevels == 0;
#pragma unroll 1
      for (int u = 0; u < kWRpt; ++u) {
        if (uint32_t(u) >= rpt) break;
        const uint32_t r = (warp * rpt + u) * 32 + lane;
        if (r < crows) {
          uint32_t c = 0;
          if (try_fast && fast_row<A_ID>(S, p, c0row + r, r, c, nnz_acc, scratch + size_t(r) * kWRowScratch))
            incl[r] = c;
          else
            S.gen[atomicAdd(&S.ngen, 1u)] = uint16_t(r);
        }
      }
      cta_sync();
      // the general walk, spread over the warps (lanes < kGenLanes of each):
      // entry i to warp i % kWarps, so the warps share the few general rows
      // of a chunk instead of one warp serialising them
      const uint32_t ngen = S.ngen;
      constexpr uint32_t kGenLanes = kWGenThreads / kWarps;
      if (uint32_t(lane) < kGenLanes) {
        const uint32_t slot = warp * kGenLanes + lane;  // the walker's run list
        for (uint32_t i = uint32_t(lane) * kWarps + warp; i < ngen; i += kWGenThreads) {
          const uint32_t r = S.gen[i];
          uint32_t c = 0;
          if (!general_row<A_ID>(S, p, uint64_t(c0row) + r, r, c, nnz_acc, scratch + size_t(r) * kWRowScratch,
                                 slot)) {
            const uint32_t j = atomicAdd(&S.nslow, 1u);
            if (j < uint32_t(kSlowMax)) {
              S.slow[j] = r;
              S.frun[r] = make_uint2(kFrunWarp, 0u);
            } else {
              c = light_row<A_ID>(nullptr, nullptr, p, c0row, r, false, &nnz_acc, [](uint64_t, uint32_t) {});
              S.frun[r] = make_uint2(kFrunLight, 0u);
            }
            atomicAdd(&p.ctl->slow_rows, 1ull);
          }
          incl[r] = c;
        }
      }
      if (tid == 0) S.next = next;
      cta_sync();
    }
    // the counted chunk's stages are dead: request the next chunk's operands
    const uint32_t tn = S.next;
    const bool pre = have && tn < p.nchunks;
    const uint32_t n0row = pre ? tn * p.chunk_rows : 0u;
    const uint32_t ncrows = pre ? min(p.chunk_rows, p.nrows - n0row) : 0u;
    if (pre) stage_req_rows<A_ID>(S, p, n0row, ncrows);
    if (have) {
      nslow = min(S.nslow, uint32_t(kSlowMax));
      if (nslow) {
        if (warp < kWDirectWarps) {
          for (uint32_t i = warp; i < nslow; i += kWDirectWarps) {
            const uint32_t r = S.slow[i];
            const uint64_t c = direct_row(p, A_ID, uint64_t(c0row) + r, dbits, dreach, &nnz_acc,
                                          [](uint64_t, uint32_t) {}, kWDirectWW);
            if (lane == 0) incl[r] = uint32_t(min(c, uint64_t(0xffffffffu)));
          }
        }
        cta_sync();
      }
      // chunk prefix over the row counts (kWRpt consecutive rows per thread:
      // a thread rewrites only its own rows) and the chunk's nnz
      {
        uint32_t loc[kWRpt];
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < kWRpt; ++k) {
          const uint32_t r = tid * kWRpt + k;
          s += r < crows ? incl[r] : 0u;
          loc[k] = uint32_t(s);
        }
        uint64_t inc = s;
        unsigned long long v = nnz_acc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint64_t u = __shfl_up_sync(kFullMask, inc, o);
          if (lane >= o) inc += u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
        if (lane == 31) S.red[warp] = inc;
        if (lane == 0) S.red_nnz[warp] = v;
        cta_sync();
        uint64_t wpre = 0;
        for (int i = 0; i < warp; ++i) wpre += S.red[i];
        const uint64_t excl = wpre + inc - s;
        if (excl + s > 0xffffffffull) raise_flag(p, &p.ctl->status, 16ull);
#pragma unroll
        for (int k = 0; k < kWRpt; ++k) {
          const uint32_t r = tid * kWRpt + k;
          if (r < crows) incl[r] = uint32_t(excl) + loc[k];
        }
      }
      cta_sync();
      for (int i = 0; i < kWarps; ++i) cnnz += S.red_nnz[i];
      cnt = incl[crows - 1];
      if (tid == 0) atomicAdd(&p.ctl->nnz, cnnz);
      staged = cnt <= p.stage_cap;
      // later chunks' look-backs wait on this word: published as soon as known
      if (staged && tid == 0) publish_aggregate(p, t, cnt);
    }
    if (pre) stage_rows_req_ranges<A_ID>(S, p, ncrows);
    if (staged) {
      // the chunk's image: every row's runs at its chunk-local offset
      uint32_t* img = stage + size_t(b) * (p.stage_cap + p.chunk_rows);
      for (uint32_t r = tid; r < crows; r += kThreads) img[p.stage_cap + r] = incl[r];
      write_rows(c0row, crows, nslow, img, p.stage_cap);
    }
    if (pre) stage_window_req_brows<A_ID>(S, p, n0row, ncrows);
    if (pend) {
      const uint32_t pend_t = S.pend_t[b ^ 1u], pend_crows = S.pend_crows[b ^ 1u];
      const unsigned long long pend_cnt = S.pend_cnt[b ^ 1u];
      const unsigned long long prefix = lookback_block(S, p, pend_t, pend_cnt, par);
      const uint32_t* img = stage + size_t(b ^ 1u) * (p.stage_cap + p.chunk_rows);
      // the pending chunk's row map: loads first, then stores (the staging
      // and the output may alias as far as the compiler knows)
      const uint32_t* pincl = img + p.stage_cap;
      const uint32_t p0row = pend_t * p.chunk_rows;
      {
        uint32_t v[kWRpt];
#pragma unroll
        for (int u = 0; u < kWRpt; ++u) {
          const uint32_t r = tid + u * kThreads;
          v[u] = r < pend_crows ? __ldcg(pincl + r) : 0u;
        }
#pragma unroll
        for (int u = 0; u < kWRpt; ++u) {
          const uint32_t r = tid + u * kThreads;
          if (r < pend_crows) p.c_rowmap[uint64_t(p0row) + r + 1] = prefix + v[u];
        }
      }
      if (pend_t == 0 && tid == 0) p.c_rowmap[0] = 0;
      // the pending chunk's image: one coalesced copy
      if (prefix + pend_cnt <= p.cap) {
        uint32_t* dst = p.c_entries + prefix;
        constexpr int kBatch = 8;
        for (uint64_t k0 = 0; k0 < pend_cnt; k0 += uint64_t(kBatch) * kThreads) {
          uint32_t v[kBatch];
#pragma unroll
          for (int u = 0; u < kBatch; ++u) {
            const uint64_t k = k0 + tid + uint64_t(u) * kThreads;
            v[u] = k < pend_cnt ? __ldcg(img + k) : 0u;
          }
#pragma unroll
          for (int u = 0; u < kBatch; ++u) {
            const uint64_t k = k0 + tid + uint64_t(u) * kThreads;
            if (k < pend_cnt) dst[k] = v[u];
          }
        }
      } else if (tid == 0 && pend_cnt) {
        raise_flag(p, &p.ctl->overflow, 1ull);
      }
      pend = false;
    }
    if (pre) stage_brows_req_branges(S, p);
    // a counted chunk whose image does not fit the staging: written in place
    if (have && !staged) {
      if (tid == 0) publish_aggregate(p, t, cnt);
      const unsigned long long pfx = lookback_block(S, p, t, cnt, par);
      for (uint32_t r = tid; r < crows; r += kThreads) p.c_rowmap[uint64_t(c0row) + r + 1] = pfx + incl[r];
      if (t == 0 && tid == 0) p.c_rowmap[0] = 0;
      write_rows(c0row, crows, nslow, p.c_entries + pfx, p.cap > pfx ? p.cap - pfx : 0ull);
    }
    if (tid == 0 && staged) {  // the image just written, in buffer b
      S.pend_t[b] = t;
      S.pend_crows[b] = crows;
      S.pend_cnt[b] = cnt;
    }
    if (staged) {
      pend = true;
      b ^= 1u;
    }
    // the next chunk; every warp must have passed the same barriers
    ++iter;
    if (lane == 0) S.phase[warp] = iter;
    if (tid == 0) {
      S.nslow = 0;
      S.ngen = 0;
    }
    cta_sync();
    if (warp == 0) {  // one read per lane, one vote
      const bool off = lane < kWarps && S.phase[lane] != iter;
      if (__any_sync(kFullMask, off) && lane == 0) raise_flag(p, &p.ctl->status, 64ull);
    }
    t = have ? tn : 0xffffffffu;
  }
  cp_async_wait();  // nothing may land after the CTA has exited
}

}  // namespace

uint32_t window_resident(dvg_context* ctx) {
  if (ctx->win_resident == 0) {
    const int smem = int(sizeof(WinSmem));
    for (void* k : {reinterpret_cast<void*>(&k_spgemm_window<false>), reinterpret_cast<void*>(&k_spgemm_window<true>)})
      DVG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    DVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<void*>(&k_spgemm_window<false>),
                                                           kThreads, smem));
    if (per_sm < 1) throw Error(DVG_ERR_DEVICE, "window spgemm: shared memory layout does not fit");
    ctx->win_resident = uint32_t(per_sm) * uint32_t(ctx->num_sms);
  }
  return ctx->win_resident;
}

void launch_rowmode_window(dvg_context* ctx, const RowLaunch& L, const RowLaunchShape& s) {
  if (L.nrows == 0) return;
  window_resident(ctx);  // sets the kernels' shared-memory attribute
  FusedArgs p{};
  p.a_rowmap = L.a_identity ? nullptr : L.a_rowmap;
  p.a_entries = L.a_identity ? nullptr : L.a_entries;
  p.b_rowmap = L.b_rowmap;
  p.b_entries = L.b_entries;
  p.c_rowmap = L.c_rowmap;
  p.c_entries = L.c_entries;
  p.cap = L.cap;
  p.desc = static_cast<ChunkDesc*>(L.desc);
  p.ticket = L.ticket;
  p.ctl = L.ctl;
  p.nrows = L.nrows;
  p.chunk_rows = s.chunk_rows;
  p.nchunks = s.nchunks;
  p.row_mode = 1;
  p.d_rowmap = L.d_identity ? nullptr : L.d_rowmap;
  p.d_entries = L.d_identity ? nullptr : L.d_entries;
  p.d_identity = L.d_identity ? 1u : 0u;
  p.abort = L.abort;
  p.stage_buf = L.stage_buf;
  p.stage_cap = L.stage_buf ? uint32_t(kWRowStagePerRow) * s.chunk_rows : 0u;
  p.a_shift = L.a_identity ? L.a_shift : 0u;
  p.b_nrows = L.b_nrows;
  p.nlevels = L.nlevels;
  for (uint32_t k = 0; k < L.nlevels && k < uint32_t(kMaxLevels); ++k) {
    p.lv_rowmap[k] = L.lv_rowmap[k];
    p.lv_entries[k] = L.lv_entries[k];
  }
  const int smem = int(sizeof(WinSmem));
  if (L.a_identity) k_spgemm_window<true><<<s.grid, kThreads, smem, ctx->stream>>>(p);
  else k_spgemm_window<false><<<s.grid, kThreads, smem, ctx->stream>>>(p);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
  ctx->stats.spgemm_light++;
  ctx->stats.spgemm_window++;
}

}  // namespace dvg
