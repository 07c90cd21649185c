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
// Rows are walked twice from shared memory: once to count (runs, nnz), once,
// after the chunk's prefix, to emit the runs into the chunk's image -- the
// operands are on chip, so recomputing is cheaper than keeping every row's
// runs (the other kernel's run-list slots).  A row's closed runs sit in a
// 4-run list in shared memory while it is walked; rows with more runs take
// the warp-cooperative path.  Output order, deferred write-out through per-CTA
// staging buffers, the CTA-wide decoupled look-back, bounded waits, the abort
// word of planned builds and every self-check are those of k_spgemm_rowmode.
#include <algorithm>

#include "dvg_spgemm_common.cuh"

namespace dvg {
namespace {

constexpr int kWRows = kChunkMax;          // rows per chunk (upper bound)
constexpr int kWRpt = kWRows / kThreads;   // rows per thread at the largest chunk
constexpr int kWAEnt = 2048;               // A ranges staged per chunk
constexpr int kWDEnt = 2048;               // addend ranges staged per chunk
constexpr int kWBRows = 2559;              // B rows in the staged window (at most)
constexpr int kWBEnt = 2560;               // B ranges staged per chunk
constexpr int kWList = 8;                  // run-list entries per thread (four closed runs)
constexpr int kWDirectWarps = 4;           // warps that run the warp path
constexpr int kWDirectWW = 192;            // warp path: 32-bit window words per warp
constexpr int kWRowStagePerRow = 16;       // image entries per chunk row, as the staging buffers are sized

// Shared memory of one CTA.  The two 64-bit row-pointer runs of the next
// chunk land in `bent` + `list` (adjacent) before they are compacted to
// 32 bits, and the B window's row pointers land in `bent` before the B
// ranges do: those arrays are free while a chunk is being staged.
struct WinSmem {
  uint2 aent[kWAEnt];     // the chunk's A ranges (from abase on)
  uint2 dent[kWDEnt];     // the chunk's addend ranges (from dbase on)
  uint2 bent[kWBEnt];     // the B window's ranges (from bbase on)
  uint32_t list[kWList * kThreads];  // closed runs of the row in hand: entry k of thread t at [k * kThreads + t]
  // low 32 bits of range offsets (rowmap / 2): A and addend rows c0 .. c0 + crows,
  // B rows wlo .. whi + 1; row r spans [x[r] - x[0], x[r + 1] - x[0]) of its stage
  uint32_t arow[kWRows + 1];
  uint32_t drow[kWRows + 1];
  uint32_t brow[kWBRows + 1];
  uint32_t incl[kWRows];      // the counted chunk's (then chunk-local inclusive) row counts
  uint32_t slow[kSlowMax];    // rows of the counted chunk left to the warp path
  uint32_t direct[2 * kWDirectWW * kWDirectWarps];  // warp path: bits + reach per warp
  unsigned long long red[kWarps];
  unsigned long long red_nnz[kWarps];
  unsigned long long lb_sum[2][kWarps];  // look-back records by round parity, per warp
  uint32_t lb_flag[2][kWarps];
  uint32_t phase[kWarps];                // iterations per warp, checked at every iteration's end
  uint32_t wmin[kWarps], wmax[kWarps];   // per-warp bounds of the chunk's A ranges
  unsigned long long abase, dbase, bbase;  // 64-bit range offset of each stage's first range
  unsigned long long pend_cnt;           // the staged chunk waiting in buffer b ^ 1
  uint32_t na, nd, nb;                   // ranges staged
  uint32_t rows_ok;                      // bit 0: arow usable, bit 1: drow usable
  uint32_t wlo, wn;                      // staged B rows [wlo, wlo + wn)
  uint32_t wn_req;                       // B rows whose row pointers were requested (from wlo)
  uint32_t pend_t, pend_crows;
  uint32_t next;                         // the chunk taken for the next iteration
  uint32_t nslow;
};
static_assert(sizeof(WinSmem) <= 115712, "two CTAs per SM must fit");
static_assert(offsetof(WinSmem, list) == offsetof(WinSmem, bent) + sizeof(uint2) * kWBEnt, "bent, list adjacent");
static_assert(sizeof(uint2) * kWBEnt + sizeof(uint32_t) * kWList * kThreads >= 2 * 8 * (kWRows + 1),
              "the next chunk's row pointers fit bent + list");
static_assert(sizeof(uint2) * kWBEnt >= 8 * (kWBRows + 1), "the B window's row pointers fit bent");

// ---- staging ------------------------------------------------------------------
// Four phases, each ended by the next one's wait: (1) request the chunk's A
// and addend row pointers; (2) compact them, request the A and addend ranges;
// (3) bound the B rows the staged A ranges name, request their row pointers;
// (4) clip the window to the B-range capacity, compact, request the B ranges.
// Every phase is called by the whole CTA (uniform branches).

template <bool A_ID>
__device__ void stage_req_rows(WinSmem& S, const FusedArgs& p, uint32_t c0row, uint32_t crows) {
  uint64_t* rawA = reinterpret_cast<uint64_t*>(S.bent);
  uint64_t* rawD = rawA + (kWRows + 1);
  for (uint32_t k = threadIdx.x; k <= crows; k += kThreads) {
    if (!A_ID) cp_async8(rawA + k, p.a_rowmap + uint64_t(c0row) + k);
    if (p.d_rowmap) cp_async8(rawD + k, p.d_rowmap + uint64_t(c0row) + k);
  }
  cp_async_commit();
}

template <bool A_ID>
__device__ void stage_rows_req_ranges(WinSmem& S, const FusedArgs& p, uint32_t crows) {
  const uint64_t* rawA = reinterpret_cast<const uint64_t*>(S.bent);
  const uint64_t* rawD = rawA + (kWRows + 1);
  cp_async_wait();
  cta_sync();
  for (uint32_t k = threadIdx.x; k <= crows; k += kThreads) {
    if (!A_ID) S.arow[k] = uint32_t(rawA[k] >> 1);
    if (p.d_rowmap) S.drow[k] = uint32_t(rawD[k] >> 1);
  }
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
  const uint32_t na = uint32_t(min(na64, uint64_t(kWAEnt)));
  const uint32_t nd = uint32_t(min(nd64, uint64_t(kWDEnt)));
  if (threadIdx.x == 0) {
    S.abase = abase;
    S.dbase = dbase;
    S.na = na;
    S.nd = nd;
    // 32-bit row offsets hold while a chunk's ranges stay below 2^31
    S.rows_ok = (na64 < (1ull << 31) ? 1u : 0u) | (nd64 < (1ull << 31) ? 2u : 0u);
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
  for (uint32_t k = tid; k <= wn && wn; k += kThreads) S.brow[k] = uint32_t(raw[k] >> 1);
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

// Walks C row `row` (chunk row r) from the stages (HBM for what is not
// staged) into the thread's run list.  EMIT = false: count = entries of the
// row, nnz accumulated; returns false, leaving no trace in nnz, when the runs
// overflow the list.  EMIT = true: writes the row's `n` entries to out[0..n)
// and returns false if the row does not have exactly n.
template <bool A_ID, bool EMIT>
__device__ bool win_row(WinSmem& S, const FusedArgs& p, uint64_t row, uint32_t r, uint32_t& count,
                        unsigned long long& nnz, uint32_t* out, uint32_t n_out) {
  uint32_t* L = S.list + threadIdx.x;  // run k: lo at L[2k*kT], hi at L[(2k+1)*kT]
  constexpr uint32_t max_runs = kWList / 2;
  uint32_t nr = 0;
  // merges [x, y] into the list; false when it needs more runs than fit
  auto merge = [&](uint32_t x, uint32_t y) -> bool {
    uint32_t k = 0;
    while (k < nr && uint64_t(L[(2 * k + 1) * kThreads]) + 1 < x) ++k;
    if (k == nr || uint64_t(y) + 1 < L[2 * k * kThreads]) {
      if (nr == max_runs) return false;
      for (uint32_t m = nr; m > k; --m) {
        L[2 * m * kThreads] = L[2 * (m - 1) * kThreads];
        L[(2 * m + 1) * kThreads] = L[(2 * m - 1) * kThreads];
      }
      L[2 * k * kThreads] = x;
      L[(2 * k + 1) * kThreads] = y;
      ++nr;
      return true;
    }
    uint32_t lo = min(L[2 * k * kThreads], x), hi = max(L[(2 * k + 1) * kThreads], y);
    uint32_t m = k + 1;
    while (m < nr && uint64_t(hi) + 1 >= L[2 * m * kThreads]) {
      hi = max(hi, L[(2 * m + 1) * kThreads]);
      ++m;
    }
    L[2 * k * kThreads] = lo;
    L[(2 * k + 1) * kThreads] = hi;
    const uint32_t gone = m - k - 1;
    if (gone) {
      for (uint32_t q = m; q < nr; ++q) {
        L[2 * (q - gone) * kThreads] = L[2 * q * kThreads];
        L[(2 * (q - gone) + 1) * kThreads] = L[(2 * q + 1) * kThreads];
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
      d0 = S.drow[r] - S.drow[0];
      d1 = S.drow[r + 1] - S.drow[0];
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
      a0 = S.arow[r] - S.arow[0];
      a1 = S.arow[r + 1] - S.arow[0];
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
      const uint32_t t0 = S.brow[ar.x - wlo] - S.brow[0], t1 = S.brow[ar.y + 1 - wlo] - S.brow[0];
      for (uint32_t t = t0; t < t1; ++t)
        if (!take(S.bent[t])) return false;
    } else {
      const uint64_t t0 = __ldg(p.b_rowmap + ar.x) >> 1, t1 = __ldg(p.b_rowmap + uint64_t(ar.y) + 1) >> 1;
      for (uint64_t t = t0; t < t1; ++t)
        if (!take(load_range(p.b_entries, t))) return false;
    }
  }
  if (any && !merge(run_lo, run_hi)) return false;
  if (EMIT) {
    if (2 * nr != n_out) return false;
    for (uint32_t k = 0; k < nr; ++k) {
      out[2 * k] = L[2 * k * kThreads];
      out[2 * k + 1] = L[(2 * k + 1) * kThreads];
    }
  } else {
    uint64_t n = 0;
    for (uint32_t k = 0; k < nr; ++k) n += uint64_t(L[(2 * k + 1) * kThreads]) - L[2 * k * kThreads] + 1;
    count = 2 * nr;
    nnz += n;
  }
  return true;
}

// ---- the kernel --------------------------------------------------------------------
// With rpt = ceil(chunk_rows / kThreads) rows per thread, thread (warp, lane)
// owns chunk rows (warp * rpt + u) * 32 + lane, u < rpt: the lanes of a warp
// take consecutive rows.  An iteration counts chunk t (staged), takes its
// prefix, writes its image to staging buffer b (or, when it does not fit,
// resolves it in place), and resolves the chunk staged one iteration before
// while the next chunk's operands are requested.
template <bool A_ID>
__global__ void __launch_bounds__(kThreads, 2) k_spgemm_window(FusedArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WinSmem& S = *reinterpret_cast<WinSmem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* dbits = S.direct + size_t(warp < kWDirectWarps ? warp : 0) * 2 * kWDirectWW;
  uint32_t* dreach = dbits + kWDirectWW;
  const uint32_t rpt = (p.chunk_rows + kThreads - 1) / kThreads;  // 1..kWRpt
  // per CTA two buffers: a chunk's image (stage_cap entries), then its
  // chunk-local inclusive row counts (chunk_rows words)
  uint32_t* const stage =
      p.stage_buf ? p.stage_buf + size_t(blockIdx.x) * 2 * (p.stage_cap + p.chunk_rows) : nullptr;
  // a planned build stops at the first step whose output is unusable
  auto take_ticket = [&]() -> uint32_t {
    const bool stop = p.abort && *reinterpret_cast<volatile unsigned long long*>(p.abort) != 0;
    return stop ? 0xffffffffu : atomicAdd(p.ticket, 1u);
  };
  if (tid == 0) {
    S.next = take_ticket();
    S.nslow = 0;
  }
  cta_sync();
  uint32_t t = S.next, b = 0, par = 0;
  bool pend = false;  // a staged chunk waits in buffer b ^ 1 (described in S.pend_*)
  if (t < p.nchunks) stage_chunk<A_ID>(S, p, t);
  uint32_t iter = 0;
  while (t < p.nchunks || pend) {
    const bool have = t < p.nchunks;
    // the stage of chunk t may still be landing (requested last iteration)
    cp_async_wait();
    cta_sync();
    const bool stop = tid == 0 && p.abort && *reinterpret_cast<volatile unsigned long long*>(p.abort) != 0;
    uint32_t next = 0xffffffffu;
    const uint32_t c0row = have ? t * p.chunk_rows : 0u;
    const uint32_t crows = have ? min(p.chunk_rows, p.nrows - c0row) : 0u;
    uint32_t* const incl = S.incl;
    unsigned long long nnz_acc = 0, cnt = 0, cnnz = 0;
    uint32_t fast_mask = 0, nslow = 0, nslow_all = 0;
    bool staged = false;
    if (have) {
      // count: every row from the stages
#pragma unroll 1
      for (int u = 0; u < kWRpt; ++u) {
        if (uint32_t(u) >= rpt) break;
        const uint32_t r = (warp * rpt + u) * 32 + lane;
        if (r < crows) {
          uint32_t c = 0;
          if (win_row<A_ID, false>(S, p, uint64_t(c0row) + r, r, c, nnz_acc, nullptr, 0)) {
            fast_mask |= 1u << u;
          } else {
            const uint32_t i = atomicAdd(&S.nslow, 1u);
            if (i < uint32_t(kSlowMax)) {
              S.slow[i] = r;
            } else {
              c = light_row<A_ID>(nullptr, nullptr, p, c0row, r, false, &nnz_acc, [](uint64_t, uint32_t) {});
            }
            atomicAdd(&p.ctl->slow_rows, 1ull);
          }
          incl[r] = c;
        }
      }
      cta_sync();
      if (tid == 0 && !stop) next = atomicAdd(p.ticket, 1u);
      nslow_all = S.nslow;
      nslow = min(nslow_all, uint32_t(kSlowMax));
      if (warp < kWDirectWarps) {
        for (uint32_t i = warp; i < nslow; i += kWDirectWarps) {
          const uint32_t r = S.slow[i];
          const uint64_t c = direct_row(p, A_ID, uint64_t(c0row) + r, dbits, dreach, &nnz_acc,
                                        [](uint64_t, uint32_t) {}, kWDirectWW);
          if (lane == 0) incl[r] = uint32_t(min(c, uint64_t(0xffffffffu)));
        }
      }
      cta_sync();
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
      staged = stage != nullptr && cnt <= p.stage_cap;
      if (staged) {
        // the chunk's image: every row walked again, runs at its chunk-local offset
        uint32_t* img = stage + size_t(b) * (p.stage_cap + p.chunk_rows);
        if (tid == 0) publish_aggregate(p, t, cnt);
        for (uint32_t r = tid; r < crows; r += kThreads) img[p.stage_cap + r] = incl[r];
#pragma unroll 1
        for (int u = 0; u < kWRpt; ++u) {
          if (uint32_t(u) >= rpt) break;
          const uint32_t r = (warp * rpt + u) * 32 + lane;
          if (r >= crows || !((fast_mask >> u) & 1u)) continue;
          const uint32_t o = r ? incl[r - 1] : 0u;
          const uint32_t n = incl[r] - o;
          uint32_t c = 0;
          unsigned long long z = 0;
          if (!win_row<A_ID, true>(S, p, uint64_t(c0row) + r, r, c, z, img + o, n))
            raise_flag(p, &p.ctl->status, 8ull);
        }
        if (warp < kWDirectWarps) {
          for (uint32_t i = warp; i < nslow; i += kWDirectWarps) {
            const uint32_t r = S.slow[i];
            const uint32_t o = r ? incl[r - 1] : 0u;
            const uint32_t n = incl[r] - o;
            if (n == 0) continue;
            bool bad = false;
            const uint64_t c = direct_row(p, A_ID, uint64_t(c0row) + r, dbits, dreach, nullptr,
                                          [&](uint64_t k, uint32_t v) {
                                            if (k < n) img[o + k] = v;
                                            else bad = true;
                                          },
                                          kWDirectWW);
            if (bad || c != n) raise_flag(p, &p.ctl->status, 8ull);
          }
        }
        if (nslow_all > uint32_t(kSlowMax)) {
#pragma unroll 1
          for (int u = 0; u < kWRpt; ++u) {
            if (uint32_t(u) >= rpt) break;
            const uint32_t r = (warp * rpt + u) * 32 + lane;
            if (r >= crows || ((fast_mask >> u) & 1u)) continue;
            bool listed = false;
            for (uint32_t i = 0; i < nslow && !listed; ++i) listed = S.slow[i] == r;
            if (listed) continue;
            const uint32_t o = r ? incl[r - 1] : 0u;
            const uint32_t n = incl[r] - o;
            if (n == 0) continue;
            const uint32_t c = light_row<A_ID>(nullptr, nullptr, p, c0row, r, false, nullptr,
                                               [&](uint64_t k, uint32_t v) {
                                                 if (k < n) img[o + k] = v;
                                               });
            if (c != n) raise_flag(p, &p.ctl->status, 8ull);
          }
        }
      }
    }
    if (tid == 0) S.next = next;
    // every thread is done with the stages, the run lists, the slow list and
    // the counted chunk's image
    cta_sync();
    const uint32_t tn = S.next;
    // after a staged chunk the stages are free: the next chunk's operands
    // are requested phase by phase between the steps of the pending
    // chunk's write-out, so both latencies overlap
    const bool pre = have && staged && tn < p.nchunks;
    const uint32_t n0row = pre ? tn * p.chunk_rows : 0u;
    const uint32_t ncrows = pre ? min(p.chunk_rows, p.nrows - n0row) : 0u;
    if (pre) stage_req_rows<A_ID>(S, p, n0row, ncrows);
    unsigned long long prefix = 0;
    uint32_t pend_t = 0, pend_crows = 0;
    unsigned long long pend_cnt = 0;
    const uint32_t* img = nullptr;
    if (pend) {
      pend_t = S.pend_t;
      pend_crows = S.pend_crows;
      pend_cnt = S.pend_cnt;
      prefix = lookback_block(S, p, pend_t, pend_cnt, par);
      img = stage + size_t(b ^ 1u) * (p.stage_cap + p.chunk_rows);
    }
    if (pre) stage_rows_req_ranges<A_ID>(S, p, ncrows);
    if (pend) {
      // the pending chunk's row map: loads first, then stores (the staging
      // and the output may alias as far as the compiler knows)
      const uint32_t* pincl = img + p.stage_cap;
      const uint32_t p0row = pend_t * p.chunk_rows;
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
      if (pend_t == 0 && tid == 0) p.c_rowmap[0] = 0;
    }
    if (pre) stage_window_req_brows<A_ID>(S, p, n0row, ncrows);
    if (pend) {
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
    // a counted chunk that was not staged is resolved now, in place, from its
    // stages (nothing was requested over them)
    if (have && !staged) {
      if (tid == 0) publish_aggregate(p, t, cnt);
      const unsigned long long pfx = lookback_block(S, p, t, cnt, par);
      for (uint32_t r = tid; r < crows; r += kThreads) p.c_rowmap[uint64_t(c0row) + r + 1] = pfx + incl[r];
      if (t == 0 && tid == 0) p.c_rowmap[0] = 0;
#pragma unroll 1
      for (int u = 0; u < kWRpt; ++u) {
        if (uint32_t(u) >= rpt) break;
        const uint32_t r = (warp * rpt + u) * 32 + lane;
        if (r >= crows || !((fast_mask >> u) & 1u)) continue;
        const unsigned long long dst = pfx + (r ? incl[r - 1] : 0u);
        const uint32_t n = incl[r] - (r ? incl[r - 1] : 0u);
        if (n && dst + n > p.cap) {
          raise_flag(p, &p.ctl->overflow, 1ull);
          continue;
        }
        uint32_t c = 0;
        unsigned long long z = 0;
        if (!win_row<A_ID, true>(S, p, uint64_t(c0row) + r, r, c, z, p.c_entries + dst, n))
          raise_flag(p, &p.ctl->status, 8ull);
      }
      if (warp < kWDirectWarps) {
        for (uint32_t i = warp; i < nslow; i += kWDirectWarps) {
          const uint32_t r = S.slow[i];
          const unsigned long long dst = pfx + (r ? incl[r - 1] : 0u);
          const uint32_t n = incl[r] - (r ? incl[r - 1] : 0u);
          if (n == 0 || dst + n > p.cap) continue;
          uint32_t* out = p.c_entries + dst;
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
      if (nslow_all > uint32_t(kSlowMax)) {
#pragma unroll 1
        for (int u = 0; u < kWRpt; ++u) {
          if (uint32_t(u) >= rpt) break;
          const uint32_t r = (warp * rpt + u) * 32 + lane;
          if (r >= crows || ((fast_mask >> u) & 1u)) continue;
          bool listed = false;
          for (uint32_t i = 0; i < nslow && !listed; ++i) listed = S.slow[i] == r;
          if (listed) continue;
          const unsigned long long dst = pfx + (r ? incl[r - 1] : 0u);
          const uint32_t n = incl[r] - (r ? incl[r - 1] : 0u);
          if (n == 0 || dst + n > p.cap) continue;
          uint32_t* out = p.c_entries + dst;
          const uint32_t c = light_row<A_ID>(nullptr, nullptr, p, c0row, r, false, nullptr,
                                             [&](uint64_t k, uint32_t v) {
                                               if (k < n) out[k] = v;
                                             });
          if (c != n) raise_flag(p, &p.ctl->status, 8ull);
        }
      }
      cta_sync();  // the stages are read until here
    }
    // the next chunk was not requested above: stage it now, whole
    if (!pre && tn < p.nchunks) stage_chunk<A_ID>(S, p, tn);
    if (staged) {
      pend = true;
      b ^= 1u;
    }
    // the next chunk; every warp must have passed the same barriers
    ++iter;
    if (lane == 0) S.phase[warp] = iter;
    if (tid == 0) {
      if (staged) {
        S.pend_t = t;
        S.pend_crows = crows;
        S.pend_cnt = cnt;
      }
      S.nslow = 0;
    }
    cta_sync();
    if (warp == 0) {  // one read per lane, one vote
      const bool off = lane < kWarps && S.phase[lane] != iter;
      if (__any_sync(kFullMask, off) && lane == 0) raise_flag(p, &p.ctl->status, 64ull);
    }
    t = tn;
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
