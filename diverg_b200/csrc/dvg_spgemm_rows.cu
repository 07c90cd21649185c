// dvg_spgemm_rows.cu -- single-pass range SpGEMM, one C row per thread:
// C = A B or C = D + A B (D a matrix of C's shape, or the identity).
//
// Same result as the reference's symbolic + numeric SpGEMM
// (include/diverg/range_sparse.hpp:1132-1442 in cartoonist/diverg, dispatched
// by range_spgemm :2215-2281) followed, for the sums, by range_spadd
// (:112-357) on canonical operands: row r of C is the union of D's row r and
// of all ranges of B rows s..f for every range [s,f] of A's row r, emitted as
// sorted maximal runs.
//
// For the products of an index build the rows of C are a handful of runs,
// however wide: the union is accumulated as a sorted list of disjoint,
// non-adjacent runs -- exactly the canonical output -- held in the thread's
// output slot in shared memory.  A range that overlaps or touches the open run
// (kept in registers) extends it; any other range first merges the open run
// into the list (insert, or merge with the runs it overlaps or touches: start
// <= hi + 1, as the reference's accumulators merge).  The cost is output
// sensitive and independent of the row's column span.  The shared footprint
// is small (the slots, the chunk's row counts and the warp path's window), so
// most of the SM's L1 caches the B ranges the threads read: the lanes of a
// warp take consecutive rows, whose B slices overlap, and neighbouring warps
// cover neighbouring rows.
//
// The kernel is persistent: CTAs take chunks of consecutive rows from an
// atomic ticket; a chunk's rows are counted (runs into the slots), rows whose
// runs overflow the slot are deferred to a warp-cooperative bitvector path, a
// warp-parallel decoupled look-back over the chunk order gives the chunk's
// output offset, and the slots are written out.  No symbolic pass, no scan
// kernel.  Look-back waits are bounded (a timeout is recorded on expiry).
#include <algorithm>
#include <mutex>

#include "dvg_spgemm_common.cuh"

namespace dvg {
namespace {

constexpr int kRowRowsMax = kChunkMax / kThreads;  // rows per thread at the largest chunk
constexpr int kRowDirectWW = 192;  // warp path: 32-bit window words per warp (6,144 columns)
constexpr int kAStage = 2048;      // A ranges of a chunk staged in shared memory
constexpr int kRowStagePerRow = 16;  // staged entries per chunk row (a chunk with more is written in place)
// general-walk list entries: the chunk row, and whether it went on to the
// warp path or (past kSlowMax of those) to the light path
constexpr uint32_t kGenRow = 0x0fffu, kGenWarp = 0x4000u, kGenLight = 0x8000u;
static_assert(kChunkMax <= int(kGenRow) + 1, "chunk rows must fit the general-walk list entries");

// The chunk's A row pointers and (up to kAStage of) its A ranges, loaded with
// coalesced reads before the rows are walked; the warp path's windows reuse
// the space once the rows have been counted.
struct AStage {
  uint64_t arow[kChunkMax + 1];
  uint2 aent[kAStage];
};
union RowScratch {
  uint32_t direct[2 * kRowDirectWW * kWarps];  // warp path: bits + reach per warp
  AStage a;
};

// Two chunks can be in flight per CTA: the one being counted (buffer b) and
// the previous one (buffer b ^ 1), counted and staged in global memory,
// waiting to be written out.
template <int SLOT>
struct RowSmem {
  uint32_t slot[SLOT * kThreads];       // entry k of thread t at [k * kThreads + t]
  RowScratch u;
  uint32_t incl[kChunkMax];             // the counted chunk's (then chunk-local inclusive) row counts
  uint32_t slow[kSlowMax];              // rows of the counted chunk left to the warp path
  uint16_t gen[kChunkMax];              // rows left to the general walk (| kGenWarp, kGenLight: how it ended)
  unsigned long long red[kWarps];
  unsigned long long red_nnz[kWarps];
  unsigned long long lb_sum[2][kWarps];  // look-back records by round parity, per warp
  uint32_t lb_flag[2][kWarps];
  uint32_t phase[kWarps];               // iterations per warp, checked at every iteration's end
  // the staged chunk waiting in image buffer k, kept per buffer: its readers
  // (the next iteration) and the writer of the next one (that iteration's
  // end, which a look-back of no rounds may not separate from them by a
  // barrier) never meet on one slot
  unsigned long long pend_cnt[2];
  uint32_t pend_t[2], pend_crows[2];
  uint32_t next;                        // the chunk taken for the next iteration
  uint32_t nslow;
  uint32_t ngen;
};

// Accumulates chunk row r (C row `row`) into the thread's slot from entry
// `pos` on.  A's row pointers come from the stage, its ranges from the stage
// when they are among the chunk's first kAStage ranges (abase: the chunk's
// first range, nst: the number staged).  Returns false, leaving no trace in
// nnz, when the runs overflow the slot.
template <bool A_ID, int SLOT>
__device__ bool row_runs(RowSmem<SLOT>& S, const FusedArgs& p, uint64_t row, uint32_t r, uint64_t abase,
                         uint32_t nst, uint32_t pos, uint32_t& count, unsigned long long& nnz) {
  uint32_t* L = S.slot + threadIdx.x + size_t(pos) * kThreads;  // run k: lo at L[2k*kT], hi at L[(2k+1)*kT]
  const uint32_t max_runs = (uint32_t(SLOT) - pos) >> 1;
  uint64_t a0, a1;
  if (A_ID) {
    a0 = 0;
    a1 = 1;
  } else {
    a0 = S.u.a.arow[r] >> 1;
    a1 = S.u.a.arow[r + 1] >> 1;
  }
  auto a_range = [&](uint64_t k) -> uint2 {
    if (A_ID) return id_range(p, row);
    return k - abase < nst ? S.u.a.aent[k - abase] : load_range(p.a_entries, k);
  };
  // an A range of at least 4 rows reads union levels when B has them
  auto leveled = [&](uint2 ar) { return p.nlevels && ar.y >= ar.x && ar.y - ar.x >= 3u; };
  // the first A range's B row pointers are requested before the addend is
  // walked, so their latency overlaps it
  uint2 ar0 = make_uint2(1, 0);
  uint64_t tb0 = 0, tb1 = 0;
  if (a0 < a1) {
    ar0 = a_range(a0);
    if (ar0.x <= ar0.y && !leveled(ar0)) {
      tb0 = __ldg(p.b_rowmap + ar0.x) >> 1;
      tb1 = __ldg(p.b_rowmap + uint64_t(ar0.y) + 1) >> 1;
    }
  }
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
  if (p.d_identity) {
    take(make_uint2(uint32_t(row), uint32_t(row)));
  } else if (p.d_rowmap) {
    const uint64_t d0 = __ldg(p.d_rowmap + row) >> 1, d1 = __ldg(p.d_rowmap + row + 1) >> 1;
    for (uint64_t t = d0; t < d1; ++t)
      if (!take(load_range(p.d_entries, t))) return false;
  }
  for (uint64_t k = a0; k < a1; ++k) {
    const uint2 ar = k == a0 ? ar0 : a_range(k);
    if (ar.y < ar.x) continue;
    if (leveled(ar)) {
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
    uint64_t t0 = tb0, t1 = tb1;
    if (k != a0) {
      t0 = __ldg(p.b_rowmap + ar.x) >> 1;
      t1 = __ldg(p.b_rowmap + uint64_t(ar.y) + 1) >> 1;
    }
    for (uint64_t t = t0; t < t1; ++t)
      if (!take(load_range(p.b_entries, t))) return false;
  }
  if (any && !merge(run_lo, run_hi)) return false;
  uint64_t n = 0;
  for (uint32_t k = 0; k < nr; ++k) n += uint64_t(L[(2 * k + 1) * kThreads]) - L[2 * k * kThreads] + 1;
  count = 2 * nr;
  nnz += n;
  return true;
}

// The union of at most two ranges (an empty one has y < x) into the slot at
// `pos`: one run, or two when they neither overlap nor touch.  Columns are
// below 2^32 - 2, so hi + 1 does not wrap.  False when the runs do not fit.
template <int SLOT>
__device__ __forceinline__ bool two_ranges(RowSmem<SLOT>& S, uint2 x, uint2 y, uint32_t pos, uint32_t& count,
                                           unsigned long long& nnz) {
  if (x.y < x.x) x = y;
  if (y.y < y.x) y = x;
  if (y.x < x.x) {
    const uint2 s = x;
    x = y;
    y = s;
  }
  uint32_t nr = 0;
  if (x.x <= x.y) nr = y.x <= x.y + 1 ? 1u : 2u;
  if (nr > (uint32_t(SLOT) - pos) >> 1) return false;
  uint32_t* L = S.slot + threadIdx.x + size_t(pos) * kThreads;
  uint64_t n = 0;
  if (nr == 1) x.y = max(x.y, y.y);
  if (nr) {
    L[0] = x.x;
    L[kThreads] = x.y;
    n = uint64_t(x.y) - x.x + 1;
  }
  if (nr == 2) {
    L[2 * kThreads] = y.x;
    L[3 * kThreads] = y.y;
    n += uint64_t(y.y) - y.x + 1;
  }
  count = 2 * nr;
  nnz += n;
  return true;
}

// The row kernel.  With rpt = ceil(chunk_rows / kThreads) rows per thread,
// thread (warp, lane) owns chunk rows (warp * rpt + u) * 32 + lane, u < rpt:
// the lanes of a warp take consecutive rows.
//
// An iteration counts chunk t into buffer b: stage A, walk the rows into the
// slots, count the rows that missed the slots on the warp path, the
// chunk-local prefix.  When the CTA has a staging area (p.stage_buf) and the
// chunk's runs fit it, the iteration publishes t's aggregate and writes the
// chunk's complete image -- every row's runs at its chunk-local offset -- to
// staging buffer b, and resolves t one iteration later: by then the chunks
// before it have long published their aggregates, so the look-back rarely
// waits, and the write-out is the row map plus one coalesced copy.  Any
// other chunk is resolved in its own iteration (look-back, then rows written
// in place).  Every barrier of the loop is reached by the whole CTA.
template <bool A_ID, int SLOT>
__global__ void __launch_bounds__(kThreads, 2) k_spgemm_rowmode(FusedArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RowSmem<SLOT>& S = *reinterpret_cast<RowSmem<SLOT>*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* dbits = S.u.direct + size_t(warp) * 2 * kRowDirectWW;
  uint32_t* dreach = dbits + kRowDirectWW;
  const uint32_t rpt = (p.chunk_rows + kThreads - 1) / kThreads;  // 1..kRowRowsMax
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
    S.ngen = 0;
  }
  cta_sync();
  uint32_t t = S.next, b = 0, par = 0;
  bool pend = false;  // a staged chunk waits in buffer b ^ 1 (described in S.pend_*)
  bool pre = false;   // the A stage of chunk t was requested during the previous iteration
  // the asynchronous stage copies 8-byte words
  const bool a_async = !A_ID && ((reinterpret_cast<uintptr_t>(p.a_rowmap) | reinterpret_cast<uintptr_t>(p.a_entries)) & 7u) == 0;
  uint32_t iter = 0;
  // Writes the counted chunk's rows at out + their chunk-local offsets, where
  // `room` entries fit: the common rows from their owners' slots, the general
  // rows from their walkers' slots (light-path rows recomputed by their
  // walkers), the warp-path rows recomputed by the warps.  Rows past `room`
  // are skipped (and, with flag, reported as an overflow).
  auto write_rows = [&](uint32_t* out, unsigned long long room, bool flag, uint32_t c0row, uint32_t crows,
                        uint32_t fast_mask, uint32_t ngen, uint32_t nslow) {
    const uint32_t* incl = S.incl;
    uint32_t spos = 0;
#pragma unroll 1
    for (int u = 0; u < kRowRowsMax; ++u) {
      if (uint32_t(u) >= rpt) break;
      const uint32_t r = (warp * rpt + u) * 32 + lane;
      if (r >= crows || !((fast_mask >> u) & 1u)) continue;
      const uint32_t o = r ? incl[r - 1] : 0u;
      const uint32_t n = incl[r] - o;
      if (uint64_t(o) + n <= room) {
        // a run (two entries at an even offset) a store
        for (uint32_t k = 0; k < n; k += 2)
          *reinterpret_cast<uint2*>(out + o + k) =
              make_uint2(S.slot[(spos + k) * kThreads + tid], S.slot[(spos + k + 1) * kThreads + tid]);
      } else if (flag && n) {
        raise_flag(p, &p.ctl->overflow, 1ull);
      }
      spos += n;
    }
    for (uint32_t i = uint32_t(lane) * kWarps + warp; i < ngen; i += kThreads) {
      const uint32_t e = S.gen[i], r = e & kGenRow;
      if (e & kGenWarp) continue;
      const uint32_t o = r ? incl[r - 1] : 0u;
      const uint32_t n = incl[r] - o;
      if (uint64_t(o) + n > room) {
        if (flag && n) raise_flag(p, &p.ctl->overflow, 1ull);
      } else if (e & kGenLight) {
        uint32_t* dst = out + o;
        const uint32_t c = light_row<A_ID>(nullptr, nullptr, p, c0row, r, false, nullptr,
                                           [&](uint64_t k, uint32_t v) {
                                             if (k < n) dst[k] = v;
                                           });
        if (c != n) raise_flag(p, &p.ctl->status, 8ull);
      } else {
        for (uint32_t k = 0; k < n; k += 2)
          *reinterpret_cast<uint2*>(out + o + k) =
              make_uint2(S.slot[(spos + k) * kThreads + tid], S.slot[(spos + k + 1) * kThreads + tid]);
      }
      if (!(e & kGenLight)) spos += n;
    }
    for (uint32_t i = warp; i < nslow; i += kWarps) {
      const uint32_t r = S.slow[i];
      const uint32_t o = r ? incl[r - 1] : 0u;
      const uint32_t n = incl[r] - o;
      if (n == 0 || uint64_t(o) + n > room) continue;
      uint32_t* dst = out + o;
      bool bad = false;
      const uint64_t c = direct_row(p, A_ID, uint64_t(c0row) + r, dbits, dreach, nullptr,
                                    [&](uint64_t k, uint32_t v) {
                                      if (k < n) dst[k] = v;
                                      else bad = true;
                                    },
                                    kRowDirectWW);
      if (bad || c != n) raise_flag(p, &p.ctl->status, 8ull);
    }
  };
  while (t < p.nchunks || pend) {
    const bool have = t < p.nchunks;
    // thread 0 takes the next ticket while the rows are walked (its latency
    // hides behind the chunk); a planned build takes none once aborted
    const bool stop = tid == 0 && p.abort && *reinterpret_cast<volatile unsigned long long*>(p.abort) != 0;
    uint32_t next = 0xffffffffu;
    const uint32_t c0row = have ? t * p.chunk_rows : 0u;
    const uint32_t crows = have ? min(p.chunk_rows, p.nrows - c0row) : 0u;
    uint32_t* const incl = S.incl;
    unsigned long long nnz_acc = 0, cnt = 0, cnnz = 0;
    uint32_t fast_mask = 0, nslow = 0, ngen = 0;
    bool staged = false;
    LookbackAhead ahead{0ull, 0ull, false};
    if (have) {
      // stage A's row pointers and ranges of the chunk (coalesced)
      uint64_t abase = 0;
      uint32_t nst = 0;
      if (!A_ID) {
        if (pre) {
          // requested during the previous iteration
          cp_async_wait();
          cta_sync();
        } else {
          for (uint32_t r = tid; r <= crows; r += kThreads) S.u.a.arow[r] = __ldg(p.a_rowmap + uint64_t(c0row) + r);
          cta_sync();
        }
        abase = S.u.a.arow[0] >> 1;
        const uint64_t nrange = (S.u.a.arow[crows] >> 1) - abase;
        nst = nrange < uint64_t(kAStage) ? uint32_t(nrange) : uint32_t(kAStage);
        if (!pre) {
          for (uint32_t k = tid; k < nst; k += kThreads) S.u.a.aent[k] = load_range(p.a_entries, abase + k);
          cta_sync();
        }
      }
      // Rows of the common shape -- one A range whose B rows hold at most one
      // range, an addend row of at most one range -- are counted from loads
      // issued for all of the thread's rows at once: two dependent trips to
      // memory for all of them, where a walk takes two or three per row.
      uint32_t quick = 0;
      uint2 qx[kRowRowsMax], qy[kRowRowsMax];
      {
        uint64_t t0[kRowRowsMax], t1[kRowRowsMax], d0[kRowRowsMax], d1[kRowRowsMax];
        uint32_t one = 0;  // rows with one A range, staged and not read through levels
#pragma unroll
        for (int u = 0; u < kRowRowsMax; ++u) {
          t0[u] = t1[u] = d0[u] = d1[u] = 0;
          const uint32_t r = (warp * rpt + u) * 32 + lane;
          if (uint32_t(u) >= rpt || r >= crows) continue;
          uint2 ar = make_uint2(1u, 0u);
          bool single = true;
          if (A_ID) {
            ar = id_range(p, uint64_t(c0row) + r);
          } else {
            const uint64_t a0 = S.u.a.arow[r] >> 1, a1 = S.u.a.arow[r + 1] >> 1;
            single = a1 - a0 == 1 && a0 - abase < nst;
            if (single) ar = S.u.a.aent[a0 - abase];
          }
          if (!single || (ar.x <= ar.y && p.nlevels && ar.y - ar.x >= 3u)) continue;
          one |= 1u << u;
          if (ar.x <= ar.y) {
            t0[u] = __ldg(p.b_rowmap + ar.x);
            t1[u] = __ldg(p.b_rowmap + uint64_t(ar.y) + 1);
          }
          if (p.d_rowmap) {
            d0[u] = __ldg(p.d_rowmap + uint64_t(c0row) + r);
            d1[u] = __ldg(p.d_rowmap + uint64_t(c0row) + r + 1);
          }
        }
#pragma unroll
        for (int u = 0; u < kRowRowsMax; ++u) {
          const uint64_t b0 = t0[u] >> 1, b1 = t1[u] >> 1, e0 = d0[u] >> 1, e1 = d1[u] >> 1;
          qx[u] = qy[u] = make_uint2(1u, 0u);
          if (!((one >> u) & 1u) || b1 - b0 > 1 || e1 - e0 > 1) continue;
          quick |= 1u << u;
          if (b1 > b0) qx[u] = load_range(p.b_entries, b0);
          if (e1 > e0) qy[u] = load_range(p.d_entries, e0);
        }
      }
      // the common rows into the thread's slot, in row order; the others are
      // listed for the general walk, so that a warp whose lanes hold a few
      // of them does not make the other lanes wait through it
      uint32_t pos = 0;
#pragma unroll
      for (int u = 0; u < kRowRowsMax; ++u) {
        const uint32_t r = (warp * rpt + u) * 32 + lane;
        if (uint32_t(u) >= rpt || r >= crows) continue;
        uint32_t c = 0;
        const uint2 qd = p.d_identity ? make_uint2(c0row + r, c0row + r) : qy[u];
        if (((quick >> u) & 1u) && two_ranges<SLOT>(S, qx[u], qd, pos, c, nnz_acc)) {
          fast_mask |= 1u << u;
          pos += c;
          incl[r] = c;
        } else {
          S.gen[atomicAdd(&S.ngen, 1u)] = uint16_t(r);
        }
      }
      cta_sync();
      // the general walk, entry i by lane i / kWarps of warp i % kWarps: the
      // warps share a chunk's few general rows; each row's runs go to the
      // walker's slot after its own rows.  Rows that miss the slot wait for
      // the warp-cooperative pass below, so one wide row never holds a whole
      // chunk behind a single thread.
      ngen = S.ngen;
      for (uint32_t i = uint32_t(lane) * kWarps + warp; i < ngen; i += kThreads) {
        const uint32_t r = S.gen[i];
        uint32_t c = 0;
        if (row_runs<A_ID, SLOT>(S, p, uint64_t(c0row) + r, r, abase, nst, pos, c, nnz_acc)) {
          pos += c;
        } else {
          const uint32_t j = atomicAdd(&S.nslow, 1u);
          if (j < uint32_t(kSlowMax)) {
            S.slow[j] = r;
            S.gen[i] = uint16_t(r | kGenWarp);
          } else {
            c = light_row<A_ID>(nullptr, nullptr, p, c0row, r, false, &nnz_acc, [](uint64_t, uint32_t) {});
            S.gen[i] = uint16_t(r | kGenLight);
          }
          atomicAdd(&p.ctl->slow_rows, 1ull);
        }
        incl[r] = c;
      }
      cta_sync();
      if (tid == 0 && !stop) next = atomicAdd(p.ticket, 1u);
      // the stage is dead from here on: the warp path may use the space
      nslow = min(S.nslow, uint32_t(kSlowMax));
      if (nslow) {
        for (uint32_t i = warp; i < nslow; i += kWarps) {
          const uint32_t r = S.slow[i];
          const uint64_t c = direct_row(p, A_ID, uint64_t(c0row) + r, dbits, dreach, &nnz_acc,
                                        [](uint64_t, uint32_t) {}, kRowDirectWW);
          if (lane == 0) incl[r] = uint32_t(min(c, uint64_t(0xffffffffu)));
        }
        cta_sync();
      }
      // chunk prefix over the row counts (kRowRowsMax consecutive rows per
      // thread: a thread rewrites only its own rows) and the chunk's nnz
      {
        uint32_t loc[kRowRowsMax];
        uint64_t s = 0;
#pragma unroll
        for (int k = 0; k < kRowRowsMax; ++k) {
          const uint32_t r = tid * kRowRowsMax + k;
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
        for (int k = 0; k < kRowRowsMax; ++k) {
          const uint32_t r = tid * kRowRowsMax + k;
          if (r < crows) incl[r] = uint32_t(excl) + loc[k];
        }
      }
      cta_sync();
      for (int i = 0; i < kWarps; ++i) cnnz += S.red_nnz[i];
      cnt = incl[crows - 1];
      if (tid == 0) atomicAdd(&p.ctl->nnz, cnnz);
      staged = stage != nullptr && cnt <= p.stage_cap;
      // the pending chunk's look-back reads its first descriptors now, so
      // the reads are in flight while the image is written
      if (pend) ahead = lookback_read_ahead(p, S.pend_t[b ^ 1u]);
      if (staged) {
        // the chunk's image: fast rows from the slots, the rest recomputed
        uint32_t* img = stage + size_t(b) * (p.stage_cap + p.chunk_rows);
        if (tid == 0) publish_aggregate(p, t, cnt);
        for (uint32_t r = tid; r < crows; r += kThreads) img[p.stage_cap + r] = incl[r];
        write_rows(img, ~0ull, false, c0row, crows, fast_mask, ngen, nslow);
      }
    }
    if (tid == 0) S.next = next;
    // every thread is done with the slots, the slow list and the counted
    // chunk's image; the warp path's windows are free again
    cta_sync();
    // after a staged chunk the shared stage stays free until the next
    // iteration: request the next chunk's A row pointers now, its ranges once
    // those have landed, so both arrive behind the pending chunk's write-out
    pre = !A_ID && have && staged && S.next < p.nchunks && a_async;
    uint32_t n0row = 0, nrows1 = 0;
    if (pre) {
      n0row = S.next * p.chunk_rows;
      nrows1 = min(p.chunk_rows, p.nrows - n0row);
      if ((reinterpret_cast<uintptr_t>(p.a_rowmap) & 15u) == 0) {
        // pairs of row pointers in 16-byte copies (chunks start at a multiple
        // of 32 rows, so every pair is aligned in both spaces), the last odd one alone
        for (uint32_t q = tid; q < (nrows1 + 1) / 2; q += kThreads)
          cp_async16(&S.u.a.arow[2 * q], p.a_rowmap + uint64_t(n0row) + 2 * q);
        if (tid == 0 && !(nrows1 & 1u)) cp_async8(&S.u.a.arow[nrows1], p.a_rowmap + uint64_t(n0row) + nrows1);
      } else {
        for (uint32_t r = tid; r <= nrows1; r += kThreads) cp_async8(&S.u.a.arow[r], p.a_rowmap + uint64_t(n0row) + r);
      }
      cp_async_commit();
    }
    // the pending chunk: look-back, row map, one coalesced copy
    if (pend) {
      const uint32_t pend_t = S.pend_t[b ^ 1u], pend_crows = S.pend_crows[b ^ 1u];
      const unsigned long long pend_cnt = S.pend_cnt[b ^ 1u];
      const unsigned long long prefix = lookback_block(S, p, pend_t, pend_cnt, par, ahead);
      const uint32_t* img = stage + size_t(b ^ 1u) * (p.stage_cap + p.chunk_rows);
      const uint32_t* pincl = img + p.stage_cap;
      const uint32_t p0row = pend_t * p.chunk_rows;
      // loads first, then stores: the staging and the output may alias as
      // far as the compiler knows, and a load after a store would wait
      {
        uint32_t v[kRowRowsMax];
#pragma unroll
        for (int u = 0; u < kRowRowsMax; ++u) {
          const uint32_t r = tid + u * kThreads;
          v[u] = r < pend_crows ? __ldcg(pincl + r) : 0u;
        }
#pragma unroll
        for (int u = 0; u < kRowRowsMax; ++u) {
          const uint32_t r = tid + u * kThreads;
          if (r < pend_crows) p.c_rowmap[uint64_t(p0row) + r + 1] = prefix + v[u];
        }
      }
      if (pend_t == 0 && tid == 0) p.c_rowmap[0] = 0;
      if (prefix + pend_cnt <= p.cap) {
        // ranges of 8 bytes: images start 8-byte aligned (17 words a chunk row,
        // chunks of a multiple of 32 rows) and prefix is even
        uint2* dst = reinterpret_cast<uint2*>(p.c_entries + prefix);
        const uint2* src = reinterpret_cast<const uint2*>(img);
        const uint64_t npend = pend_cnt / 2;
        constexpr int kBatch = 4;
        for (uint64_t k0 = 0; k0 < npend; k0 += uint64_t(kBatch) * kThreads) {
          uint2 v[kBatch];
#pragma unroll
          for (int u = 0; u < kBatch; ++u) {
            const uint64_t k = k0 + tid + uint64_t(u) * kThreads;
            v[u] = k < npend ? __ldcg(src + k) : make_uint2(0u, 0u);
          }
#pragma unroll
          for (int u = 0; u < kBatch; ++u) {
            const uint64_t k = k0 + tid + uint64_t(u) * kThreads;
            if (k < npend) dst[k] = v[u];
          }
        }
      } else if (tid == 0 && pend_cnt) {
        raise_flag(p, &p.ctl->overflow, 1ull);
      }
      pend = false;
    }
    if (pre) {
      cp_async_wait();
      cta_sync();
      const uint64_t nbase = S.u.a.arow[0] >> 1;
      const uint64_t nrange = (S.u.a.arow[nrows1] >> 1) - nbase;
      const uint32_t nst1 = nrange < uint64_t(kAStage) ? uint32_t(nrange) : uint32_t(kAStage);
      for (uint32_t k = tid; k < nst1; k += kThreads) cp_async8(&S.u.a.aent[k], p.a_entries + 2 * (nbase + k));
      cp_async_commit();
    }
    // a counted chunk that was not staged is resolved now, in place
    if (have && !staged) {
      if (tid == 0) publish_aggregate(p, t, cnt);
      const unsigned long long prefix = lookback_block(S, p, t, cnt, par);
      for (uint32_t r = tid; r < crows; r += kThreads) p.c_rowmap[uint64_t(c0row) + r + 1] = prefix + incl[r];
      if (t == 0 && tid == 0) p.c_rowmap[0] = 0;
      write_rows(p.c_entries + prefix, p.cap > prefix ? p.cap - prefix : 0ull, true, c0row, crows, fast_mask, ngen,
                 nslow);
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
    t = S.next;
  }
}

// One CTA runs the look-back of chunk t over descriptors nothing publishes,
// so its bounded wait must run out (the library's self-test of that path).
__global__ void __launch_bounds__(kThreads, 1) k_lookback_selftest(FusedArgs p, uint32_t t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RowSmem<16>& S = *reinterpret_cast<RowSmem<16>*>(smem_raw);
  uint32_t par = 0;
  (void)lookback_block(S, p, t, 0ull, par);
}

template <bool A_ID, int SLOT>
struct RowKernel {
  static void* get() { return reinterpret_cast<void*>(&k_spgemm_rowmode<A_ID, SLOT>); }
  static constexpr int smem() { return int(sizeof(RowSmem<SLOT>)); }
};

}  // namespace

int row_slot_entries(int variant) {
  static const int kSlots[] = {16, 24, 32};
  return kSlots[std::min(std::max(variant, 0), 2)];
}

RowLaunchShape row_launch_shape(dvg_context* ctx, uint32_t nrows, int64_t chunk_rows_opt, int slot_variant) {
  const int v = std::min(std::max(slot_variant, 0), 2);
  // occupancy is a property of the kernel: queried once per context
  if (ctx->row_resident[v] == 0) {
    void* kern[3] = {RowKernel<false, 16>::get(), RowKernel<false, 24>::get(), RowKernel<false, 32>::get()};
    void* kern_id[3] = {RowKernel<true, 16>::get(), RowKernel<true, 24>::get(), RowKernel<true, 32>::get()};
    const int smem[3] = {RowKernel<false, 16>::smem(), RowKernel<false, 24>::smem(), RowKernel<false, 32>::smem()};
    for (void* k : {kern[v], kern_id[v]})
      DVG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem[v]));
    int per_sm = 0;
    DVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern[v], kThreads, smem[v]));
    if (per_sm < 1) throw Error(DVG_ERR_DEVICE, "row spgemm: shared memory layout does not fit");
    ctx->row_resident[v] = uint32_t(per_sm) * uint32_t(ctx->num_sms);
  }
  RowLaunchShape s{};
  s.resident = ctx->row_resident[v];
  // chunk rows: as large as possible (fewer look-back steps) while keeping
  // about four chunks per resident CTA
  uint32_t chunk_rows = kChunkMax;
  while (chunk_rows > 64 && (uint64_t(nrows) + chunk_rows - 1) / chunk_rows < 4ull * s.resident) chunk_rows >>= 1;
  if (chunk_rows_opt > 0) chunk_rows = uint32_t(std::min<int64_t>(chunk_rows_opt, kChunkMax));
  s.chunk_rows = chunk_rows;
  s.nchunks = uint32_t((uint64_t(nrows) + chunk_rows - 1) / chunk_rows);
  s.grid = uint32_t(std::min<uint64_t>(s.nchunks, s.resident));
  s.desc_bytes = size_t(s.nchunks) * sizeof(ChunkDesc);
  s.stage_bytes = size_t(s.grid) * 2 * (kRowStagePerRow + 1) * s.chunk_rows * sizeof(uint32_t);
  return s;
}

void selftest_bounded_wait(dvg_context* ctx, uint32_t spin_limit) {
  // two descriptors, both empty: chunk 1 waits on chunk 0 for good
  void* desc = dalloc(ctx, 2 * sizeof(ChunkDesc));
  try {
    DVG_CUDA(cudaMemsetAsync(desc, 0, 2 * sizeof(ChunkDesc), ctx->stream));
    FusedArgs p{};
    p.desc = static_cast<ChunkDesc*>(desc);
    p.ctl = ctx->d_ctl;
    p.nchunks = 2;
    p.cap = ~0ull;
    p.spin_limit = spin_limit ? spin_limit : 1;
    const int smem = int(sizeof(RowSmem<16>));
    DVG_CUDA(cudaFuncSetAttribute(k_lookback_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_lookback_selftest<<<1, kThreads, smem, ctx->stream>>>(p, 1u);
    DVG_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
  } catch (...) {
    dfree(ctx, desc);
    throw;
  }
  dfree(ctx, desc);
}

void launch_rowmode(dvg_context* ctx, const RowLaunch& L, const RowLaunchShape& s) {
  if (L.nrows == 0) return;
  const int v = std::min(std::max(L.slot_variant, 0), 2);
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
  p.stage_cap = L.stage_buf ? uint32_t(kRowStagePerRow) * s.chunk_rows : 0u;
  p.a_shift = L.a_identity ? L.a_shift : 0u;
  p.b_nrows = L.b_nrows;
  p.nlevels = L.nlevels;
  for (uint32_t k = 0; k < L.nlevels && k < uint32_t(kMaxLevels); ++k) {
    p.lv_rowmap[k] = L.lv_rowmap[k];
    p.lv_entries[k] = L.lv_entries[k];
  }
  const int smem[3] = {RowKernel<false, 16>::smem(), RowKernel<false, 24>::smem(), RowKernel<false, 32>::smem()};
  const dim3 grid(s.grid), block(kThreads);
  if (L.a_identity) {
    if (v == 0) k_spgemm_rowmode<true, 16><<<grid, block, smem[v], ctx->stream>>>(p);
    else if (v == 1) k_spgemm_rowmode<true, 24><<<grid, block, smem[v], ctx->stream>>>(p);
    else k_spgemm_rowmode<true, 32><<<grid, block, smem[v], ctx->stream>>>(p);
  } else {
    if (v == 0) k_spgemm_rowmode<false, 16><<<grid, block, smem[v], ctx->stream>>>(p);
    else if (v == 1) k_spgemm_rowmode<false, 24><<<grid, block, smem[v], ctx->stream>>>(p);
    else k_spgemm_rowmode<false, 32><<<grid, block, smem[v], ctx->stream>>>(p);
  }
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
  ctx->stats.spgemm_light++;
}

}  // namespace dvg
