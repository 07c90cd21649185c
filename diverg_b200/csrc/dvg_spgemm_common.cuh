// dvg_spgemm_common.cuh -- pieces shared by the two single-pass range SpGEMM
// kernels (tile-staged: dvg_spgemm_fused.cu; thread per row:
// dvg_spgemm_rows.cu): launch constants, the chunk descriptors of the
// decoupled look-back, the kernel arguments, the warp-cooperative row path for
// rows too wide for the fast paths, the look-back itself and the per-thread
// windowed fallback.  Included by both translation units (internal linkage).
#pragma once

#include "dvg_device.cuh"
#include "dvg_internal.h"

namespace dvg {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kSubRows = 64;      // rows per staged sub-tile
constexpr int kChunkMax = 2048;   // rows per look-back chunk (upper bound)
constexpr int kSubMax = kChunkMax / kSubRows;
constexpr int kAChunk = 3072;     // A ranges staged per chunk
constexpr int kSpanMax = 384;     // B rows staged per sub-tile
constexpr int kBMax = 768;        // B ranges staged per sub-tile
constexpr int kBitWords = 6144;   // union bitmaps (PRE, SUF, BU) or direct windows
constexpr int kStageMax = 6144;   // output entries staged per chunk
constexpr int kMaxBlock = 32;     // union block rows (at most a warp)
constexpr int kSlowMax = 512;     // row mode: rows per chunk deferred to the warp path
constexpr int kDirectWW = kBitWords / (2 * kWarps);  // direct path window words per warp
constexpr int kMaxLevels = 12;    // union levels of B (blocks of up to 4096 rows)
constexpr unsigned long long kFlag = 1ull << 63;
constexpr uint32_t kSpinLimit = 1u << 22;

// agg and incl are adjacent (one 16-byte load reads both); each is a
// self-contained flag | value word.
struct ChunkDesc {
  unsigned long long agg;       // kFlag | entries of the chunk
  unsigned long long incl;      // kFlag | entries of chunks 0..t
  unsigned long long agg_nnz;   // (tiled kernel) nnz of the chunk, valid once agg is flagged
  unsigned long long incl_nnz;  // (tiled kernel) nnz of chunks 0..t, valid once incl is flagged
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
  uint32_t row_mode;    // 1: a thread per row (run list); 0: tile-staged rows
  // optional addend (row mode only): C = D + A B, D with the rows and columns of C
  const uint64_t* __restrict__ d_rowmap;
  const uint32_t* __restrict__ d_entries;
  uint32_t d_identity;  // the addend is the identity (d_rowmap unused)
  // planned builds: a word every step checks before it starts and sets when
  // its output is unusable (overflow, timeout, internal error); null otherwise
  unsigned long long* abort;
  // row mode, A the identity: A's row r is column r + a_shift (empty past B's
  // last row), so C = D + S B adds B shifted up by a_shift rows
  uint32_t a_shift;
  uint32_t b_nrows;
  // row mode: union levels of B, level k (1..nlevels) row j = the union of B
  // rows j .. j + 2^k - 1 (rows past B's end count as empty); an A range of
  // 4 or more rows takes a couple of level rows instead of its B rows
  uint32_t nlevels;
  const uint64_t* lv_rowmap[kMaxLevels];
  const uint32_t* lv_entries[kMaxLevels];
  // row mode: per CTA two staging buffers of stage_cap entries each, where a
  // counted chunk's output waits while the chunk's prefix resolves; null:
  // every chunk is written out in its own iteration
  uint32_t* stage_buf;
  uint32_t stage_cap;
  // polls a look-back waits before it gives up (0: kSpinLimit)
  uint32_t spin_limit;
};

// Row `row` of the (shifted) identity: column row + a_shift, or an empty
// range when that is past B's last row.
__device__ __forceinline__ uint2 id_range(const FusedArgs& p, uint64_t row) {
  const uint64_t c = row + p.a_shift;
  return (p.a_shift && c >= p.b_nrows) ? make_uint2(1u, 0u) : make_uint2(uint32_t(c), uint32_t(c));
}

// Records an error bit in the control block field and, in a planned build,
// stops the steps that follow.
__device__ __forceinline__ void raise_flag(const FusedArgs& p, unsigned long long* field, unsigned long long bits) {
  atomicOr(field, bits);
  if (p.abort) atomicOr(p.abort, 1ull);
}

// ---- small helpers -----------------------------------------------------------

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Gathers the runs of one 32-bit accumulator word per lane of a group of g lanes
// (map01 / map10 boundary masks, ffs); see the callers.
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

// ---- direct path: one C row by a warp, bitvector window in shared memory ----

template <class Emit>
__device__ uint64_t direct_row(const FusedArgs& p, bool a_identity, uint64_t row, uint32_t* bits, uint32_t* reach,
                               unsigned long long* nnz_acc, Emit&& emit, uint32_t ww = kDirectWW) {
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
      const uint2 r = id_range(p, row);
      s = r.x;
      f = r.y;
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
  uint64_t d0 = 0, d1 = 0;  // the addend's ranges of this row
  if (p.d_rowmap) {
    d0 = p.d_rowmap[row] >> 1;
    d1 = p.d_rowmap[row + 1] >> 1;
  }
  for (uint64_t t = d0 + lg; t < d1; t += 32) {
    uint2 r = load_range(p.d_entries, t);
    if (r.y < r.x) continue;
    mn = min(mn, r.x);
    mx = max(mx, r.y);
  }
  if (p.d_identity && lg == 0) {
    mn = min(mn, uint32_t(row));
    mx = max(mx, uint32_t(row));
  }
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
  for (uint64_t w0 = 0; w0 < nw_total; w0 += ww) {
    const uint32_t nwc = uint32_t(min(uint64_t(ww), nw_total - w0));
    const uint64_t cb = base + 32 * w0;
    const uint64_t ce = cb + 32ull * nwc - 1;
    for (uint32_t w = lg; w < nwc; w += 32) {
      bits[w] = 0;
      reach[w] = 0;
    }
    __syncwarp();
    auto put = [&](uint2 r) {
      uint64_t cs = max(uint64_t(r.x), cb);
      uint64_t cf = min(uint64_t(r.y), ce);
      if (cs > cf || r.y < r.x) return;
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
    };
    for (uint64_t t = d0 + lg; t < d1; t += 32) put(load_range(p.d_entries, t));
    if (p.d_identity && lg == 0) put(make_uint2(uint32_t(row), uint32_t(row)));
    for (uint64_t ai = a0; ai < a1; ai += 2) {
      uint64_t b0, b1;
      slice(ai, b0, b1);
      for (uint64_t t = b0 + lg; t < b1; t += 32) put(load_range(p.b_entries, t));
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
          if (lane == 0) raise_flag(p, &p.ctl->timeout, 1ull);
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

// ---- pieces of the thread-per-row kernel (dvg_spgemm_rows.cu) ---------------------

// CTA barrier that counts threads, not warps: the non-aligned form of
// barrier.sync, which the lanes of a warp may reach at different times.  The
// row loop leaves the lanes of a warp on paths of very different length (one
// lane walks a wide row while the others wait), and the aligned form
// (__syncthreads) is only defined for warps that arrive converged.  Every
// barrier of the row kernel is this one, on barrier 0.
__device__ __forceinline__ void cta_sync() { asm volatile("barrier.sync 0;" ::: "memory"); }

// Asynchronous 8-byte copy global -> shared (cp.async): the copy lands while
// the thread goes on; cp_async_wait() waits for all of the thread's copies.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const uint32_t sa = uint32_t(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
// The same for 16 bytes (both addresses 16-byte aligned), bypassing L1.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t sa = uint32_t(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A descriptor word (flag | value) for other CTAs' look-backs.  The word is
// all a reader takes from it -- no other data of the writer is read on its
// strength -- so a relaxed store does: a release would first wait for every
// earlier store of the thread (its share of a chunk image) to land.
__device__ __forceinline__ void st_relaxed(unsigned long long* q, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(q), "l"(v) : "memory");
}

// Publishes chunk t's aggregate (its entries) for later chunks' look-backs.
__device__ __forceinline__ void publish_aggregate(const FusedArgs& p, uint32_t t, unsigned long long cnt) {
  st_relaxed(&p.desc[t].agg, kFlag | cnt);
}

// The whole CTA walks back from chunk t (whose aggregate is published),
// kThreads descriptors a round, summing aggregates down to the nearest
// inclusive prefix; every thread gets t's exclusive prefix and thread 0
// publishes t's inclusive prefix (and, for the last chunk, the total).  A
// deferred chunk's predecessors have mostly published aggregates but not yet
// prefixes, so the walk is a few hundred descriptors deep: one round here.
// A round is one 16-byte load per thread and one barrier: each warp reduces
// its 32 descriptors (newest first) to a record -- the sum up to its first
// prefix, whether it has one, whether a descriptor before that has nothing
// yet -- and every thread scans the 16 records in order.  The records
// alternate between two sets by round (`par` runs on across calls), so a
// round's writes never meet the previous round's reads.  Waits are bounded;
// every branch is uniform over the CTA.
// The descriptor a thread reads in the first round of chunk t's look-back,
// read ahead of it (a descriptor only ever moves on from nothing to an
// aggregate to an inclusive prefix, so an early read is an earlier state).
struct LookbackAhead {
  unsigned long long agg, incl;
  bool valid;
};
__device__ __forceinline__ LookbackAhead lookback_read_ahead(const FusedArgs& p, uint32_t t) {
  LookbackAhead a{0ull, 0ull, true};
  const int64_t idx = int64_t(t) - 1 - threadIdx.x;
  if (idx >= 0)
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];"
                 : "=l"(a.agg), "=l"(a.incl)
                 : "l"(&p.desc[idx].agg)
                 : "memory");
  return a;
}

template <class SmemT>
__device__ unsigned long long lookback_block(SmemT& S, const FusedArgs& p, uint32_t t,
                                             unsigned long long cnt, uint32_t& par,
                                             LookbackAhead ahead = LookbackAhead{0ull, 0ull, false}) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  ChunkDesc* d = p.desc;
  unsigned long long pre = 0;
  int64_t j = int64_t(t) - 1;
  uint32_t spins = 0;
  while (j >= 0) {
    const int64_t idx = j - tid;
    int st = 2;  // 2: inclusive prefix (or before chunk 0), 1: aggregate, 0: nothing yet
    unsigned long long v = 0;
    if (idx >= 0) {
      unsigned long long va, vi;
      if (ahead.valid) {  // the first round, read ahead
        va = ahead.agg;
        vi = ahead.incl;
      } else {
        asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(va), "=l"(vi) : "l"(&d[idx].agg) : "memory");
      }
      if (vi & kFlag) {
        v = vi & ~kFlag;
      } else if (va & kFlag) {
        st = 1;
        v = va & ~kFlag;
      } else {
        st = 0;
      }
    }
    const unsigned im = __ballot_sync(kFullMask, st == 2), wm = __ballot_sync(kFullMask, st == 0);
    const int fi = im ? __ffs(im) - 1 : 32;
    const unsigned before = fi == 32 ? kFullMask : ((1u << fi) - 1u);
    unsigned long long sv = lane <= fi ? v : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sv += __shfl_xor_sync(kFullMask, sv, o);
    if (lane == 0) {
      S.lb_sum[par][warp] = sv;
      S.lb_flag[par][warp] = (fi < 32 ? 1u : 0u) | ((wm & before) ? 2u : 0u);
    }
    cta_sync();
    unsigned long long tot = 0;
    bool done = false, wait = false;
#pragma unroll 1
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t f = S.lb_flag[par][w];
      if (f & 2u) {
        wait = true;
        break;
      }
      tot += S.lb_sum[par][w];
      if (f & 1u) {
        done = true;
        break;
      }
    }
    par ^= 1u;
    ahead.valid = false;
    if (wait) {  // a chunk after the nearest prefix has published nothing yet
      if (++spins > (p.spin_limit ? p.spin_limit : kSpinLimit)) {
        if (tid == 0) raise_flag(p, &p.ctl->timeout, 1ull);
        break;
      }
      __nanosleep(64);
      continue;
    }
    pre += tot;
    if (done) break;
    j -= kThreads;
  }
  if (tid == 0) {
    st_relaxed(&d[t].incl, kFlag | (pre + cnt));
    if (t == p.nchunks - 1) {
      p.ctl->total = pre + cnt;
      if (pre + cnt > p.cap) raise_flag(p, &p.ctl->overflow, pre + cnt);
    }
  }
  return pre;
}

// ---- light path: one C row by one thread --------------------------------------
//
// For products whose rows union only a handful of B ranges (powers of A, the
// final A^d * (A+I)^k product) a thread per row beats any cooperative scheme:
// the row's ranges -- read from the staged chunk of A and from B through L1 --
// are ORed into a 128-column register bitmap anchored at the row's first
// column; the runs come out with the same boundary masks as the tiled gather,
// on 64-bit words.  Rows wider than the window take further 128-column
// windows, each re-reading the row's ranges.
template <bool A_ID, class Emit>
__device__ uint32_t light_row(const uint32_t* crow, const uint2* achunk, const FusedArgs& p, uint32_t c0row,
                              uint32_t r, bool a_staged, unsigned long long* nnz_acc, Emit&& emit) {
  const uint64_t row = uint64_t(c0row) + r;
  uint64_t a0, a1;
  if (A_ID) {
    a0 = 0;
    a1 = 1;
  } else if (a_staged) {
    a0 = crow[r] >> 1;
    a1 = crow[r + 1] >> 1;
  } else {
    a0 = p.a_rowmap[row] >> 1;
    a1 = p.a_rowmap[row + 1] >> 1;
  }
  auto a_range = [&](uint64_t k) -> uint2 {
    if (A_ID) return id_range(p, row);
    return a_staged ? achunk[k] : load_range(p.a_entries, k);
  };
  uint64_t d0 = 0, d1 = 0;  // the addend's ranges of this row
  if (p.d_rowmap) {
    d0 = p.d_rowmap[row] >> 1;
    d1 = p.d_rowmap[row + 1] >> 1;
  }
  // column band of the row
  uint32_t lo = 0xffffffffu, hi = 0;
  for (uint64_t t = d0; t < d1; ++t) {
    const uint2 b = load_range(p.d_entries, t);
    if (b.y < b.x) continue;
    lo = min(lo, b.x);
    hi = max(hi, b.y);
  }
  if (p.d_identity) {
    lo = min(lo, uint32_t(row));
    hi = max(hi, uint32_t(row));
  }
  for (uint64_t k = a0; k < a1; ++k) {
    const uint2 ar = a_range(k);
    if (ar.y < ar.x) continue;
    const uint64_t t0 = __ldg(p.b_rowmap + ar.x) >> 1, t1 = __ldg(p.b_rowmap + uint64_t(ar.y) + 1) >> 1;
    for (uint64_t t = t0; t < t1; ++t) {
      const uint2 b = load_range(p.b_entries, t);
      if (b.y < b.x) continue;
      lo = min(lo, b.x);
      hi = max(hi, b.y);
    }
  }
  if (lo > hi) return 0;
  uint32_t count = 0;
  uint64_t carry = 0;
  for (uint64_t wb = lo & ~63u; wb <= hi; wb += 128) {
    uint64_t w0 = 0, w1 = 0;
    auto put = [&](uint2 b) {
      const uint64_t x = max(uint64_t(b.x), wb), y = min(uint64_t(b.y), wb + 127);
      if (b.y < b.x || x > y) return;
      const uint32_t xs = uint32_t(x - wb), ys = uint32_t(y - wb);
      if (xs < 64) w0 |= (~0ull << xs) & (ys < 64 ? (~0ull >> (63 - ys)) : ~0ull);
      if (ys >= 64) w1 |= (~0ull << (xs < 64 ? 0 : xs - 64)) & (~0ull >> (127 - ys));
    };
    for (uint64_t t = d0; t < d1; ++t) put(load_range(p.d_entries, t));
    if (p.d_identity) put(make_uint2(uint32_t(row), uint32_t(row)));
    for (uint64_t k = a0; k < a1; ++k) {
      const uint2 ar = a_range(k);
      if (ar.y < ar.x) continue;
      const uint64_t t0 = __ldg(p.b_rowmap + ar.x) >> 1, t1 = __ldg(p.b_rowmap + uint64_t(ar.y) + 1) >> 1;
      for (uint64_t t = t0; t < t1; ++t) put(load_range(p.b_entries, t));
    }
    if (nnz_acc) *nnz_acc += __popcll(w0) + __popcll(w1);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint64_t x = h ? w1 : w0;
      const uint64_t sh = (x << 1) | carry;
      uint64_t bnd = ((x ^ sh) & x) | (sh & ~x);
      const uint64_t c0 = wb + 64 * h;
      while (bnd) {
        const int bit = __ffsll(bnd) - 1;
        bnd &= bnd - 1;
        emit(count, uint32_t(c0 + bit - (count & 1)));
        ++count;
      }
      carry = x >> 63;
    }
  }
  if (carry) {  // a run reaching the last window's end closes at column hi
    emit(count, hi);
    ++count;
  }
  return count;
}

// ---- warp path for rows that name many B ranges ------------------------------

// Window word w of the calling lane (32 consecutive words a warp) and its
// reach rr (one past the largest end column, in window columns, of the
// ranges that start in word w and end past it; 0: none): the bits of word w
// that ranges starting in earlier words cover -- everything from the word's
// first column to the largest reach before it.  run_reach carries the largest
// reach of the earlier 32-word blocks and is advanced past this block.
__device__ __forceinline__ uint32_t reach_cover(uint32_t w, uint32_t rr, uint32_t& run_reach, int lane) {
  const uint32_t incl = group_incl_max<32>(kFullMask, rr, lane);
  uint32_t before = __shfl_up_sync(kFullMask, incl, 1);
  before = max(lane ? before : 0u, run_reach);
  run_reach = max(run_reach, __shfl_sync(kFullMask, incl, 31));
  const uint32_t c0 = 32u * w;  // the word's first column
  if (before <= c0) return 0u;
  const uint32_t n = before - c0;  // covered columns from c0
  return n >= 32u ? ~0u : (1u << n) - 1u;
}


// Calls f(range) on this lane's share of the addend's ranges of `row` and of
// every B range the row's A ranges name.  The slice bounds of the first 32 A
// ranges are loaded once (by the lanes, together) and kept in b0 / b1.
template <class F>
__device__ __forceinline__ void wide_ranges(const FusedArgs& p, uint64_t row, uint64_t a0, uint64_t a1, uint64_t d0,
                                            uint64_t d1, uint64_t b0, uint64_t b1, F&& f) {
  const int lane = lane_id();
  for (uint64_t t = d0 + lane; t < d1; t += 32) f(load_range(p.d_entries, t));
  if (p.d_identity && lane == 0) f(make_uint2(uint32_t(row), uint32_t(row)));
  for (uint64_t g = a0; g < a1; g += 32) {
    uint64_t s0 = b0, s1 = b1;
    if (g != a0) {  // a row of more than 32 A ranges: this group's slices
      s0 = s1 = 0;
      if (g + lane < a1) {
        const uint2 ar = load_range(p.a_entries, g + lane);
        if (ar.x <= ar.y) {
          s0 = __ldg(p.b_rowmap + ar.x) >> 1;
          s1 = __ldg(p.b_rowmap + uint64_t(ar.y) + 1) >> 1;
        }
      }
    }
    const uint32_t m = uint32_t(min(uint64_t(32), a1 - g));
    for (uint32_t i = 0; i < m; ++i) {
      const uint64_t t0 = __shfl_sync(kFullMask, s0, int(i)), t1 = __shfl_sync(kFullMask, s1, int(i));
      uint64_t t = t0 + lane;
      for (; t + 32 < t1; t += 64) {  // two loads in flight a lane
        const uint2 x = load_range(p.b_entries, t), y = load_range(p.b_entries, t + 32);
        f(x);
        f(y);
      }
      if (t < t1) f(load_range(p.b_entries, t));
    }
  }
}

// One C row by the calling warp over its window of WIN words (bits, reach):
// the warp-path row of the SpGEMM kernels, faster than direct_row when a row
// names many B ranges (all its A ranges' slices are loaded at once, and a row
// that fits one window anchored at its first range takes one pass).  Emits the
// row's runs (entry k, value) and returns its entry count (the same on every
// lane); adds the row's nnz to *nnz (each lane its words).
template <uint32_t WIN, class Emit>
__device__ uint64_t wide_row(const FusedArgs& p, uint64_t row, uint32_t* bits, uint32_t* reach,
                             unsigned long long* nnz, Emit&& emit) {
  const int lane = lane_id();
  const uint64_t a0 = __ldg(p.a_rowmap + row) >> 1, a1 = __ldg(p.a_rowmap + row + 1) >> 1;
  uint64_t d0 = 0, d1 = 0;
  if (p.d_rowmap) {
    d0 = __ldg(p.d_rowmap + row) >> 1;
    d1 = __ldg(p.d_rowmap + row + 1) >> 1;
  }
  uint64_t b0 = 0, b1 = 0;  // the slice of A range a0 + lane
  if (a0 + lane < a1) {
    const uint2 ar = load_range(p.a_entries, a0 + lane);
    if (ar.x <= ar.y) {
      b0 = __ldg(p.b_rowmap + ar.x) >> 1;
      b1 = __ldg(p.b_rowmap + uint64_t(ar.y) + 1) >> 1;
    }
  }
  // First one window, anchored half a window before the row's first B range
  // (or addend range): when every range falls inside it (all but the last
  // word, which closes the last run), one pass over the ranges makes the row.
  {
    const unsigned nonempty = __ballot_sync(kFullMask, b1 > b0);
    uint32_t s0 = 0xffffffffu;
    if (nonempty) {
      const int l = __ffs(nonempty) - 1;
      const uint64_t t = __shfl_sync(kFullMask, b0, l);
      if (lane == 0) s0 = load_range(p.b_entries, t).x;
    } else if (d1 > d0) {
      if (lane == 0) s0 = load_range(p.d_entries, d0).x;
    }
    s0 = __shfl_sync(kFullMask, s0, 0);
    // (window words and the columns they start at in 32 bits: columns are
    // below 2^32 - 2, and a window starting past them would hold nothing)
    if (s0 != 0xffffffffu && s0 < 0xffffffffu - 32u * WIN) {
      const uint32_t cb = (s0 >= 32u * (WIN / 2) ? s0 - 32u * (WIN / 2) : 0u) & ~31u;
      const uint32_t span = 32u * (WIN - 1);  // the last word stays empty
      for (uint32_t w = lane; w < uint32_t(WIN); w += 32) {
        bits[w] = 0;
        reach[w] = 0;
      }
      __syncwarp();
      bool out = false;
      uint32_t top = 0, bottom = WIN;  // words in [bottom, top) hold bits
      wide_ranges(p, row, a0, a1, d0, d1, b0, b1, [&](uint2 r) {
        if (r.y < r.x) return;
        const uint32_t xs = r.x - cb, xe = r.y - cb;  // wrap when r.x < cb: then out of the window
        if (xs >= span || xe >= span) {
          out = true;
          return;
        }
        const uint32_t ws = xs >> 5, we = xe >> 5;
        const uint32_t lo = ~0u << (xs & 31);
        const uint32_t hi = ~0u >> (31 - (xe & 31));
        top = max(top, we + 1);
        bottom = min(bottom, ws);
        // the range's bits in its first word; past that word, its end column
        // (+ 1) as that word's reach: later words are covered up to the
        // largest reach of the words before them
        atomicOr(bits + ws, ws == we ? lo & hi : lo);
        if (ws != we) atomicMax(reach + ws, xe + 1u);
      });
      __syncwarp();
      if (!__any_sync(kFullMask, out)) {
        // words from the first to one past the last touched: runs close there
        const uint32_t nw = min(uint32_t(WIN), group_max<32>(kFullMask, top) + 1);
        const uint32_t w_first = group_min<32>(kFullMask, bottom) & ~31u;  // below: empty words
        uint64_t count = 0;
        uint32_t carry = 0, run_reach = 0;
        for (uint32_t wb = w_first; wb < nw; wb += 32) {
          const uint32_t w = wb + lane;
          const bool valid = w < nw;
          uint32_t x = 0, rr = 0;
          if (valid) {
            x = bits[w];
            rr = reach[w];
          }
          const uint32_t cov = reach_cover(w, rr, run_reach, lane);
          if (valid) x |= cov;
          if (nnz) *nnz += __popc(x);
          count += gather_chunk(x, valid, uint64_t(cb) + 32ull * w, 32, lane, kFullMask, carry, count,
                                min(31u, nw - 1 - wb), emit);
        }
        __syncwarp();
        return count;
      }
    }
  }
  // the general form: the row's column bounds first, then windows over them
  uint32_t mn = 0xffffffffu, mx = 0;
  wide_ranges(p, row, a0, a1, d0, d1, b0, b1, [&](uint2 r) {
    if (r.y < r.x) return;
    mn = min(mn, r.x);
    mx = max(mx, r.y);
  });
  mn = group_min<32>(kFullMask, mn);
  mx = group_max<32>(kFullMask, mx);
  if (mn > mx) return 0;
  uint64_t count = 0;
  const uint64_t base = mn & ~31u;
  const uint64_t nw_total = ((uint64_t(mx) - base) >> 5) + 2;
  uint32_t carry = 0;
  for (uint64_t w0 = 0; w0 < nw_total; w0 += WIN) {
    const uint32_t nwc = uint32_t(min(uint64_t(WIN), nw_total - w0));
    const uint64_t cb = base + 32 * w0;
    const uint64_t ce = cb + 32ull * nwc - 1;
    for (uint32_t w = lane; w < nwc; w += 32) {
      bits[w] = 0;
      reach[w] = 0;
    }
    __syncwarp();
    wide_ranges(p, row, a0, a1, d0, d1, b0, b1, [&](uint2 r) {
      const uint64_t cs = max(uint64_t(r.x), cb);
      const uint64_t cf = min(uint64_t(r.y), ce);
      if (cs > cf || r.y < r.x) return;
      const uint32_t ws = uint32_t((cs - cb) >> 5), we = uint32_t((cf - cb) >> 5);
      const uint32_t lo = ~0u << (cs & 31);
      const uint32_t hi = ~0u >> (31 - (cf & 31));
      atomicOr(bits + ws, ws == we ? lo & hi : lo);
      if (ws != we) atomicMax(reach + ws, uint32_t(cf - cb) + 1u);
    });
    __syncwarp();
    uint32_t run_reach = 0;
    for (uint32_t wb = 0; wb < nwc; wb += 32) {
      const uint32_t w = wb + lane;
      const bool valid = w < nwc;
      uint32_t x = 0, rr = 0;
      if (valid) {
        x = bits[w];
        rr = reach[w];
      }
      const uint32_t cov = reach_cover(w, rr, run_reach, lane);
      if (valid) x |= cov;
      if (nnz) *nnz += __popc(x);
      const uint32_t last = min(31u, nwc - 1 - wb);
      count += gather_chunk(x, valid, cb + 32ull * w, 32, lane, kFullMask, carry, count, last, emit);
    }
    __syncwarp();
  }
  return count;
}

}  // namespace
}  // namespace dvg
