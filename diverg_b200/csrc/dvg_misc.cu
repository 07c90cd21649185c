// dvg_misc.cu -- the streaming kernels of the path: identity, input
// validation, rowmap width conversion, the rowmap scan, range SpAdd and the
// batched membership query.
#include <algorithm>

#include "dvg_device.cuh"
#include "dvg_internal.h"

namespace dvg {
namespace {

constexpr int kThreads = 256;

unsigned grid_for(dvg_context* ctx, uint64_t work, int per_block, int per_sm = 8) {
  uint64_t want = (work + per_block - 1) / per_block;
  uint64_t cap = uint64_t(ctx->num_sms) * per_sm;
  return unsigned(std::max<uint64_t>(1, std::min(want, cap)));
}

// ---- identity: create_range_identity_matrix, range_sparse.hpp:66-88 -------
__global__ void k_identity(uint64_t* __restrict__ rowmap, uint32_t* __restrict__ entries, uint32_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    reinterpret_cast<uint2*>(entries)[i] = make_uint2(uint32_t(i), uint32_t(i));
    rowmap[i + 1] = 2 * (i + 1);
    if (i == 0) rowmap[0] = 0;
  }
}

// ---- validation: the memory-safety preconditions of every kernel ----------
// bit 1: rowmap[0] != 0; bit 2: rowmap decreasing or odd row length;
// bit 4: rowmap[n] != nentries; bit 8: an entry >= ncols.  Not an error:
// bit 16 marks a matrix whose rows are not canonical (a range with end <
// start, or a range that does not start past the previous range's end + 1).
__global__ void k_validate(const uint64_t* __restrict__ rowmap, uint32_t nrows, const uint32_t* __restrict__ entries,
                           uint64_t nentries, uint32_t ncols, DeviceControl* ctl) {
  unsigned long long bad = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  for (uint64_t i = tid; i < nrows; i += stride) {
    uint64_t a = rowmap[i], b = rowmap[i + 1];
    if (b < a || ((b - a) & 1)) {
      bad |= 2;
    } else if (b <= nentries) {
      for (uint64_t k = a; k < b; k += 2) {
        if (entries[k + 1] < entries[k] || (k > a && uint64_t(entries[k]) <= uint64_t(entries[k - 1]) + 1))
          bad |= 16;
      }
    }
  }
  if (tid == 0) {
    if (rowmap[0] != 0) bad |= 1;
    if (rowmap[nrows] != nentries) bad |= 4;
  }
  for (uint64_t i = tid; i < nentries; i += stride)
    if (entries[i] >= ncols) bad |= 8;
  if (bad) atomicOr(&ctl->invalid, bad);
}

__global__ void k_widen(const uint32_t* __restrict__ src, uint64_t* __restrict__ dst, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    dst[i] = src[i];
}

__global__ void k_narrow(const uint64_t* __restrict__ src, uint32_t* __restrict__ dst, uint64_t n) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    dst[i] = uint32_t(src[i]);
}

// ---- scan: rowmap[1..n] inclusive, in three passes (tile sums, tile
// prefixes, apply) so no kernel waits on another CTA -------------------------
constexpr int kScanItems = 16;
constexpr int kScanTile = kThreads * kScanItems;

template <class T>
__device__ T block_excl_scan(T v, T* warp_sums, T* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(kFullMask, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (warp == 0) {
    T s = lane < nw ? warp_sums[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T u = __shfl_up_sync(kFullMask, s, o);
      if (lane >= o) s += u;
    }
    if (lane < nw) warp_sums[lane] = s;  // inclusive per warp
  }
  __syncthreads();
  T base = warp ? warp_sums[warp - 1] : T(0);
  if (total) *total = warp_sums[nw - 1];
  T r = base + incl - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kThreads) k_scan_reduce(const uint64_t* __restrict__ data, uint64_t n,
                                                          uint64_t* __restrict__ tile_sums) {
  __shared__ uint64_t ws[32];
  const uint64_t base = uint64_t(blockIdx.x) * kScanTile;
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint64_t i = base + uint64_t(k) * kThreads + threadIdx.x;
    if (i < n) s += data[i];
  }
  uint64_t total;
  block_excl_scan<uint64_t>(s, ws, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_tiles(uint64_t* __restrict__ tile_sums, uint64_t nt) {
  __shared__ uint64_t ws[32];
  const uint64_t per = (nt + blockDim.x - 1) / blockDim.x;
  const uint64_t b = threadIdx.x * per, e = std::min<uint64_t>(nt, b + per);
  uint64_t s = 0;
  for (uint64_t i = b; i < e; ++i) s += tile_sums[i];
  uint64_t run = block_excl_scan<uint64_t>(s, ws, nullptr);
  for (uint64_t i = b; i < e; ++i) {
    uint64_t v = tile_sums[i];
    tile_sums[i] = run;  // exclusive prefix of the tile
    run += v;
  }
}

__global__ void __launch_bounds__(kThreads) k_scan_apply(uint64_t* __restrict__ data, uint64_t n,
                                                         const uint64_t* __restrict__ tile_prefix) {
  __shared__ uint64_t tile[kScanTile];
  __shared__ uint64_t ws[32];
  const uint64_t base = uint64_t(blockIdx.x) * kScanTile;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint64_t i = base + uint64_t(k) * kThreads + threadIdx.x;
    tile[k * kThreads + threadIdx.x] = i < n ? data[i] : 0;
  }
  __syncthreads();
  uint64_t v[kScanItems];
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s += tile[threadIdx.x * kScanItems + k];
    v[k] = s;
  }
  uint64_t pre = block_excl_scan<uint64_t>(s, ws, nullptr) + tile_prefix[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) tile[threadIdx.x * kScanItems + k] = v[k] + pre;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint64_t i = base + uint64_t(k) * kThreads + threadIdx.x;
    if (i < n) data[i] = tile[k * kThreads + threadIdx.x];
  }
}

// ---- SpAdd: range_spadd_symbolic / _numeric, range_sparse.hpp:145-224 and
// :273-356.  One thread per row merges the two sorted range lists, merging a
// range whose start is <= hi + 1 into the open one; after one list runs out
// the other is merged up to its first non-merging range and copied verbatim
// from there, exactly as the reference does. --------------------------------
template <class Emit>
__device__ __forceinline__ void spadd_row(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb,
                                          Emit&& emit) {
  uint64_t ai = 0, bi = 0;
  if (ai < na && bi < nb) {
    uint32_t lo, hi;
    if (a[ai] <= b[bi]) { lo = a[ai]; hi = a[ai + 1]; ai += 2; }
    else { lo = b[bi]; hi = b[bi + 1]; bi += 2; }
    while (ai < na && bi < nb) {
      uint32_t rs, re;
      if (a[ai] <= b[bi]) { rs = a[ai]; re = a[ai + 1]; ai += 2; }
      else { rs = b[bi]; re = b[bi + 1]; bi += 2; }
      if (uint64_t(rs) <= uint64_t(hi) + 1) { lo = min(lo, rs); hi = max(hi, re); continue; }
      emit(lo, hi);
      lo = rs; hi = re;
    }
    while (ai < na || bi < nb) {
      uint32_t rs, re;
      if (ai == na) { rs = b[bi]; re = b[bi + 1]; bi += 2; }
      else { rs = a[ai]; re = a[ai + 1]; ai += 2; }
      if (uint64_t(rs) <= uint64_t(hi) + 1) { lo = min(lo, rs); hi = max(hi, re); continue; }
      emit(lo, hi);
      lo = rs; hi = re;
      break;
    }
    emit(lo, hi);
  }
  for (; ai < na; ai += 2) emit(a[ai], a[ai + 1]);
  for (; bi < nb; bi += 2) emit(b[bi], b[bi + 1]);
}

struct SpaddArgs {
  const uint64_t* __restrict__ a_rowmap;
  const uint32_t* __restrict__ a_entries;
  const uint64_t* __restrict__ b_rowmap;
  const uint32_t* __restrict__ b_entries;
  uint64_t* __restrict__ c_rowmap;
  uint32_t* __restrict__ c_entries;
  DeviceControl* ctl;
  uint32_t nrows;
};

template <bool B_IDENTITY, bool FILL>
__global__ void __launch_bounds__(kThreads) k_spadd(SpaddArgs p) {
  __shared__ unsigned long long cta_nnz;
  if (threadIdx.x == 0) cta_nnz = 0;
  __syncthreads();
  unsigned long long my_nnz = 0;
  for (uint64_t r = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; r < p.nrows;
       r += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t a0 = p.a_rowmap[r], a1 = p.a_rowmap[r + 1];
    uint32_t id[2] = {uint32_t(r), uint32_t(r)};
    const uint32_t* b;
    uint64_t nb;
    if constexpr (B_IDENTITY) {
      b = id;
      nb = 2;
    } else {
      b = p.b_entries + p.b_rowmap[r];
      nb = p.b_rowmap[r + 1] - p.b_rowmap[r];
    }
    if constexpr (FILL) {
      uint64_t pos = p.c_rowmap[r];
      const uint64_t end = p.c_rowmap[r + 1];
      spadd_row(p.a_entries + a0, a1 - a0, b, nb, [&](uint32_t lo, uint32_t hi) {
        if (pos + 2 <= end) {
          p.c_entries[pos] = lo;
          p.c_entries[pos + 1] = hi;
        } else {
          atomicOr(&p.ctl->status, 4ull);
        }
        pos += 2;
      });
    } else {
      uint64_t cnt = 0;
      spadd_row(p.a_entries + a0, a1 - a0, b, nb, [&](uint32_t lo, uint32_t hi) {
        cnt += 2;
        my_nnz += uint64_t(hi) - lo + 1;
      });
      p.c_rowmap[r + 1] = cnt;
    }
  }
  if constexpr (!FILL) {
    atomicAdd(&cta_nnz, my_nnz);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&p.ctl->nnz, cta_nnz);
  }
}

// ---- SpAdd in one pass ----------------------------------------------------------
// The same rows as k_spadd (the merge of spadd_row), with no counting pass and
// no scan: a persistent CTA takes chunks of kAddThreads rows from a ticket,
// copies the chunk's row pointers and ranges of A and B -- contiguous in HBM --
// into shared memory with asynchronous copies, merges a row per thread
// (count), takes the chunk-local prefix, publishes the chunk's entry count
// for later chunks' look-backs and merges again into a shared image of the
// chunk's output.  The image waits in shared memory (two buffers) and is
// resolved one iteration later: by then the chunks before it have long
// published their counts, so its decoupled look-back rarely waits, and it is
// written out with coalesced stores.  Rows whose ranges lie past the stages
// read HBM; a chunk whose output exceeds its image buffer is resolved and
// written straight to C in its own iteration.  Reads A and B once, writes C
// once.
constexpr int kAddThreads = 128;
constexpr int kAddStage = 6 * kAddThreads;   // ranges of each operand staged per chunk
constexpr int kAddImage = 16 * kAddThreads;  // output entries of a chunk held in an image buffer
constexpr unsigned long long kAddFlag = 1ull << 63;
constexpr uint32_t kAddSpinLimit = 1u << 22;

struct AddSmem {
  uint2 a[kAddStage];
  uint2 b[kAddStage];
  uint2 img[2][kAddImage / 2];            // images of the counted and the pending chunk (ranges)
  uint32_t incl[2][kAddThreads];          // their chunk-local inclusive row counts
  unsigned long long arow[kAddThreads + 1];  // the chunk's row pointers (entry offsets)
  unsigned long long brow[kAddThreads + 1];
  uint32_t wsum[kAddThreads / 32];
  unsigned long long wnnz[kAddThreads / 32];
  unsigned long long prefix[2];           // exclusive prefixes: the pending chunk's, a chunk written in place
  // the pending chunk (in buffer k), per buffer: its readers and the writer of
  // the next one never meet on one slot
  uint32_t pend_t[2], pend_rows[2], pend_cnt[2];
  uint32_t next;
};

// barrier.sync in its non-aligned form: the lanes of a warp leave the row
// merges at different times
__device__ __forceinline__ void add_sync() { asm volatile("barrier.sync 0;" ::: "memory"); }
__device__ __forceinline__ void add_cp8(void* smem, const void* gmem) {
  const uint32_t sa = uint32_t(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void add_cp_wait() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_all;" ::: "memory");
}

struct SpaddChunkArgs {
  const uint64_t* __restrict__ a_rowmap;
  const uint32_t* __restrict__ a_entries;
  const uint64_t* __restrict__ b_rowmap;
  const uint32_t* __restrict__ b_entries;
  uint64_t* __restrict__ c_rowmap;
  uint32_t* __restrict__ c_entries;
  unsigned long long* desc;  // per chunk: aggregate, inclusive prefix (flag | value words)
  unsigned* ticket;
  DeviceControl* ctl;
  uint64_t cap;              // entries C can hold
  uint32_t nrows, nchunks;
  uint32_t spin_limit;       // polls a look-back waits before it gives up (0: kAddSpinLimit)
};

// Warp 0 walks back from chunk t (whose aggregate is published) to the
// nearest inclusive prefix, publishes t's inclusive prefix and leaves t's
// exclusive prefix in *out (shared); the caller's barrier makes it visible.
__device__ void add_lookback(unsigned long long* out, const SpaddChunkArgs& p, uint32_t t, uint32_t cnt) {
  const int lane = threadIdx.x & 31;
  unsigned long long pre = 0;
  int64_t j = int64_t(t) - 1;
  uint32_t spins = 0;
  const uint32_t limit = p.spin_limit ? p.spin_limit : kAddSpinLimit;
  while (j >= 0) {
    const int64_t idx = j - lane;
    int st = 2;  // 2: inclusive prefix (or before chunk 0), 1: aggregate, 0: nothing yet
    unsigned long long v = 0;
    if (idx >= 0) {
      unsigned long long va, vi;
      asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];"
                   : "=l"(va), "=l"(vi) : "l"(p.desc + 2 * size_t(idx)) : "memory");
      if (vi & kAddFlag) {
        v = vi & ~kAddFlag;
      } else if (va & kAddFlag) {
        st = 1;
        v = va & ~kAddFlag;
      } else {
        st = 0;
      }
    }
    const unsigned im = __ballot_sync(kFullMask, st == 2), wm = __ballot_sync(kFullMask, st == 0);
    const int fi = im ? __ffs(im) - 1 : 32;
    const unsigned before = fi == 32 ? kFullMask : ((1u << fi) - 1u);
    if (wm & before) {
      if (++spins > limit) {
        if (lane == 0) atomicOr(&p.ctl->timeout, 1ull);  // the wait ran out
        break;
      }
      __nanosleep(32);
      continue;
    }
    unsigned long long sv = lane <= fi ? v : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sv += __shfl_xor_sync(kFullMask, sv, o);
    pre += sv;
    if (fi < 32) break;
    j -= 32;
  }
  if (lane == 0) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p.desc + 2 * size_t(t) + 1), "l"(kAddFlag | (pre + cnt))
                 : "memory");
    *out = pre;
    if (t == p.nchunks - 1) p.ctl->total = pre + cnt;
  }
}

template <bool B_ID>
__global__ void __launch_bounds__(kAddThreads) k_spadd_chunks(SpaddChunkArgs p) {
  extern __shared__ __align__(16) unsigned char add_smem_raw[];
  AddSmem& S = *reinterpret_cast<AddSmem*>(add_smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned long long nnz_cta = 0;
  if (tid == 0) S.next = atomicAdd(p.ticket, 1u);
  add_sync();
  uint32_t t = S.next, b = 0;
  bool pend = false;  // a counted chunk waits in image buffer b ^ 1
  while (t < p.nchunks || pend) {
    const bool have = t < p.nchunks;
    const uint32_t c0 = have ? t * uint32_t(kAddThreads) : 0u;
    const uint32_t crows = have ? min(uint32_t(kAddThreads), p.nrows - c0) : 0u;
    uint32_t cnt = 0, excl = 0, cnt_r = 0;
    bool imaged = false;
    const uint2* ap = nullptr;
    const uint2* bp = nullptr;
    uint32_t na = 0, nb = 0;  // ranges of this thread's row
    uint2 id;
    const uint32_t r = tid;
    const bool has = r < crows;
    if (have) {
      // 1. the chunk's row pointers
      for (uint32_t k = tid; k <= crows; k += kAddThreads) {
        add_cp8(&S.arow[k], p.a_rowmap + uint64_t(c0) + k);
        if (!B_ID) add_cp8(&S.brow[k], p.b_rowmap + uint64_t(c0) + k);
      }
      add_cp_wait();
      add_sync();
      const uint64_t abase = S.arow[0], bbase = B_ID ? 0 : S.brow[0];
      const uint64_t ra = (S.arow[crows] - abase) / 2, rb = B_ID ? 0 : (S.brow[crows] - bbase) / 2;
      const uint32_t nas = ra < uint64_t(kAddStage) ? uint32_t(ra) : uint32_t(kAddStage);
      const uint32_t nbs = rb < uint64_t(kAddStage) ? uint32_t(rb) : uint32_t(kAddStage);
      // 2. their ranges (rows start at even entries: a range is one 8-byte copy)
      for (uint32_t k = tid; k < nas; k += kAddThreads) add_cp8(&S.a[k], p.a_entries + abase + 2 * uint64_t(k));
      if (!B_ID)
        for (uint32_t k = tid; k < nbs; k += kAddThreads) add_cp8(&S.b[k], p.b_entries + bbase + 2 * uint64_t(k));
      add_cp_wait();
      add_sync();
      // 3. count this thread's row
      if (has) {
        const uint64_t a0 = (S.arow[r] - abase) / 2, a1 = (S.arow[r + 1] - abase) / 2;
        na = uint32_t(a1 - a0);
        ap = a1 <= nas ? S.a + a0 : reinterpret_cast<const uint2*>(p.a_entries + abase) + a0;
        if (B_ID) {
          id = make_uint2(c0 + r, c0 + r);
          bp = &id;
          nb = 1;
        } else {
          const uint64_t b0 = (S.brow[r] - bbase) / 2, b1 = (S.brow[r + 1] - bbase) / 2;
          nb = uint32_t(b1 - b0);
          bp = b1 <= nbs ? S.b + b0 : reinterpret_cast<const uint2*>(p.b_entries + bbase) + b0;
        }
        spadd_row(reinterpret_cast<const uint32_t*>(ap), 2ull * na, reinterpret_cast<const uint32_t*>(bp), 2ull * nb, [&](uint32_t lo, uint32_t hi) {
          cnt_r += 2;
          nnz_cta += uint64_t(hi - lo) + 1;
        });
      }
      // 4. chunk-local prefix; the aggregate for later chunks at once
      uint32_t incl = cnt_r;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(kFullMask, incl, o);
        if (lane >= o) incl += u;
      }
      if (lane == 31) S.wsum[warp] = incl;
      add_sync();
      uint32_t wpre = 0;
#pragma unroll
      for (int w = 0; w < kAddThreads / 32; ++w) {
        const uint32_t v = S.wsum[w];
        if (w < warp) wpre += v;
        cnt += v;
      }
      excl = wpre + incl - cnt_r;
      if (tid == 0) {
        asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p.desc + 2 * size_t(t)), "l"(kAddFlag | cnt)
                     : "memory");
        S.next = atomicAdd(p.ticket, 1u);  // the next chunk, taken once this one is counted
      }
      // 5. the chunk's image in buffer b (its inclusive row counts beside it)
      imaged = cnt <= uint32_t(kAddImage);
      if (imaged) {
        S.incl[b][r] = excl + cnt_r;
        if (has)
          spadd_row(reinterpret_cast<const uint32_t*>(ap), 2ull * na, reinterpret_cast<const uint32_t*>(bp), 2ull * nb, [&, k = excl / 2](uint32_t lo, uint32_t hi) mutable {
            S.img[b][k++] = make_uint2(lo, hi);
          });
      }
    }
    // 6. the pending chunk (counted last iteration): look-back, row map, entries
    if (pend) {
      const uint32_t pt = S.pend_t[b ^ 1u], prow = S.pend_rows[b ^ 1u], pcnt = S.pend_cnt[b ^ 1u];
      if (warp == 0) add_lookback(&S.prefix[0], p, pt, pcnt);
      add_sync();
      const unsigned long long prefix = S.prefix[0];
      if (uint32_t(tid) < prow) p.c_rowmap[uint64_t(pt) * kAddThreads + tid + 1] = prefix + S.incl[b ^ 1u][tid];
      if (pt == 0 && tid == 0) p.c_rowmap[0] = 0;
      if (prefix + pcnt <= p.cap) {
        uint2* dst = reinterpret_cast<uint2*>(p.c_entries + prefix);  // prefix is even: 8-byte aligned
        for (uint32_t k = tid; k < pcnt / 2; k += kAddThreads) dst[k] = S.img[b ^ 1u][k];
      } else if (tid == 0 && pcnt) {
        atomicOr(&p.ctl->overflow, 1ull);
      }
      pend = false;
    }
    // 7. a chunk whose output does not fit its image: resolved now, in place
    if (have && !imaged) {
      if (warp == 0) add_lookback(&S.prefix[1], p, t, cnt);
      add_sync();
      const unsigned long long prefix = S.prefix[1];
      if (has) p.c_rowmap[uint64_t(c0) + r + 1] = prefix + excl + cnt_r;
      if (t == 0 && tid == 0) p.c_rowmap[0] = 0;
      if (prefix + cnt > p.cap) {
        if (tid == 0 && cnt) atomicOr(&p.ctl->overflow, 1ull);
      } else if (has) {
        uint32_t* dst = p.c_entries + prefix + excl;
        spadd_row(reinterpret_cast<const uint32_t*>(ap), 2ull * na, reinterpret_cast<const uint32_t*>(bp), 2ull * nb, [&, k = 0u](uint32_t lo, uint32_t hi) mutable {
          dst[k] = lo;
          dst[k + 1] = hi;
          k += 2;
        });
      }
    }
    if (have && imaged) {
      if (tid == 0) {
        S.pend_t[b] = t;
        S.pend_rows[b] = crows;
        S.pend_cnt[b] = cnt;
      }
      pend = true;
      b ^= 1u;
    }
    // every thread is done with the stages and the images it needs; S.next
    // (written after the prefix) and the pending record are visible
    add_sync();
    t = have ? S.next : 0xffffffffu;
  }
  // the product's nnz: one atomic per CTA
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nnz_cta += __shfl_xor_sync(kFullMask, nnz_cta, o);
  if (lane == 0) S.wnnz[warp] = nnz_cta;
  add_sync();
  if (tid == 0) {
    unsigned long long s = 0;
    for (int w = 0; w < kAddThreads / 32; ++w) s += S.wnnz[w];
    atomicAdd(&p.ctl->nnz, s);
  }
}

// ---- query: crs_matrix::binary_search(..., RangeGroup), crs_matrix.hpp:
// 149-169, one thread per pair ------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_query(const uint64_t* __restrict__ rowmap,
                                                    const uint32_t* __restrict__ entries, uint32_t nrows,
                                                    uint32_t ncols, uint64_t nentries,
                                                    const uint2* __restrict__ pairs, uint64_t npairs,
                                                    uint8_t* __restrict__ out, DeviceControl* ctl) {
  unsigned long long bad = 0;
  bool corrupt = false;
  for (uint64_t q = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; q < npairs;
       q += uint64_t(gridDim.x) * blockDim.x) {
    uint2 ij = pairs[q];
    uint8_t ans = 0;
    if (ij.x < nrows && ij.y < ncols) {
      uint64_t lo = __ldg(rowmap + ij.x), hi = __ldg(rowmap + ij.x + 1);
      if (lo > hi || hi > nentries) {  // row pointers outside the entries: never read past them
        corrupt = true;
        lo = hi = 0;
      }
      uint64_t first = lo, len = hi - lo;
      while (len > 0) {
        uint64_t half = len >> 1;
        if (__ldg(entries + first + half) < ij.y) {
          first += half + 1;
          len -= half + 1;
        } else {
          len = half;
        }
      }
      if ((first - lo) & 1) --first;
      ans = (first != hi && __ldg(entries + first) <= ij.y) ? 1 : 0;
    } else {
      ++bad;
    }
    out[q] = ans;
  }
  if (bad) atomicAdd(&ctl->invalid, bad);
  if (corrupt) atomicOr(&ctl->status, kQueryCorrupt);
}

// Four consecutive pairs a thread, their loads interleaved: the pairs (two
// 16-byte loads), the four rows' bounds, then -- for rows of at most two
// ranges, nearly all rows of an index -- each row's entries in two 8-byte
// loads, searched in registers by the same binary search as k_query (so the
// answers are the same on any row, sorted or not); longer rows search HBM.
// The four answers go out as one 4-byte store.
__device__ __forceinline__ uint32_t pick4(uint2 e0, uint2 e1, uint64_t k) {
  return k == 0 ? e0.x : k == 1 ? e0.y : k == 2 ? e1.x : e1.y;
}

__global__ void __launch_bounds__(kThreads) k_query4(const uint64_t* __restrict__ rowmap,
                                                     const uint32_t* __restrict__ entries, uint32_t nrows,
                                                     uint32_t ncols, uint64_t nentries,
                                                     const uint4* __restrict__ pairs, uint64_t ngroups,
                                                     uchar4* __restrict__ out, DeviceControl* ctl) {
  unsigned long long bad = 0;
  bool corrupt = false;
  for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < ngroups;
       g += uint64_t(gridDim.x) * blockDim.x) {
    const uint4 p01 = __ldg(pairs + 2 * g), p23 = __ldg(pairs + 2 * g + 1);
    const uint32_t qi[4] = {p01.x, p01.z, p23.x, p23.z}, qj[4] = {p01.y, p01.w, p23.y, p23.w};
    bool ok[4];
    uint64_t lo[4], hi[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      ok[k] = qi[k] < nrows && qj[k] < ncols;
      bad += ok[k] ? 0 : 1;
      lo[k] = ok[k] ? __ldg(rowmap + qi[k]) : 0;
      hi[k] = ok[k] ? __ldg(rowmap + qi[k] + 1) : 0;
      if (lo[k] > hi[k] || hi[k] > nentries) {  // row pointers outside the entries: never read past them
        corrupt = true;
        lo[k] = hi[k] = 0;
      }
    }
    uint2 e0[4], e1[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint64_t len = hi[k] - lo[k];
      e0[k] = e1[k] = make_uint2(0u, 0u);
      if (len > 0 && len <= 4) {
        e0[k] = __ldg(reinterpret_cast<const uint2*>(entries + lo[k]));
        if (len > 2) e1[k] = __ldg(reinterpret_cast<const uint2*>(entries + lo[k] + 2));
      }
    }
    uint8_t ans[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint64_t n = hi[k] - lo[k];
      const uint32_t j = qj[k];
      uint64_t first = 0, len = n;
      if (n <= 4) {
        while (len > 0) {
          const uint64_t half = len >> 1;
          if (pick4(e0[k], e1[k], first + half) < j) {
            first += half + 1;
            len -= half + 1;
          } else {
            len = half;
          }
        }
        if (first & 1) --first;
        ans[k] = (first != n && pick4(e0[k], e1[k], first) <= j) ? 1 : 0;
      } else {
        const uint32_t* e = entries + lo[k];
        while (len > 0) {
          const uint64_t half = len >> 1;
          if (__ldg(e + first + half) < j) {
            first += half + 1;
            len -= half + 1;
          } else {
            len = half;
          }
        }
        if (first & 1) --first;
        ans[k] = (first != n && __ldg(e + first) <= j) ? 1 : 0;
      }
      if (!ok[k]) ans[k] = 0;
    }
    out[g] = make_uchar4(ans[0], ans[1], ans[2], ans[3]);
  }
  if (bad) atomicAdd(&ctl->invalid, bad);
  if (corrupt) atomicOr(&ctl->status, kQueryCorrupt);
}

// ---- random reads: the denominator of the query's roofline -------------------
// Independent 8-byte reads at uniformly random word addresses of a buffer,
// kRandReads a thread in flight at once: each touches one DRAM sector, as a
// membership query's row-pointer and range reads do.  Addresses are
// SplitMix64 (Steele, Lea and Flood) of the read's index, scaled into
// [0, nwords) by the high half of a 64 x 64-bit product.
constexpr int kRandReads = 16;

__global__ void __launch_bounds__(kThreads) k_random_reads(const uint64_t* __restrict__ buf, uint64_t nwords,
                                                           uint64_t nthreads, unsigned long long* sink) {
  uint64_t acc = 0;
  for (uint64_t g = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; g < nthreads;
       g += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t v[kRandReads];
#pragma unroll
    for (int k = 0; k < kRandReads; ++k) {
      uint64_t z = (g * kRandReads + uint64_t(k) + 1) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      v[k] = __ldg(buf + __umul64hi(z, nwords));
    }
#pragma unroll
    for (int k = 0; k < kRandReads; ++k) acc ^= v[k];
  }
  // keeps the reads observable: one atomic a warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc ^= __shfl_xor_sync(kFullMask, acc, o);
  if ((threadIdx.x & 31) == 0) atomicXor(sink, acc);
}

}  // namespace

double calibrate_random_reads(dvg_context* ctx, uint64_t bytes) {
  const uint64_t nwords = std::max<uint64_t>(bytes / 8, 1u << 20);
  const uint64_t nthreads = uint64_t(1) << 22;  // 2^26 reads a launch
  void* mem = dalloc(ctx, nwords * 8 + 256);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float best = 0.f;
  try {
    auto* buf = static_cast<uint64_t*>(mem);
    auto* sink = reinterpret_cast<unsigned long long*>(static_cast<char*>(mem) + nwords * 8);
    DVG_CUDA(cudaMemsetAsync(mem, 0, nwords * 8 + 8, ctx->stream));
    DVG_CUDA(cudaEventCreate(&e0));
    DVG_CUDA(cudaEventCreate(&e1));
    const unsigned grid = grid_for(ctx, nthreads, kThreads);
    for (int rep = 0; rep < 4; ++rep) {  // the first is a warm-up; the best of the rest
      DVG_CUDA(cudaEventRecord(e0, ctx->stream));
      k_random_reads<<<grid, kThreads, 0, ctx->stream>>>(buf, nwords, nthreads, sink);
      DVG_CUDA(cudaGetLastError());
      DVG_CUDA(cudaEventRecord(e1, ctx->stream));
      DVG_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      DVG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    ctx->stats.kernel_launches += 4;
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    dfree(ctx, mem);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dfree(ctx, mem);
  return best > 0.f ? double(nthreads) * kRandReads / (double(best) * 1e-3) : 0.0;
}

void launch_identity(dvg_context* ctx, dvg_matrix* out) {
  if (out->nrows == 0) {
    DVG_CUDA(cudaMemsetAsync(out->rowmap, 0, sizeof(uint64_t), ctx->stream));
    return;
  }
  k_identity<<<grid_for(ctx, out->nrows, kThreads), kThreads, 0, ctx->stream>>>(out->rowmap, out->entries,
                                                                                out->nrows);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

void launch_validate(dvg_context* ctx, const uint64_t* rowmap, uint32_t nrows, const uint32_t* entries,
                     uint64_t nentries, uint32_t ncols) {
  k_validate<<<grid_for(ctx, std::max<uint64_t>(nrows, nentries) + 1, kThreads), kThreads, 0, ctx->stream>>>(
      rowmap, nrows, entries, nentries, ncols, ctx->d_ctl);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

void launch_widen_rowmap(dvg_context* ctx, const uint32_t* src, uint64_t* dst, uint64_t n) {
  k_widen<<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>(src, dst, n);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

void launch_narrow_rowmap(dvg_context* ctx, const uint64_t* src, uint32_t* dst, uint64_t n) {
  k_narrow<<<grid_for(ctx, n, kThreads), kThreads, 0, ctx->stream>>>(src, dst, n);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

void launch_rowmap_scan(dvg_context* ctx, uint64_t* rowmap, uint64_t n) {
  if (n == 0) return;
  uint64_t* data = rowmap + 1;
  const uint64_t nt = (n + kScanTile - 1) / kScanTile;
  if (nt > ctx->tile_sums_cap) {
    if (ctx->d_tile_sums) dfree(ctx, ctx->d_tile_sums);
    ctx->d_tile_sums = nullptr;
    ctx->tile_sums_cap = 0;
    ctx->d_tile_sums = static_cast<uint64_t*>(dalloc(ctx, nt * sizeof(uint64_t)));
    ctx->tile_sums_cap = nt;
  }
  k_scan_reduce<<<unsigned(nt), kThreads, 0, ctx->stream>>>(data, n, ctx->d_tile_sums);
  DVG_CUDA(cudaGetLastError());
  k_scan_tiles<<<1, 1024, 0, ctx->stream>>>(ctx->d_tile_sums, nt);
  DVG_CUDA(cudaGetLastError());
  k_scan_apply<<<unsigned(nt), kThreads, 0, ctx->stream>>>(data, n, ctx->d_tile_sums);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches += 3;
}

void launch_spadd(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, bool b_identity, uint64_t* c_rowmap,
                  uint32_t* c_entries, bool fill) {
  if (a->nrows == 0) return;
  SpaddArgs p{};
  p.a_rowmap = a->rowmap;
  p.a_entries = a->entries;
  p.b_rowmap = b_identity ? nullptr : b->rowmap;
  p.b_entries = b_identity ? nullptr : b->entries;
  p.c_rowmap = c_rowmap;
  p.c_entries = c_entries;
  p.ctl = ctx->d_ctl;
  p.nrows = a->nrows;
  const unsigned grid = grid_for(ctx, a->nrows, kThreads);
  if (b_identity) {
    if (fill) k_spadd<true, true><<<grid, kThreads, 0, ctx->stream>>>(p);
    else k_spadd<true, false><<<grid, kThreads, 0, ctx->stream>>>(p);
  } else {
    if (fill) k_spadd<false, true><<<grid, kThreads, 0, ctx->stream>>>(p);
    else k_spadd<false, false><<<grid, kThreads, 0, ctx->stream>>>(p);
  }
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

uint64_t spadd_single_pass_scratch(uint32_t nrows) {
  const uint64_t nchunks = (uint64_t(nrows) + kAddThreads - 1) / kAddThreads;
  return nchunks * 16 + 256;
}

void launch_spadd_single_pass(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, bool b_identity,
                              uint64_t* c_rowmap, uint32_t* c_entries, uint64_t cap, void* scratch) {
  const uint32_t n = a->nrows;
  if (n == 0) return;
  const uint32_t nchunks = uint32_t((uint64_t(n) + kAddThreads - 1) / kAddThreads);
  // per chunk 16 bytes of descriptors, then the ticket
  DVG_CUDA(cudaMemsetAsync(scratch, 0, spadd_single_pass_scratch(n), ctx->stream));
  SpaddChunkArgs p{};
  p.a_rowmap = a->rowmap;
  p.a_entries = a->entries;
  p.b_rowmap = b_identity ? nullptr : b->rowmap;
  p.b_entries = b_identity ? nullptr : b->entries;
  p.c_rowmap = c_rowmap;
  p.c_entries = c_entries;
  p.desc = static_cast<unsigned long long*>(scratch);
  p.ticket = reinterpret_cast<unsigned*>(static_cast<char*>(scratch) + size_t(nchunks) * 16);
  p.ctl = ctx->d_ctl;
  p.cap = cap;
  p.nrows = n;
  p.nchunks = nchunks;
  const int smem = int(sizeof(AddSmem));
  DVG_CUDA(cudaFuncSetAttribute(k_spadd_chunks<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  DVG_CUDA(cudaFuncSetAttribute(k_spadd_chunks<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int per_sm = 0;
  DVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spadd_chunks<false>, kAddThreads, smem));
  const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(nchunks, uint64_t(std::max(per_sm, 1)) * ctx->num_sms)));
  if (b_identity) k_spadd_chunks<true><<<grid, kAddThreads, smem, ctx->stream>>>(p);
  else k_spadd_chunks<false><<<grid, kAddThreads, smem, ctx->stream>>>(p);
  DVG_CUDA(cudaGetLastError());
  ctx->stats.kernel_launches++;
}

void launch_query(dvg_context* ctx, const dvg_matrix* idx, const uint32_t* d_pairs, uint64_t npairs, uint8_t* d_out,
                  DeviceControl* ctl) {
  if (npairs == 0) return;
  DeviceControl* c = ctl ? ctl : ctx->d_ctl;
  // four pairs a thread when the buffers allow 16-byte pair loads and
  // 4-byte answer stores; the last npairs % 4 pairs (or all) one a thread
  uint64_t done = 0;
  const bool vec = ((reinterpret_cast<uintptr_t>(d_pairs) & 15u) | (reinterpret_cast<uintptr_t>(d_out) & 3u) |
                    (reinterpret_cast<uintptr_t>(idx->entries) & 7u)) == 0;
  if (vec && npairs >= 4) {
    const uint64_t groups = npairs / 4;
    k_query4<<<grid_for(ctx, groups, kThreads, 8), kThreads, 0, ctx->stream>>>(
        idx->rowmap, idx->entries, idx->nrows, idx->ncols, idx->nentries, reinterpret_cast<const uint4*>(d_pairs), groups,
        reinterpret_cast<uchar4*>(d_out), c);
    DVG_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
    done = 4 * groups;
  }
  if (done < npairs) {
    k_query<<<grid_for(ctx, npairs - done, kThreads, 16), kThreads, 0, ctx->stream>>>(
        idx->rowmap, idx->entries, idx->nrows, idx->ncols, idx->nentries, reinterpret_cast<const uint2*>(d_pairs) + done,
        npairs - done, d_out + done, c);
    DVG_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches++;
  }
}

}  // namespace dvg
