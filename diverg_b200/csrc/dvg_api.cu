// dvg_api.cu -- the C ABI of include/dvg.h and the host orchestration of the
// range operations: products, sums, powers and the distance index.  Every
// entry point converts internal failures into a dvg_status.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "dvg_internal.h"

namespace {
thread_local std::string g_last_error;

dvg_status fail(dvg_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

template <class F>
dvg_status guarded(F&& f) {
  try {
    f();
    return DVG_OK;
  } catch (const dvg::Error& e) {
    return fail(e.status, e.what());
  } catch (const std::bad_alloc&) {
    return fail(DVG_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(DVG_ERR_DEVICE, e.what());
  }
}

using dvg::require;

struct Lock {
  dvg_context* ctx;
  explicit Lock(dvg_context* c) : ctx(c) {
    require(c != nullptr, "null context");
    ctx->mu.lock();
    DVG_CUDA(cudaSetDevice(ctx->device));
  }
  ~Lock() { ctx->mu.unlock(); }
};
}  // namespace

namespace dvg {

void require(bool ok, const char* msg) {
  if (!ok) throw Error(DVG_ERR_INVALID_ARG, msg);
}

void record_error(const std::string& msg) { g_last_error = msg; }

void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  dvg_status s = (e == cudaErrorMemoryAllocation) ? DVG_ERR_OOM : DVG_ERR_DEVICE;
  throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
}

uint64_t now_ns() {
  return uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(
                      std::chrono::steady_clock::now().time_since_epoch()).count());
}

// Returns every cached block to the stream-ordered pool.
static void release_cached(dvg_context* ctx) {
  for (auto& kv : ctx->free_blocks) DVG_CUDA(cudaFreeAsync(kv.second, ctx->stream));
  ctx->free_blocks.clear();
  ctx->owned_bytes -= std::min(ctx->owned_bytes, ctx->cached_bytes);
  ctx->cached_bytes = 0;
}

// Device allocation for the context's stream.  A freed block whose size is
// within [bytes, bytes + bytes/4] is reused (best fit); otherwise the request
// goes to cudaMallocAsync, and when that fails the cache is released and the
// request retried once.  Re-mapping GB-sized buffers in the pool on every
// product costs tens to hundreds of milliseconds per index build.
// Allocation sizes are rounded up to classes -- 256-byte granules up to
// 1 MiB, above that quarter steps of a power of two (at most 25 % more) -- so
// the requests of differently sized builds meet in the cache instead of each
// growing the pool.
static size_t size_class(size_t bytes) {
  bytes = (std::max<size_t>(bytes, 16) + 255) & ~size_t(255);
  if (bytes <= (size_t(1) << 20)) return bytes;
  const int k = 63 - __builtin_clzll(uint64_t(bytes));
  const size_t step = size_t(1) << (k - 2);
  return (bytes + step - 1) & ~(step - 1);
}

void* dalloc(dvg_context* ctx, size_t bytes) {
  const uint64_t t0 = now_ns();
  bytes = size_class(bytes);
  auto it = ctx->free_blocks.lower_bound(bytes);
  if (it != ctx->free_blocks.end() && it->first <= bytes + bytes / 4) {
    void* p = it->second;
    ctx->live_blocks[p] = it->first;
    ctx->cached_bytes -= it->first;
    ctx->free_blocks.erase(it);
    ctx->stats.host_alloc_ns += now_ns() - t0;
    return p;
  }
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, ctx->stream);
  if (e == cudaErrorMemoryAllocation && !ctx->free_blocks.empty()) {
    (void)cudaGetLastError();
    release_cached(ctx);
    DVG_CUDA(cudaStreamSynchronize(ctx->stream));
    e = cudaMallocAsync(&p, bytes, ctx->stream);
  }
  ctx->stats.host_alloc_ns += now_ns() - t0;
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw Error(e == cudaErrorMemoryAllocation ? DVG_ERR_OOM : DVG_ERR_DEVICE,
                std::string("device allocation of ") + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
  }
  ctx->live_blocks[p] = bytes;
  ctx->owned_bytes += bytes;
  return p;
}

// Free device memory for planning.  cudaMemGetInfo is a driver round trip
// that has taken tens of milliseconds on a busy machine, so an answer is
// reused for up to a second, corrected by what this context has allocated
// or released since.  A plan sized on a stale answer fails its allocation
// and falls back like any other out-of-memory plan.
size_t device_free_bytes(dvg_context* ctx) {
  constexpr uint64_t kTtlNs = 1000000000ull;
  const uint64_t t0 = now_ns();
  if (ctx->mi_ns == 0 || t0 - ctx->mi_ns > kTtlNs) {
    size_t free_b = 0, total_b = 0;
    DVG_CUDA(cudaMemGetInfo(&free_b, &total_b));
    ctx->mi_ns = now_ns();
    ctx->stats.host_meminfo_ns += ctx->mi_ns - t0;
    ctx->mi_free = free_b;
    ctx->mi_owned = ctx->owned_bytes;
    return free_b;
  }
  const size_t grew = ctx->owned_bytes > ctx->mi_owned ? ctx->owned_bytes - ctx->mi_owned : 0;
  const size_t shrank = ctx->mi_owned > ctx->owned_bytes ? ctx->mi_owned - ctx->owned_bytes : 0;
  return grew >= ctx->mi_free + shrank ? 0 : ctx->mi_free + shrank - grew;
}

void dfree(dvg_context* ctx, void* p) {
  if (!p) return;
  auto it = ctx->live_blocks.find(p);
  if (it == ctx->live_blocks.end()) {
    DVG_CUDA(cudaFreeAsync(p, ctx->stream));
    return;
  }
  ctx->free_blocks.emplace(it->second, p);
  ctx->cached_bytes += it->second;
  ctx->live_blocks.erase(it);
}


dvg_matrix* new_matrix(dvg_context* ctx, uint32_t nrows, uint32_t ncols, uint64_t nentries) {
  auto* m = new dvg_matrix();
  m->nrows = nrows;
  m->ncols = ncols;
  m->nentries = nentries;
  m->device = ctx->device;
  try {
    m->rowmap = static_cast<uint64_t*>(dalloc(ctx, (size_t(nrows) + 1) * sizeof(uint64_t)));
    m->entries = static_cast<uint32_t*>(dalloc(ctx, entries_alloc_bytes(nentries)));
  } catch (...) {
    free_matrix(ctx, m);
    throw;
  }
  return m;
}

void free_matrix(dvg_context* ctx, dvg_matrix* m) {
  if (!m) return;
  if (m->owned) {
    dfree(ctx, m->rowmap);
    dfree(ctx, m->entries);
  }
  delete m;
}

static cudaEvent_t take_event(dvg_context* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  DVG_CUDA(cudaEventCreate(&e));
  return e;
}

cudaEvent_t span_begin(dvg_context* ctx) {
  if (!ctx->opt_timing) return nullptr;
  cudaEvent_t e = take_event(ctx);
  DVG_CUDA(cudaEventRecord(e, ctx->stream));
  return e;
}

void span_end(dvg_context* ctx, cudaEvent_t begin, TimedKind kind) {
  if (!begin) return;
  cudaEvent_t e = take_event(ctx);
  DVG_CUDA(cudaEventRecord(e, ctx->stream));
  ctx->timed.push_back({begin, e, int(kind)});
}

// After a stream synchronisation every recorded span has completed.
void resolve_spans(dvg_context* ctx) {
  for (auto& t : ctx->timed) {
    float ms = 0.f;
    DVG_CUDA(cudaEventElapsedTime(&ms, t.begin, t.end));
    uint64_t ns = uint64_t(double(ms) * 1e6);
    switch (t.kind) {
      case kProduct: ctx->stats.spgemm_ns += ns; break;
      case kLevels: ctx->stats.spgemm_levels_ns += ns; break;
      case kScan: ctx->stats.scan_ns += ns; break;
      case kQuery: ctx->stats.query_ns += ns; break;
      default: ctx->stats.spadd_ns += ns; break;
    }
    ctx->event_pool.push_back(t.begin);
    ctx->event_pool.push_back(t.end);
  }
  ctx->timed.clear();
}

void reset_control(dvg_context* ctx) {
  DVG_CUDA(cudaMemsetAsync(ctx->d_ctl, 0, sizeof(DeviceControl), ctx->stream));
}

DeviceControl read_control(dvg_context* ctx) {
  DVG_CUDA(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(DeviceControl), cudaMemcpyDeviceToHost, ctx->stream));
  const uint64_t t0 = now_ns();
  DVG_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->stats.host_sync_ns += now_ns() - t0;
  ctx->stats.host_syncs++;
  resolve_spans(ctx);
  DeviceControl c = *ctx->h_ctl;
  if (c.status) throw Error(DVG_ERR_DEVICE, "internal consistency check failed on the device (code " +
                                                std::to_string(c.status) + ")");
  return c;
}

// Reads rowmap[n] of a freshly scanned rowmap together with the control block.
static DeviceControl read_total(dvg_context* ctx, const uint64_t* rowmap_last, uint64_t* total) {
  uint64_t* h_total = reinterpret_cast<uint64_t*>(ctx->h_ctl + 1);
  DVG_CUDA(cudaMemcpyAsync(h_total, rowmap_last, sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream));
  DeviceControl c = read_control(ctx);
  *total = *h_total;
  return c;
}

// Mean A range length from which a product reads union levels of B.
constexpr double kLevelMean = 4.0;

// Union levels of b: level k row j = the union of b's rows j .. j + 2^k - 1,
// built as U_k = U_(k-1) + S U_(k-1) (S: identity shifted by 2^(k-1) rows).
// A union of two rows has at most their entries together, so the capacity is
// exact.
static std::vector<dvg_matrix*> build_levels(dvg_context* ctx, const dvg_matrix* b, uint32_t nlevels) {
  std::vector<dvg_matrix*> lv;
  try {
    const dvg_matrix* prev = b;
    for (uint32_t k = 1; k <= nlevels; ++k) {
      const uint64_t cap = 2 * prev->nentries + 64;
      dvg_matrix* c = new_matrix(ctx, b->nrows, b->ncols, cap);
      lv.push_back(c);
      DVG_CUDA(cudaMemsetAsync(c->rowmap, 0, sizeof(uint64_t), ctx->stream));
      reset_control(ctx);
      cudaEvent_t t0 = span_begin(ctx);
      launch_row_shifted_sum(ctx, prev, 1u << (k - 1), c->rowmap, c->entries, cap);
      span_end(ctx, t0, kLevels);
      const DeviceControl ctl = read_control(ctx);
      if (ctl.timeout) throw Error(DVG_ERR_TIMEOUT, "union levels: chunk look-back wait expired");
      if (ctl.overflow) throw Error(DVG_ERR_DEVICE, "union levels: capacity overflow");
      c->nentries = ctl.total;
      c->nnz = ctl.nnz;
      ctx->stats.spgemm_levels++;
      ctx->stats.alg_bytes += 2 * matrix_bytes(prev) + matrix_bytes(c);
      prev = c;
    }
  } catch (...) {
    for (dvg_matrix* m : lv) free_matrix(ctx, m);
    throw;
  }
  return lv;
}

static dvg_matrix* range_spgemm_fused(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b,
                                      const dvg_matrix* d = nullptr) {
  const uint32_t n = a_identity ? b->nrows : a->nrows;
  // long A ranges: walk union levels of B instead of every B row
  std::vector<dvg_matrix*> levels;
  struct LevelGuard {
    dvg_context* ctx;
    std::vector<dvg_matrix*>& lv;
    ~LevelGuard() {
      for (dvg_matrix* m : lv) free_matrix(ctx, m);
    }
  } level_guard{ctx, levels};
  if (!a_identity && !d && ctx->opt_levels && ctx->opt_spgemm_mode != 1 && ctx->opt_spgemm_mode != 3 &&
      a->nentries > 0 && b->nrows > 0) {
    const double mean = double(a->nnz) / double(a->nentries / 2);
    // automatic mode stages tiles above kWideRangeMean (faster there than
    // levels on the banded and power-of-(A+I) products measured); levels serve
    // the ranges between, and every long range when the row kernel is forced
    if (mean >= kLevelMean && (ctx->opt_spgemm_mode == 2 || mean <= 8.0)) {
      uint32_t nlv = 1;
      while (nlv < 12 && double(1u << (nlv + 1)) <= 2.0 * mean) ++nlv;
      levels = build_levels(ctx, b, nlv);
    }
  }
  // speculative output capacity; an overflow is detected and re-run exactly
  const uint64_t a_ent = a_identity ? 2ull * n : a->nentries;
  uint64_t cap = std::max<uint64_t>({2 * a_ent, 2 * b->nentries, d ? 2 * d->nentries : 0, 4ull * n, 64});
  dvg_matrix* c = new_matrix(ctx, n, b->ncols, cap);
  try {
    DVG_CUDA(cudaMemsetAsync(c->rowmap, 0, sizeof(uint64_t), ctx->stream));
    DeviceControl ctl{};
    for (int attempt = 0; attempt < 2; ++attempt) {
      reset_control(ctx);
      cudaEvent_t t0 = span_begin(ctx);
      launch_spgemm_fused(ctx, a, a_identity, b, d, c->rowmap, c->entries, cap, levels.empty() ? nullptr : &levels);
      span_end(ctx, t0, kProduct);
      ctl = read_control(ctx);
      if (ctl.timeout) throw Error(DVG_ERR_TIMEOUT, "range_spgemm: tile look-back wait expired");
      if (!ctl.overflow) break;
      if (attempt == 1) throw Error(DVG_ERR_DEVICE, "range_spgemm: output capacity overflow after resize");
      ctx->stats.spgemm_reruns++;
      cap = ctl.total;
      dfree(ctx, c->entries);
      c->entries = nullptr;
      c->entries = static_cast<uint32_t*>(dalloc(ctx, entries_alloc_bytes(cap)));
    }
    c->nentries = ctl.total;
    c->nnz = ctl.nnz;
    c->canonical = true;
    ctx->max_product_entries = std::max(ctx->max_product_entries, c->nentries);
    ctx->stats.spgemm_calls++;
    ctx->stats.spgemm_direct_tiles += ctl.tiles_direct;
    ctx->stats.spgemm_slow_rows += ctl.slow_rows;
    uint64_t bytes = (a_identity ? 0 : matrix_bytes(a)) + matrix_bytes(b) + matrix_bytes(c) + (d ? matrix_bytes(d) : 0);
    ctx->stats.alg_bytes += bytes;
    ctx->stats.spgemm_alg_bytes += bytes;
    if (d) ctx->stats.spgemm_fused_adds++;
  } catch (...) {
    free_matrix(ctx, c);
    throw;
  }
  return c;
}

// C = D + A B as one canonical union.  The row kernel merges D's ranges into
// each row's run list; the other kernels take the product and an SpAdd.  Only
// the sum-of-powers schedule calls it, on canonical operands, where both give
// the same canonical matrix.
static dvg_matrix* range_spgemm_add(dvg_context* ctx, const dvg_matrix* d, const dvg_matrix* a, const dvg_matrix* b) {
  require(a->ncols == b->nrows && d->nrows == a->nrows && d->ncols == b->ncols, "range_spgemm_add: shapes");
  if (ctx->opt_spgemm_mode != 1) return range_spgemm_fused(ctx, a, false, b, d);
  dvg_matrix* t = range_spgemm(ctx, a, false, b);
  try {
    dvg_matrix* c = range_spadd(ctx, d, t, false);
    free_matrix(ctx, t);
    return c;
  } catch (...) {
    free_matrix(ctx, t);
    throw;
  }
}

dvg_matrix* range_spgemm(dvg_context* ctx, const dvg_matrix* a, bool a_identity, const dvg_matrix* b) {
  if (!a_identity) require(a->ncols == b->nrows, "range_spgemm: a.numCols() != b.numRows()");
  return range_spgemm_fused(ctx, a, a_identity, b);
}

dvg_matrix* range_spadd(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, bool b_identity) {
  if (!b_identity) {
    require(a->nrows == b->nrows, "range_spadd: row counts differ");
    require(a->ncols == b->ncols, "range_spadd: column counts differ");
  } else {
    require(a->nrows <= a->ncols, "range_spadd: identity does not fit the matrix");
  }
  const uint32_t n = a->nrows;
  // the one-pass kernel stages ranges with 8-byte asynchronous copies
  const bool aligned = ((reinterpret_cast<uintptr_t>(a->entries) |
                         reinterpret_cast<uintptr_t>(b_identity ? nullptr : b->entries)) & 7u) == 0;
  if (ctx->opt_spadd_single && n > 0 && aligned) {
    // one pass: the output never holds more entries than both inputs
    const uint64_t cap = a->nentries + (b_identity ? 2ull * n : b->nentries);
    dvg_matrix* c = new_matrix(ctx, n, a->ncols, cap);
    void* scratch = nullptr;
    try {
      scratch = dalloc(ctx, spadd_single_pass_scratch(n));
      reset_control(ctx);
      cudaEvent_t t0 = span_begin(ctx);
      launch_spadd_single_pass(ctx, a, b, b_identity, c->rowmap, c->entries, cap, scratch);
      span_end(ctx, t0, kSpadd);
      const DeviceControl ctl = read_control(ctx);
      dfree(ctx, scratch);
      scratch = nullptr;
      if (ctl.timeout) throw Error(DVG_ERR_TIMEOUT, "range_spadd: chunk look-back wait expired");
      if (ctl.overflow) throw Error(DVG_ERR_DEVICE, "range_spadd: output capacity overflow");
      c->nentries = ctl.total;
      c->nnz = ctl.nnz;
      c->canonical = a->canonical && (b_identity || b->canonical);
      ctx->stats.spadd_calls++;
      ctx->stats.alg_bytes += matrix_bytes(a) + (b_identity ? 0 : matrix_bytes(b)) + matrix_bytes(c);
    } catch (...) {
      if (scratch) dfree(ctx, scratch);
      free_matrix(ctx, c);
      throw;
    }
    return c;
  }
  dvg_matrix* c = new_matrix(ctx, n, a->ncols, 0);
  try {
    DVG_CUDA(cudaMemsetAsync(c->rowmap, 0, sizeof(uint64_t), ctx->stream));
    reset_control(ctx);
    cudaEvent_t t0 = span_begin(ctx);
    launch_spadd(ctx, a, b, b_identity, c->rowmap, nullptr, false);
    span_end(ctx, t0, kSpadd);
    t0 = span_begin(ctx);
    launch_rowmap_scan(ctx, c->rowmap, n);
    span_end(ctx, t0, kScan);
    uint64_t total = 0;
    DeviceControl ctl = read_total(ctx, c->rowmap + n, &total);
    if (total > 0) {
      dfree(ctx, c->entries);
      c->entries = nullptr;
      c->entries = static_cast<uint32_t*>(dalloc(ctx, entries_alloc_bytes(total)));
      c->nentries = total;
      t0 = span_begin(ctx);
      launch_spadd(ctx, a, b, b_identity, c->rowmap, c->entries, true);
      span_end(ctx, t0, kSpadd);
    }
    c->nnz = ctl.nnz;
    c->canonical = a->canonical && (b_identity || b->canonical);
    ctx->stats.spadd_calls++;
    ctx->stats.alg_bytes += matrix_bytes(a) + (b_identity ? 0 : matrix_bytes(b)) + matrix_bytes(c);
  } catch (...) {
    free_matrix(ctx, c);
    throw;
  }
  return c;
}

dvg_matrix* identity(dvg_context* ctx, uint32_t n) {
  dvg_matrix* m = new_matrix(ctx, n, n, 2ull * n);
  try {
    launch_identity(ctx, m);
  } catch (...) {
    free_matrix(ctx, m);
    throw;
  }
  m->nnz = n;
  return m;
}

// range_power_inplace, range_sparse.hpp:2370-2431: C = I; for each bit of k
// from the lowest, C <- C*A if it is set, then A <- A*A while bits remain.
// The first C*A has C = I and runs with an implicit identity operand.
dvg_matrix* range_power(dvg_context* ctx, const dvg_matrix* a, unsigned k) {
  require(a->nrows == a->ncols, "range_power: matrix is not square");
  if (k == 0) return identity(ctx, a->ncols);
  dvg_matrix* c = nullptr;
  const dvg_matrix* p = a;  // current power of a (a itself is not owned)
  try {
    while (true) {
      if (k & 1) {
        dvg_matrix* nc = c ? range_spgemm(ctx, c, false, p) : range_spgemm(ctx, nullptr, true, p);
        free_matrix(ctx, c);
        c = nc;
      }
      k >>= 1;
      if (k == 0) break;
      dvg_matrix* np = range_spgemm(ctx, p, false, p);
      if (p != a) free_matrix(ctx, const_cast<dvg_matrix*>(p));
      p = np;
    }
  } catch (...) {
    free_matrix(ctx, c);
    if (p != a) free_matrix(ctx, const_cast<dvg_matrix*>(p));
    throw;
  }
  if (p != a) free_matrix(ctx, const_cast<dvg_matrix*>(p));
  return c;
}

// util::create_distance_index, dindex.hpp:46-189, as the reference
// schedules it: rai = I + A; rad = A^dlo and raid = rai^(dup-dlo) by
// square-and-multiply; d = rad * raid.
static dvg_matrix* distance_index_reference(dvg_context* ctx, const dvg_matrix* a, unsigned dlo, unsigned dup) {
  dvg_matrix* rai = range_spadd(ctx, a, nullptr, true);  // I + A (fused identity)
  dvg_matrix* rad = nullptr;
  dvg_matrix* raid = nullptr;
  dvg_matrix* d = nullptr;
  try {
    if (dlo != 0) rad = range_power(ctx, a, dlo);
    raid = range_power(ctx, rai, dup - dlo);
    free_matrix(ctx, rai);
    rai = nullptr;
    if (dlo != 0) {
      d = range_spgemm(ctx, rad, false, raid);
      free_matrix(ctx, rad);
      free_matrix(ctx, raid);
    } else {
      d = raid;
    }
  } catch (...) {
    free_matrix(ctx, rai);
    free_matrix(ctx, rad);
    free_matrix(ctx, raid);
    throw;
  }
  return d;
}

// The same index, T = A^dlo * (A+I)^K with K = dup - dlo, scheduled so that
// every product has a power of A -- whose rows hold a few narrow ranges -- as
// its left operand.  Over the Boolean semiring (A+I)^n = sum_{j<=n} A^j, so
//   (A+I)^(a+b) = (A+I)^a + A^a (A+I)^b     for every Boolean matrix A.
// With P_m = A^(2^m) (square A) and Q_m = (A+I)^(2^m):
//   Q_0 = A + I,  Q_(m+1) = Q_m + P_m Q_m,
// (A+I)^K is assembled over the set bits of K with the same identity, and
// A^dlo by square-and-multiply over the P_m.  T is the same canonical matrix
// as the reference's A^dlo * (A+I)^K (both equal sum_{dlo<=j<=dup} A^j), so
// the output is identical, while the wide-row squarings of (A+I)^k -- whose
// rows name ~k B rows each -- are gone.
static dvg_matrix* distance_index_powersum(dvg_context* ctx, const dvg_matrix* a, unsigned dlo, unsigned dup) {
  const unsigned K = dup - dlo;
  std::vector<dvg_matrix*> P;  // P[m] = A^(2^m); P[0] is `a` (not owned)
  std::vector<dvg_matrix*> owned;
  auto own = [&](dvg_matrix* m) {
    owned.push_back(m);
    return m;
  };
  auto release = [&](dvg_matrix* m) {
    for (auto& o : owned)
      if (o == m) {
        free_matrix(ctx, o);
        o = nullptr;
      }
  };
  int top_k = -1, top_lo = -1;
  for (int b = 31; b >= 0; --b) {
    if (top_k < 0 && (K >> b) & 1u) top_k = b;
    if (top_lo < 0 && (dlo >> b) & 1u) top_lo = b;
  }
  const int need_p = std::max(top_k, top_lo);  // highest P_m used
  try {
    P.push_back(const_cast<dvg_matrix*>(a));
    for (int m = 1; m <= need_p; ++m) P.push_back(own(range_spgemm(ctx, P[m - 1], false, P[m - 1])));

    // (A+I)^K
    dvg_matrix* R = nullptr;   // (A+I)^e, e = sum of the bits of K handled so far
    dvg_matrix* Ae = nullptr;  // A^e (nullptr: e has one bit, A^e = P[that bit])
    unsigned e = 0;
    if (K == 0) {
      R = own(identity(ctx, a->ncols));
    } else {
      dvg_matrix* Q = own(range_spadd(ctx, a, nullptr, true));  // Q_0 = A + I
      for (int m = 0; m <= top_k; ++m) {
        if ((K >> m) & 1u) {
          if (!R) {
            R = Q;
            e = 1u << m;
          } else {
            // (A+I)^(e + 2^m) = (A+I)^e + A^e Q_m
            const dvg_matrix* Aexp = Ae ? Ae : P[__builtin_ctz(e)];
            dvg_matrix* nr = own(range_spgemm_add(ctx, R, Aexp, Q));
            if (R != Q) release(R);
            R = nr;
            // A^(e + 2^m) = A^e P_m, needed only for a later bit
            if ((K >> (m + 1)) != 0) {
              dvg_matrix* na = own(range_spgemm(ctx, Aexp, false, P[m]));
              if (Ae) release(Ae);
              Ae = na;
            }
            e += 1u << m;
          }
        }
        if (m < top_k) {
          // Q_(m+1) = Q_m + P_m Q_m
          dvg_matrix* nq = own(range_spgemm_add(ctx, Q, P[m], Q));
          if (Q != R) release(Q);
          Q = nq;
        }
      }
      if (Q != R) release(Q);
      if (Ae) release(Ae);
    }

    // A^dlo by square-and-multiply over the P_m, then T = A^dlo (A+I)^K
    dvg_matrix* T = nullptr;
    if (dlo == 0) {
      T = R;
    } else {
      dvg_matrix* Ad = nullptr;  // nullptr: a single P_m so far
      int first = -1;
      for (int m = 0; m <= top_lo; ++m) {
        if (!((dlo >> m) & 1u)) continue;
        if (first < 0) {
          first = m;
        } else {
          dvg_matrix* n2 = own(range_spgemm(ctx, Ad ? Ad : P[first], false, P[m]));
          if (Ad) release(Ad);
          Ad = n2;
        }
      }
      T = range_spgemm(ctx, Ad ? Ad : P[first], false, R);
      if (Ad) release(Ad);
      release(R);
    }
    for (auto& o : owned)
      if (o && o != T) free_matrix(ctx, o);
    owned.clear();
    return T;
  } catch (...) {
    for (auto& o : owned)
      if (o) free_matrix(ctx, o);
    throw;
  }
}

dvg_matrix* create_distance_index(dvg_context* ctx, const dvg_matrix* a, unsigned dlo, unsigned dup) {
  require(dlo <= dup && dup != 0, "create_distance_index: requires dmin <= dmax and dmax != 0");
  require(a->nrows == a->ncols, "create_distance_index: adjacency matrix is not square");
  // the sum-of-powers schedule ends on SpAdds when dlo == 0; those keep rows
  // canonical only for canonical inputs, while the reference's squarings
  // canonicalise any input
  if (ctx->opt_dindex_schedule == 1 || (dlo == 0 && !a->canonical)) return distance_index_reference(ctx, a, dlo, dup);
  if (ctx->opt_planned && ctx->opt_spgemm_mode != 1 && a->nrows > 0) {
    PlannedBuild pb;
    bool planned = true;
    try {
      pb = prepare_build(ctx, plan_index(dlo, dup), a);
    } catch (const Error& e) {
      if (e.status != DVG_ERR_OOM) throw;
      planned = false;  // the estimates do not fit: exact sizes on the read-back path
    }
    if (!planned) return distance_index_powersum(ctx, a, dlo, dup);
    try {
      launch_build(ctx, pb, ctx->opt_timing);
    } catch (...) {
      release_build(ctx, pb);
      throw;
    }
    if (dvg_matrix* t = finish_build(ctx, pb)) return t;
    // a step outgrew its estimate: build on the read-back path and size the
    // next planned builds from its largest product
    ctx->stats.spgemm_reruns++;
    ctx->max_product_entries = 0;
    dvg_matrix* t = distance_index_powersum(ctx, a, dlo, dup);
    const double grow = double(ctx->max_product_entries) / double(std::max<uint64_t>(a->nentries, 1));
    ctx->plan_growth = std::max(ctx->plan_growth, 1.25 * grow + 0.25);
    return t;
  }
  return distance_index_powersum(ctx, a, dlo, dup);
}

}  // namespace dvg

using namespace dvg;

extern "C" {

const char* dvg_last_error(void) { return g_last_error.c_str(); }

const char* dvg_status_string(dvg_status s) {
  switch (s) {
    case DVG_OK: return "ok";
    case DVG_ERR_INVALID_ARG: return "invalid argument";
    case DVG_ERR_OOM: return "out of memory";
    case DVG_ERR_DEVICE: return "device error";
    case DVG_ERR_TIMEOUT: return "device wait timed out";
    case DVG_ERR_NOT_INITIALIZED: return "not initialized";
    case DVG_ERR_OVERFLOW: return "overflow";
  }
  return "unknown";
}

dvg_status dvg_init(int device, dvg_context** out) {
  if (!out) return fail(DVG_ERR_INVALID_ARG, "null output pointer");
  *out = nullptr;
  dvg_context* ctx = new dvg_context();
  dvg_status s = guarded([&] {
    int count = 0;
    DVG_CUDA(cudaGetDeviceCount(&count));
    require(device >= 0 && device < count, "no such CUDA device");
    cudaDeviceProp prop{};
    DVG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
      throw Error(DVG_ERR_DEVICE, std::string("libdvg is built for sm_100a (B200); device is ") + prop.name);
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    DVG_CUDA(cudaSetDevice(device));
    DVG_CUDA(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
    ctx->stream = ctx->own_stream;
    cudaMemPool_t pool;
    DVG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = ~0ull;
    DVG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    DVG_CUDA(cudaMalloc(&ctx->d_ctl, sizeof(DeviceControl)));
    DVG_CUDA(cudaMemset(ctx->d_ctl, 0, sizeof(DeviceControl)));
    // control block mirror plus one word for size read-backs
    DVG_CUDA(cudaMallocHost(&ctx->h_ctl, 2 * sizeof(DeviceControl)));
  });
  if (s != DVG_OK) {
    if (ctx->d_ctl) cudaFree(ctx->d_ctl);
    if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return s;
  }
  *out = ctx;
  return DVG_OK;
}

dvg_status dvg_shutdown(dvg_context* ctx) {
  if (!ctx) return fail(DVG_ERR_INVALID_ARG, "null context");
  dvg_status s = guarded([&] {
    Lock lk(ctx);
    if (ctx->d_tile_sums) dfree(ctx, ctx->d_tile_sums);
    if (ctx->d_pairs) dfree(ctx, ctx->d_pairs);
    if (ctx->d_answers) dfree(ctx, ctx->d_answers);
    if (ctx->d_tile_desc) dfree(ctx, ctx->d_tile_desc);
    if (ctx->d_row_stage) dfree(ctx, ctx->d_row_stage);
    if (ctx->d_ticket) dfree(ctx, ctx->d_ticket);
    release_cached(ctx);
    DVG_CUDA(cudaStreamSynchronize(ctx->stream));
    resolve_spans(ctx);
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    ctx->event_pool.clear();
    DVG_CUDA(cudaFree(ctx->d_ctl));
    DVG_CUDA(cudaFreeHost(ctx->h_ctl));
    if (ctx->h_stage) DVG_CUDA(cudaFreeHost(ctx->h_stage));
    for (void* h : ctx->h_retired) DVG_CUDA(cudaFreeHost(h));
    ctx->h_retired.clear();
    if (ctx->own_stream) DVG_CUDA(cudaStreamDestroy(ctx->own_stream));
  });
  delete ctx;
  return s;
}

dvg_status dvg_set_stream(dvg_context* ctx, void* stream) {
  return guarded([&] {
    Lock lk(ctx);
    DVG_CUDA(cudaStreamSynchronize(ctx->stream));
    resolve_spans(ctx);
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  });
}

dvg_status dvg_synchronize(dvg_context* ctx) {
  return guarded([&] {
    Lock lk(ctx);
    read_control(ctx);
  });
}

dvg_status dvg_set_option(dvg_context* ctx, const char* key, int64_t value) {
  return guarded([&] {
    Lock lk(ctx);
    require(key != nullptr, "null option key");
    if (!std::strcmp(key, "algo")) {
      // the single-pass kernels are the only SpGEMM; 0 is accepted for callers that set it
      require(value == 0, "algo must be 0 (single-pass SpGEMM)");
    } else if (!std::strcmp(key, "dindex_schedule")) {
      require(value == 0 || value == 1, "dindex_schedule must be 0 (sum of powers) or 1 (reference squaring)");
      ctx->opt_dindex_schedule = value;
    } else if (!std::strcmp(key, "spgemm_mode")) {
      require(value >= 0 && value <= 3, "spgemm_mode must be 0 (automatic), 1 (tiled), 2 (light) or 3 (wide)");
      ctx->opt_spgemm_mode = value;
    } else if (!std::strcmp(key, "planned_build")) {
      require(value == 0 || value == 1, "planned_build must be 0 or 1");
      ctx->opt_planned = value;
    } else if (!std::strcmp(key, "plan_growth")) {
      require(value >= 0 && value <= 100000, "plan_growth is a percentage in [0, 100000]");
      ctx->plan_growth = double(value) / 100.0;
    } else if (!std::strcmp(key, "autotune")) {
      require(value == 0 || value == 1, "autotune must be 0 or 1");
      ctx->opt_autotune = value;
    } else if (!std::strcmp(key, "spgemm_levels")) {
      require(value == 0 || value == 1, "spgemm_levels must be 0 or 1");
      ctx->opt_levels = value;
    } else if (!std::strcmp(key, "row_stage")) {
      require(value == 0 || value == 1, "row_stage must be 0 or 1");
      ctx->opt_row_stage = value;
    } else if (!std::strcmp(key, "spadd_single")) {
      require(value == 0 || value == 1, "spadd_single must be 0 or 1");
      ctx->opt_spadd_single = value;
    } else if (!std::strcmp(key, "row_slot")) {
      require(value >= 0 && value <= 2, "row_slot must be 0 (16 entries), 1 (24) or 2 (32)");
      ctx->opt_row_slot = value;
    } else if (!std::strcmp(key, "chunk_rows")) {
      require(value >= 0 && value <= 2048 && value % 32 == 0, "chunk_rows must be 0 or a multiple of 32 up to 2048");
      ctx->opt_chunk_rows = value;
    } else if (!std::strcmp(key, "timing")) {
      DVG_CUDA(cudaStreamSynchronize(ctx->stream));
      resolve_spans(ctx);
      ctx->opt_timing = value != 0;
    } else {
      require(false, "unknown option");
    }
  });
}

dvg_status dvg_trim(dvg_context* ctx) {
  return guarded([&] {
    Lock lk(ctx);
    release_cached(ctx);
    DVG_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

dvg_status dvg_get_stats(const dvg_context* ctx, dvg_stats* out) {
  if (!ctx || !out) return fail(DVG_ERR_INVALID_ARG, "null argument");
  *out = ctx->stats;
  return DVG_OK;
}

dvg_status dvg_stats_reset(dvg_context* ctx) {
  if (!ctx) return fail(DVG_ERR_INVALID_ARG, "null context");
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  ctx->stats = dvg_stats{};
  return DVG_OK;
}

}  // extern "C"

namespace dvg {
std::string validation_message(unsigned long long bits) {
  std::string why;
  if (bits & 1) why += " rowmap[0] != 0;";
  if (bits & 2) why += " rowmap decreasing or odd row length;";
  if (bits & 4) why += " rowmap[nrows] != number of entries;";
  if (bits & 8) why += " column index >= ncols;";
  return why;
}
}  // namespace dvg

extern "C" {

static void validate_uploaded(dvg_context* ctx, dvg_matrix* m) {
  reset_control(ctx);
  launch_validate(ctx, m->rowmap, m->nrows, m->entries, m->nentries, m->ncols);
  DeviceControl c = read_control(ctx);
  m->canonical = !(c.invalid & 16);
  c.invalid &= ~16ull;
  if (c.invalid) throw Error(DVG_ERR_INVALID_ARG, "malformed range-CRS matrix:" + validation_message(c.invalid));
}

static uint64_t count_nnz_host(const uint32_t* e, uint64_t n) {
  uint64_t c = 0;
  for (uint64_t i = 0; i + 1 < n; i += 2) c += uint64_t(e[i + 1]) - e[i] + 1;
  return c;
}

}  // extern "C"

namespace dvg {
dvg_matrix* upload_matrix(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint64_t* rowmap,
                          const uint32_t* entries, uint64_t nnz) {
  require(rowmap != nullptr, "null argument");
  require(ncols <= 0xFFFFFFFEu, "ncols must be below 2^32 - 1");
  const uint64_t ne = rowmap[nrows];
  require(ne == 0 || entries, "null entries");
  dvg_matrix* m = new_matrix(ctx, nrows, ncols, ne);
  try {
    DVG_CUDA(cudaMemcpyAsync(m->rowmap, rowmap, (size_t(nrows) + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (ne) DVG_CUDA(cudaMemcpyAsync(m->entries, entries, ne * 4, cudaMemcpyHostToDevice, ctx->stream));
    ctx->stats.h2d_bytes += (uint64_t(nrows) + 1) * 8 + ne * 4;
    validate_uploaded(ctx, m);
    m->nnz = nnz ? nnz : count_nnz_host(entries, ne);
  } catch (...) {
    free_matrix(ctx, m);
    throw;
  }
  return m;
}
}  // namespace dvg

extern "C" {

dvg_status dvg_matrix_upload(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint64_t* rowmap,
                             const uint32_t* entries, uint64_t nnz, dvg_matrix** out) {
  return guarded([&] {
    Lock lk(ctx);
    require(out != nullptr, "null argument");
    *out = upload_matrix(ctx, nrows, ncols, rowmap, entries, nnz);
  });
}

dvg_status dvg_matrix_upload_u32(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint32_t* rowmap,
                                 const uint32_t* entries, uint64_t nnz, dvg_matrix** out) {
  return guarded([&] {
    Lock lk(ctx);
    require(out && rowmap, "null argument");
    require(ncols <= 0xFFFFFFFEu, "ncols must be below 2^32 - 1");
    const uint64_t ne = rowmap[nrows];
    require(ne == 0 || entries, "null entries");
    dvg_matrix* m = new_matrix(ctx, nrows, ncols, ne);
    uint32_t* tmp = nullptr;
    try {
      tmp = static_cast<uint32_t*>(dalloc(ctx, (size_t(nrows) + 1) * 4));
      DVG_CUDA(cudaMemcpyAsync(tmp, rowmap, (size_t(nrows) + 1) * 4, cudaMemcpyHostToDevice, ctx->stream));
      launch_widen_rowmap(ctx, tmp, m->rowmap, uint64_t(nrows) + 1);
      dfree(ctx, tmp);
      tmp = nullptr;
      if (ne) DVG_CUDA(cudaMemcpyAsync(m->entries, entries, ne * 4, cudaMemcpyHostToDevice, ctx->stream));
      ctx->stats.h2d_bytes += (uint64_t(nrows) + 1) * 4 + ne * 4;
      validate_uploaded(ctx, m);
      m->nnz = nnz ? nnz : count_nnz_host(entries, ne);
    } catch (...) {
      if (tmp) dfree(ctx, tmp);
      free_matrix(ctx, m);
      throw;
    }
    *out = m;
  });
}

dvg_status dvg_matrix_wrap_device(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint64_t* d_rowmap,
                                  const uint32_t* d_entries, uint64_t nentries, uint64_t nnz, dvg_matrix** out) {
  return guarded([&] {
    Lock lk(ctx);
    require(out && d_rowmap && (nentries == 0 || d_entries), "null argument");
    require(ncols <= 0xFFFFFFFEu, "ncols must be below 2^32 - 1");
    require((reinterpret_cast<uintptr_t>(d_entries) & 7) == 0, "entries must be 8-byte aligned");
    auto* m = new dvg_matrix();
    m->nrows = nrows;
    m->ncols = ncols;
    m->nentries = nentries;
    m->rowmap = const_cast<uint64_t*>(d_rowmap);
    m->entries = const_cast<uint32_t*>(d_entries);
    m->owned = false;
    m->device = ctx->device;
    try {
      validate_uploaded(ctx, m);
    } catch (...) {
      delete m;
      throw;
    }
    m->nnz = nnz;
    *out = m;
  });
}

dvg_status dvg_matrix_info(const dvg_matrix* m, uint32_t* nrows, uint32_t* ncols, uint64_t* nentries, uint64_t* nnz) {
  if (!m) return fail(DVG_ERR_INVALID_ARG, "null matrix");
  if (nrows) *nrows = m->nrows;
  if (ncols) *ncols = m->ncols;
  if (nentries) *nentries = m->nentries;
  if (nnz) *nnz = m->nnz;
  return DVG_OK;
}

dvg_status dvg_matrix_device_arrays(const dvg_matrix* m, const uint64_t** d_rowmap, const uint32_t** d_entries) {
  if (!m) return fail(DVG_ERR_INVALID_ARG, "null matrix");
  if (d_rowmap) *d_rowmap = m->rowmap;
  if (d_entries) *d_entries = m->entries;
  return DVG_OK;
}

dvg_status dvg_matrix_download(dvg_context* ctx, const dvg_matrix* m, uint64_t* rowmap, uint32_t* entries) {
  return guarded([&] {
    Lock lk(ctx);
    require(m && rowmap && (m->nentries == 0 || entries), "null argument");
    DVG_CUDA(cudaMemcpyAsync(rowmap, m->rowmap, (size_t(m->nrows) + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (m->nentries)
      DVG_CUDA(cudaMemcpyAsync(entries, m->entries, m->nentries * 4, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->stats.d2h_bytes += (uint64_t(m->nrows) + 1) * 8 + m->nentries * 4;
    read_control(ctx);
  });
}

dvg_status dvg_matrix_download_u32(dvg_context* ctx, const dvg_matrix* m, uint32_t* rowmap, uint32_t* entries) {
  return guarded([&] {
    Lock lk(ctx);
    require(m && rowmap && (m->nentries == 0 || entries), "null argument");
    if (m->nentries > 0xFFFFFFFFull) throw Error(DVG_ERR_OVERFLOW, "entries do not fit a 32-bit rowmap");
    uint32_t* tmp = static_cast<uint32_t*>(dalloc(ctx, (size_t(m->nrows) + 1) * 4));
    try {
      launch_narrow_rowmap(ctx, m->rowmap, tmp, uint64_t(m->nrows) + 1);
      DVG_CUDA(cudaMemcpyAsync(rowmap, tmp, (size_t(m->nrows) + 1) * 4, cudaMemcpyDeviceToHost, ctx->stream));
      if (m->nentries)
        DVG_CUDA(cudaMemcpyAsync(entries, m->entries, m->nentries * 4, cudaMemcpyDeviceToHost, ctx->stream));
      ctx->stats.d2h_bytes += (uint64_t(m->nrows) + 1) * 4 + m->nentries * 4;
      read_control(ctx);
    } catch (...) {
      dfree(ctx, tmp);
      throw;
    }
    dfree(ctx, tmp);
  });
}

dvg_status dvg_matrix_free(dvg_context* ctx, dvg_matrix* m) {
  if (!m) return DVG_OK;
  return guarded([&] {
    Lock lk(ctx);
    free_matrix(ctx, m);
  });
}

dvg_status dvg_range_identity(dvg_context* ctx, uint32_t n, dvg_matrix** out) {
  return guarded([&] {
    Lock lk(ctx);
    require(out != nullptr, "null output");
    *out = identity(ctx, n);
  });
}

dvg_status dvg_range_spadd(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, dvg_matrix** c) {
  return guarded([&] {
    Lock lk(ctx);
    require(a && b && c, "null argument");
    *c = range_spadd(ctx, a, b, false);
  });
}

dvg_status dvg_range_spgemm(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, dvg_matrix** c) {
  return guarded([&] {
    Lock lk(ctx);
    require(a && b && c, "null argument");
    dvg_matrix* r = range_spgemm(ctx, a, false, b);
    try {
      read_control(ctx);
    } catch (...) {
      free_matrix(ctx, r);
      throw;
    }
    *c = r;
  });
}

dvg_status dvg_range_power(dvg_context* ctx, const dvg_matrix* a, unsigned k, dvg_matrix** c) {
  return guarded([&] {
    Lock lk(ctx);
    require(a && c, "null argument");
    dvg_matrix* r = range_power(ctx, a, k);
    try {
      read_control(ctx);
    } catch (...) {
      free_matrix(ctx, r);
      throw;
    }
    *c = r;
  });
}

dvg_status dvg_selftest_bounded_wait(dvg_context* ctx, uint32_t spin_limit) {
  return guarded([&] {
    Lock lk(ctx);
    reset_control(ctx);
    selftest_bounded_wait(ctx, spin_limit);
    const DeviceControl c = read_control(ctx);
    if (c.timeout) throw Error(DVG_ERR_TIMEOUT, "self-test: the look-back wait ran out, as it must");
    throw Error(DVG_ERR_DEVICE, "self-test: a wait on a chunk nothing publishes returned without a timeout");
  });
}

dvg_status dvg_calibrate_range_ops(dvg_context* ctx, double* ops_per_second) {
  return guarded([&] {
    require(ctx != nullptr && ops_per_second != nullptr, "null argument");
    Lock lk(ctx);
    *ops_per_second = calibrate_range_ops(ctx);
  });
}

dvg_status dvg_calibrate_random_reads(dvg_context* ctx, uint64_t bytes, double* reads_per_second) {
  return guarded([&] {
    require(ctx != nullptr && reads_per_second != nullptr, "null argument");
    require(bytes <= (uint64_t(1) << 40), "calibrate_random_reads: bytes above 2^40");
    Lock lk(ctx);
    *reads_per_second = calibrate_random_reads(ctx, bytes);
  });
}

dvg_status dvg_adjacency_from_graph(dvg_context* ctx, uint32_t nnodes, const uint32_t* node_len, uint64_t nedges,
                                    const uint32_t* edges, uint32_t lower, uint32_t upper, dvg_matrix** out) {
  return guarded([&] {
    Lock lk(ctx);
    require(out != nullptr, "null argument");
    require(nedges == 0 || edges != nullptr, "null edges");
    for (uint64_t e = 0; e < 2 * nedges; ++e)
      require(edges[e] >= 1 && edges[e] <= nnodes, "edge endpoint is not a node id in 1..nnodes");
    *out = adjacency_from_graph(ctx, nnodes, node_len, nedges, edges, lower, upper);
  });
}

dvg_status dvg_create_distance_index(dvg_context* ctx, const dvg_matrix* ra, unsigned dmin, unsigned dmax,
                                     dvg_matrix** out) {
  return guarded([&] {
    Lock lk(ctx);
    require(ra && out, "null argument");
    dvg_matrix* r = create_distance_index(ctx, ra, dmin, dmax);
    try {
      read_control(ctx);
    } catch (...) {
      free_matrix(ctx, r);
      throw;
    }
    *out = r;
  });
}

dvg_status dvg_batch_distance_index(dvg_context* ctx, uint32_t ngraphs, const dvg_matrix* const* graphs,
                                    const unsigned* dmin, const unsigned* dmax, dvg_matrix** out) {
  return guarded([&] {
    Lock lk(ctx);
    require(ngraphs == 0 || (graphs && dmin && dmax && out), "null argument");
    batch_distance_index(ctx, ngraphs, graphs, dmin, dmax, out);
    try {
      read_control(ctx);
    } catch (...) {
      for (uint32_t k = 0; k < ngraphs; ++k) {
        free_matrix(ctx, out[k]);
        out[k] = nullptr;
      }
      throw;
    }
  });
}

dvg_status dvg_query_batch(dvg_context* ctx, const dvg_matrix* index, const uint32_t* d_pairs, uint64_t npairs,
                           uint8_t* d_out) {
  return guarded([&] {
    Lock lk(ctx);
    require(index && (npairs == 0 || (d_pairs && d_out)), "null argument");
    require((reinterpret_cast<uintptr_t>(d_pairs) & 7) == 0, "pairs must be 8-byte aligned");
    reset_control(ctx);
    cudaEvent_t t0 = span_begin(ctx);
    launch_query(ctx, index, d_pairs, npairs, d_out);
    span_end(ctx, t0, kQuery);
    ctx->stats.query_pairs += npairs;
    DeviceControl c = read_control(ctx);
    if (c.invalid) throw Error(DVG_ERR_INVALID_ARG, std::to_string(c.invalid) + " query pairs out of range");
  });
}

dvg_status dvg_query_batch_host(dvg_context* ctx, const dvg_matrix* index, const uint32_t* pairs, uint64_t npairs,
                                uint8_t* out) {
  return guarded([&] {
    Lock lk(ctx);
    require(index && (npairs == 0 || (pairs && out)), "null argument");
    if (npairs == 0) return;
    if (npairs > ctx->pairs_cap) {
      if (ctx->d_pairs) dfree(ctx, ctx->d_pairs);
      if (ctx->d_answers) dfree(ctx, ctx->d_answers);
      ctx->d_pairs = nullptr;
      ctx->d_answers = nullptr;
      ctx->pairs_cap = 0;
      ctx->d_pairs = static_cast<uint32_t*>(dalloc(ctx, npairs * 8));
      ctx->d_answers = static_cast<uint8_t*>(dalloc(ctx, npairs));
      ctx->pairs_cap = npairs;
    }
    DVG_CUDA(cudaMemcpyAsync(ctx->d_pairs, pairs, npairs * 8, cudaMemcpyHostToDevice, ctx->stream));
    reset_control(ctx);
    cudaEvent_t t0 = span_begin(ctx);
    launch_query(ctx, index, ctx->d_pairs, npairs, ctx->d_answers);
    span_end(ctx, t0, kQuery);
    ctx->stats.query_pairs += npairs;
    DVG_CUDA(cudaMemcpyAsync(out, ctx->d_answers, npairs, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->stats.h2d_bytes += npairs * 8;
    ctx->stats.d2h_bytes += npairs;
    DeviceControl c = read_control(ctx);
    if (c.invalid) throw Error(DVG_ERR_INVALID_ARG, std::to_string(c.invalid) + " query pairs out of range");
  });
}

}  // extern "C"
