// dvg_engine.cu -- planned index builds: the distance-index schedule as a fixed
// sequence of thread-per-row products whose buffers are all allocated up front.
//
// The schedule is the sum-of-powers form of the reference's
// create_distance_index (dindex.hpp:46-189 in cartoonist/diverg): over the
// Boolean semiring (A+I)^(a+b) = (A+I)^a + A^a (A+I)^b, so with P_m = A^(2^m),
// Q_0 = A + I and Q_(m+1) = Q_m + P_m Q_m the index
// T = A^dlo (A+I)^(dup-dlo) is assembled from products whose left factor is a
// power of A.  For [400, 600]: P_1..P_8, Q_0..Q_7, two steps for the bits of
// 200 above the lowest, two products for A^400 and the final one: 21 steps.
// Every step is one launch of the row kernel computing
// C = A B, C = D + A B or C = I + I A (= A + I), all canonical unions, so the
// result equals the reference's index for canonical inputs (and for any input
// when dlo > 0, where the last step is a product).
//
// Sizes of the intermediates are not known before they are computed, so each
// step gets an estimated entry capacity (a multiple of the input's entries,
// learned per context).  A step that overflows sets a device word; every later
// step reads it before taking work and returns, and the host re-runs the build
// on the synchronised path and raises its estimate.  No host round trip
// happens between the steps: a build is one memset plus one kernel per step,
// and the same sequence can be captured into a CUDA graph.
#include <algorithm>
#include <cstring>

#include "dvg_internal.h"

namespace dvg {

// Pinned host staging for read-backs.  It grows by doubling, and a buffer it
// outgrows is kept until the context shuts down: cudaFreeHost waits for the
// whole device, which would stall every other stream (a server's queries).
void* host_stage(dvg_context* ctx, size_t bytes) {
  if (bytes > ctx->h_stage_cap) {
    const size_t want = std::max<size_t>({bytes, 2 * ctx->h_stage_cap, size_t(64) << 10});
    void* p = nullptr;
    DVG_CUDA(cudaMallocHost(&p, want));
    if (ctx->h_stage) ctx->h_retired.push_back(ctx->h_stage);
    ctx->h_stage = p;
    ctx->h_stage_cap = want;
  }
  return ctx->h_stage;
}

IndexPlan plan_index(unsigned dlo, unsigned dup) {
  IndexPlan pl;
  auto step = [&](int a, bool a_id, int b, int d, bool d_id) {
    const int c = pl.nslots++;
    pl.steps.push_back(PlanStep{c, a, b, d, a_id, d_id});
    return c;
  };
  const unsigned K = dup - dlo;
  int top_k = -1, top_lo = -1;
  for (int b = 31; b >= 0; --b) {
    if (top_k < 0 && ((K >> b) & 1u)) top_k = b;
    if (top_lo < 0 && ((dlo >> b) & 1u)) top_lo = b;
  }
  const int need_p = std::max(top_k, top_lo);
  std::vector<int> P{0};  // P[m] = A^(2^m)
  for (int m = 1; m <= need_p; ++m) P.push_back(step(P[m - 1], false, P[m - 1], -1, false));
  int R = -1;  // (A+I)^e for the bits e of K handled so far (-1 with K = 0: the identity)
  if (K > 0) {
    // the bits of K from the lowest: with e the bits taken so far,
    // (A+I)^(2^m + e) = Q_m + P_m (A+I)^e, so every left factor is a power
    // P_m, whose rows are a column or two
    int Q = step(-1, true, 0, -1, true);  // Q_0 = I + I A
    for (int m = 0; m <= top_k; ++m) {
      if ((K >> m) & 1u) R = R < 0 ? Q : step(P[m], false, R, Q, false);
      if (m < top_k) Q = step(P[m], false, Q, Q, false);  // Q_(m+1) = Q_m + P_m Q_m
    }
  }
  if (dlo == 0) {
    pl.out = R;  // dup > 0, so K > 0
  } else {
    int Ad = -1, first = -1;
    for (int m = 0; m <= top_lo; ++m) {
      if (!((dlo >> m) & 1u)) continue;
      if (first < 0) first = m;
      else Ad = step(Ad >= 0 ? Ad : P[first], false, P[m], -1, false);
    }
    const int L = Ad >= 0 ? Ad : P[first];
    if (K > 0) pl.out = step(L, false, R, -1, false);
    else pl.out = L == 0 ? step(-1, true, 0, -1, false) : L;  // A^1 I: a canonical copy of A
  }
  return pl;
}

PlannedBuild prepare_build(dvg_context* ctx, const IndexPlan& plan, const dvg_matrix* a) {
  return prepare_build(ctx, plan, a, int(ctx->opt_row_slot), ctx->opt_chunk_rows);
}

PlannedBuild prepare_build(dvg_context* ctx, const IndexPlan& plan, const dvg_matrix* a, int slot_variant,
                           int64_t chunk_rows) {
  const uint64_t t_prep = now_ns();
  struct PrepTimer {
    dvg_context* ctx;
    uint64_t t0;
    ~PrepTimer() { ctx->stats.host_prepare_ns += now_ns() - t0; }
  } prep_timer{ctx, t_prep};
  PlannedBuild pb;
  pb.plan = plan;
  pb.input = a;
  pb.n = a->nrows;
  const int ns = plan.nslots;
  pb.rowmap.assign(ns, nullptr);
  pb.entries.assign(ns, nullptr);
  pb.cap.assign(ns, 0);
  pb.owner_step.assign(ns, -1);
  pb.live.assign(ns, 0);
  pb.rowmap[0] = a->rowmap;
  pb.entries[0] = a->entries;
  pb.cap[0] = a->nentries;
  pb.slot_variant = slot_variant;
  pb.shape = row_launch_shape(ctx, pb.n, chunk_rows, pb.slot_variant);
  const size_t nsteps = plan.steps.size();
  pb.desc_stride = (pb.shape.desc_bytes + 255) & ~size_t(255);
  const size_t tickets_off = pb.desc_stride * nsteps;
  const size_t ctl_off = (tickets_off + nsteps * sizeof(unsigned) + 255) & ~size_t(255);
  const size_t abort_off = ctl_off + nsteps * sizeof(DeviceControl);
  pb.scratch_bytes = abort_off + 256;
  std::vector<int> last_use(ns, -1);
  for (size_t i = 0; i < nsteps; ++i)
    for (int s : {plan.steps[i].a, plan.steps[i].b, plan.steps[i].d})
      if (s >= 0) last_use[s] = int(i);
  // most slots alive at once (outputs are allocated before their inputs retire)
  int live = 0, max_live = 1;
  for (size_t i = 0; i < nsteps; ++i) {
    max_live = std::max(max_live, ++live);
    for (int s : {plan.steps[i].a, plan.steps[i].b, plan.steps[i].d})
      if (s > 0 && last_use[s] == int(i) && s != plan.out) --live;
  }
  uint64_t est = std::max<uint64_t>(uint64_t(ctx->plan_growth * double(a->nentries)), 4ull * pb.n) + 64;
  // keep the plan within 80 % of the memory the device (and this context's
  // cache) can give; a step that then overflows re-runs on the read-back path
  const size_t free_b = device_free_bytes(ctx);
  const double avail = 0.8 * double(free_b + ctx->cached_bytes) / double(max_live) - 8.0 * (double(pb.n) + 1);
  if (avail < 4.0 * double(est)) est = std::max<uint64_t>(uint64_t(std::max(avail, 0.0) / 4.0), 4ull * pb.n + 64);
  try {
    pb.scratch = dalloc(ctx, pb.scratch_bytes);
    char* base = static_cast<char*>(pb.scratch);
    pb.tickets = reinterpret_cast<unsigned*>(base + tickets_off);
    pb.ctls = reinterpret_cast<DeviceControl*>(base + ctl_off);
    pb.abort = reinterpret_cast<unsigned long long*>(base + abort_off);
    if (ctx->opt_row_stage) pb.stage = static_cast<uint32_t*>(dalloc(ctx, pb.shape.stage_bytes));
    for (size_t i = 0; i < nsteps; ++i) {
      const int c = plan.steps[i].c;
      pb.owner_step[c] = int(i);
      pb.cap[c] = est;
      pb.rowmap[c] = static_cast<uint64_t*>(dalloc(ctx, (size_t(pb.n) + 1) * sizeof(uint64_t)));
      pb.live[c] = 1;
      pb.entries[c] = static_cast<uint32_t*>(dalloc(ctx, entries_alloc_bytes(est)));
      // intermediates whose last reader is this step go back to the cache
      // now; their pointers stay in the plan for the launches, and stream
      // order makes the reuse of the blocks by later steps safe
      for (int s : {plan.steps[i].a, plan.steps[i].b, plan.steps[i].d}) {
        if (s > 0 && last_use[s] == int(i) && s != plan.out && pb.live[s]) {
          dfree(ctx, pb.rowmap[s]);
          dfree(ctx, pb.entries[s]);
          pb.live[s] = 0;
        }
      }
    }
  } catch (...) {
    release_build(ctx, pb);
    throw;
  }
  return pb;
}

uint64_t predict_build_bytes(double growth, uint32_t n, uint64_t nentries, unsigned dlo, unsigned dup) {
  const IndexPlan plan = plan_index(dlo, dup);
  std::vector<int> last_use(plan.nslots, -1);
  for (size_t i = 0; i < plan.steps.size(); ++i)
    for (int s : {plan.steps[i].a, plan.steps[i].b, plan.steps[i].d})
      if (s >= 0) last_use[s] = int(i);
  int live = 0, max_live = 1;
  for (size_t i = 0; i < plan.steps.size(); ++i) {
    max_live = std::max(max_live, ++live);
    for (int s : {plan.steps[i].a, plan.steps[i].b, plan.steps[i].d})
      if (s > 0 && last_use[s] == int(i) && s != plan.out) --live;
  }
  const uint64_t input = 8ull * (uint64_t(n) + 1) + 4ull * nentries;
  const uint64_t est = std::max<uint64_t>(uint64_t(growth * double(nentries)), 4ull * n) + 64;
  const uint64_t slot = 8ull * (uint64_t(n) + 1) + entries_alloc_bytes(est);
  // chunk descriptors, and the row kernel's staging: two buffers of 17 words
  // a chunk row per resident CTA -- at most 136 bytes a row, and at most
  // 2 x 17 x 4 bytes x 2048 rows for each of the 2 CTAs of an SM's 148
  const uint64_t stage = std::min<uint64_t>(136ull * n, 2ull * 148 * 2 * 17 * 4 * 2048);
  const uint64_t scratch = plan.steps.size() * ((uint64_t(n) / 64 + 1) * 32 + 512) + stage;
  // the input is held twice while a batch lays it out block-diagonally
  return 2 * input + uint64_t(max_live) * slot + scratch;
}

void release_build(dvg_context* ctx, PlannedBuild& pb) {
  for (int s = 1; s < int(pb.rowmap.size()); ++s) {
    if (pb.live[s]) {
      dfree(ctx, pb.rowmap[s]);
      dfree(ctx, pb.entries[s]);
      pb.live[s] = 0;
    }
  }
  if (pb.scratch) dfree(ctx, pb.scratch);
  pb.scratch = nullptr;
  if (pb.stage) dfree(ctx, pb.stage);
  pb.stage = nullptr;
}

void launch_build(dvg_context* ctx, PlannedBuild& pb, bool timed) {
  const uint64_t t_launch = now_ns();
  struct LaunchTimer {
    dvg_context* ctx;
    uint64_t t0;
    ~LaunchTimer() { ctx->stats.host_launch_ns += now_ns() - t0; }
  } launch_timer{ctx, t_launch};
  DVG_CUDA(cudaMemsetAsync(pb.scratch, 0, pb.scratch_bytes, ctx->stream));
  ctx->stats.kernel_launches++;
  const auto& steps = pb.plan.steps;
  for (size_t i = 0; i < steps.size(); ++i) {
    const PlanStep& st = steps[i];
    RowLaunch L{};
    L.a_identity = st.a_id;
    if (!st.a_id) {
      L.a_rowmap = pb.rowmap[st.a];
      L.a_entries = pb.entries[st.a];
    }
    L.b_rowmap = pb.rowmap[st.b];
    L.b_entries = pb.entries[st.b];
    L.d_identity = st.d_id;
    if (st.d >= 0) {
      L.d_rowmap = pb.rowmap[st.d];
      L.d_entries = pb.entries[st.d];
    }
    L.c_rowmap = pb.rowmap[st.c];
    L.c_entries = pb.entries[st.c];
    L.cap = pb.cap[st.c];
    L.nrows = pb.n;
    L.b_nrows = pb.n;
    L.desc = static_cast<char*>(pb.scratch) + pb.desc_stride * i;
    L.ticket = pb.tickets + i;
    L.ctl = pb.ctls + i;
    L.abort = pb.abort;
    L.stage_buf = pb.stage;
    L.slot_variant = pb.slot_variant;
    cudaEvent_t t0 = timed ? span_begin(ctx) : nullptr;
    launch_rowmode(ctx, L, pb.shape);
    if (t0) span_end(ctx, t0, kProduct);
  }
}

dvg_matrix* finish_build(dvg_context* ctx, PlannedBuild& pb) {
  const size_t nsteps = pb.plan.steps.size();
  const size_t bytes = nsteps * sizeof(DeviceControl) + sizeof(unsigned long long);
  char* h = static_cast<char*>(host_stage(ctx, bytes));
  DVG_CUDA(cudaMemcpyAsync(h, pb.ctls, nsteps * sizeof(DeviceControl), cudaMemcpyDeviceToHost, ctx->stream));
  DVG_CUDA(cudaMemcpyAsync(h + nsteps * sizeof(DeviceControl), pb.abort, sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, ctx->stream));
  const uint64_t t0 = now_ns();
  DVG_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->stats.host_sync_ns += now_ns() - t0;
  ctx->stats.host_syncs++;
  resolve_spans(ctx);
  std::vector<DeviceControl> ctl(nsteps);
  std::memcpy(ctl.data(), h, nsteps * sizeof(DeviceControl));
  unsigned long long aborted = 0;
  std::memcpy(&aborted, h + nsteps * sizeof(DeviceControl), sizeof(aborted));
  for (size_t i = 0; i < nsteps; ++i) {
    if (ctl[i].timeout) {
      release_build(ctx, pb);
      throw Error(DVG_ERR_TIMEOUT, "planned index build: chunk look-back wait expired");
    }
    if (ctl[i].status) {
      release_build(ctx, pb);
      throw Error(DVG_ERR_DEVICE, "internal consistency check failed on the device (code " +
                                      std::to_string(ctl[i].status) + ")");
    }
  }
  // growth of the intermediates over the input (of an aborted run: of the
  // steps that completed before the overflow)
  double grow = 0.0;
  for (size_t i = 0; i < nsteps; ++i)
    if (ctl[i].total) grow = std::max(grow, double(ctl[i].total) / double(std::max<uint64_t>(pb.input->nentries, 1)));
  if (aborted) {
    // the caller re-runs the build and raises the estimate from its sizes
    ctx->plan_growth = std::max(ctx->plan_growth, grow * 1.25);
    release_build(ctx, pb);
    return nullptr;
  }
  // keep the estimate close to what the builds need (memory is reserved, not
  // touched, but it counts against what other work can use)
  ctx->plan_growth = std::max(2.0, std::min(ctx->plan_growth, grow * 1.5 + 0.5));
  // statistics: the bytes every step had to move
  std::vector<uint64_t> sz(pb.plan.nslots, 0);
  sz[0] = pb.input->nentries;
  auto mbytes = [&](int s) { return 8ull * (uint64_t(pb.n) + 1) + 4ull * sz[s]; };
  for (size_t i = 0; i < nsteps; ++i) {
    const PlanStep& st = pb.plan.steps[i];
    sz[st.c] = ctl[i].total;
    const uint64_t b = (st.a_id ? 0 : mbytes(st.a)) + mbytes(st.b) + (st.d >= 0 ? mbytes(st.d) : 0) + mbytes(st.c);
    ctx->stats.alg_bytes += b;
    ctx->stats.spgemm_alg_bytes += b;
    ctx->stats.spgemm_calls++;
    if (st.d >= 0 || st.d_id) ctx->stats.spgemm_fused_adds++;
    ctx->stats.spgemm_slow_rows += ctl[i].slow_rows;
  }
  const int out = pb.plan.out;
  const size_t out_step = size_t(pb.owner_step[out]);
  auto* m = new dvg_matrix();
  m->nrows = pb.n;
  m->ncols = pb.input->ncols;
  m->nentries = ctl[out_step].total;
  m->nnz = ctl[out_step].nnz;
  m->canonical = true;
  m->device = ctx->device;
  m->rowmap = pb.rowmap[out];
  // hand the slack of the estimated capacity back: copy into an exact buffer
  if (pb.cap[out] > m->nentries + m->nentries / 4 + (1u << 18)) {
    try {
      m->entries = static_cast<uint32_t*>(dalloc(ctx, entries_alloc_bytes(m->nentries)));
    } catch (...) {
      delete m;
      release_build(ctx, pb);
      throw;
    }
    if (m->nentries)
      DVG_CUDA(cudaMemcpyAsync(m->entries, pb.entries[out], m->nentries * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, ctx->stream));
    dfree(ctx, pb.entries[out]);
  } else {
    m->entries = pb.entries[out];
  }
  pb.live[out] = 0;
  release_build(ctx, pb);
  return m;
}

}  // namespace dvg
