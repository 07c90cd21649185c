// dvg_serve.cu -- the request loop: index builds and query batches as they
// arrive, indices resident in HBM, continuous batching.
//
// Workers share one GPU, each with its own context (stream, allocator):
//  * build_workers build workers (2 by default): a free worker admits the
//    waiting builds in arrival order while their predicted footprint
//    (predict_build_bytes: the planned build's live buffers at its estimated
//    capacities) fits the HBM budget next to the resident indices and the
//    builds in flight, uploads them and builds all admitted graphs as one
//    batch (dvg_batch.cu: one CUDA-graph launch per batch).  A build that
//    arrives while batches are on the GPU is taken by the next free worker at
//    once -- its work overlaps theirs on another stream -- or, with every
//    worker busy, joins the next batch as slots and memory free up.  Each
//    request is checked on its own upload: a malformed graph fails alone, and
//    if a batch fails as a whole its members are rebuilt one by one, so one
//    bad request never fails its batch-mates;
//  * the query worker issues every query batch whose index is resident on its
//    own stream -- pairs in, membership kernel, answers out, an event -- with
//    up to max_inflight_queries batches on the device at once, concurrently
//    with the build worker's batches, and completes them as their events
//    fire.
// A request's result does not depend on what else is in flight: a batch
// builds each graph's block exactly (block-diagonal layout), and a query
// reads one immutable index.
//
// The reference has no serving layer: it builds an index per call
// (dindex.hpp:46-189) and answers one pair per call (crs_matrix.hpp:1197-1243).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "dvg_internal.h"

namespace {

using dvg::Error;

struct BuildReq {
  uint64_t id;
  uint32_t n;
  const uint64_t* rowmap;
  const uint32_t* entries;
  uint64_t nentries;
  unsigned dmin, dmax;
  uint64_t submit_ns;
  uint64_t predicted;
};

struct QueryReq {
  uint64_t id;
  uint64_t index;
  const uint32_t* pairs;
  uint64_t npairs;
  uint8_t* answers;
  uint64_t submit_ns;
};

struct ServerIndex {
  dvg_matrix* m = nullptr;  // allocated by the build context `owner`
  dvg_context* owner = nullptr;
  int state = 0;            // 0 building, 1 resident, -1 failed
  dvg_status error = DVG_OK;
  uint64_t bytes = 0;
  uint32_t users = 0;       // query batches and downloads in flight on it
  bool released = false;
};

// One query batch's device and pinned host buffers, reused.
struct QuerySlot {
  uint32_t* d_pairs = nullptr;
  uint8_t* d_out = nullptr;
  DeviceControl* d_ctl = nullptr;
  uint32_t* h_pairs = nullptr;
  uint8_t* h_out = nullptr;
  DeviceControl* h_ctl = nullptr;
  uint64_t cap = 0;  // pairs (device buffers)
  uint64_t h_pairs_cap = 0, h_out_cap = 0;  // bytes (pinned staging)
  cudaEvent_t done = nullptr;
  bool busy = false;
  QueryReq req{};
  uint64_t start_ns = 0;
  bool staged_out = false;
};

}  // namespace

struct dvg_server {
  dvg_server_config cfg{};
  std::vector<dvg_context*> bctxs;  // one per build worker
  dvg_context* qctx = nullptr;
  std::mutex mu;
  std::condition_variable cv_build, cv_query, cv_done;
  std::deque<BuildReq> builds;
  std::deque<QueryReq> queries;
  std::unordered_map<uint64_t, ServerIndex> indices;
  std::vector<std::pair<dvg_context*, dvg_matrix*>> to_free;  // released indices (owner, matrix)
  std::vector<void*> retired_host;   // outgrown pinned staging, freed at shutdown
  std::deque<dvg_completion> done;
  uint64_t next_id = 1;
  uint64_t resident = 0, reserved = 0;
  double growth = 3.0;  // the build context's capacity estimate, for admission
  dvg_server_stats st{};
  bool stop = false;
  std::vector<std::thread> tbs;
  std::thread tq;
  std::vector<QuerySlot> slots;
};

namespace {

uint64_t now() {
  return uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(
                      std::chrono::steady_clock::now().time_since_epoch()).count());
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Caller holds s->mu.
void complete(dvg_server* s, const dvg_completion& c) {
  s->done.push_back(c);
  s->cv_done.notify_all();
}

// Caller holds s->mu: drops a released index once nothing uses it.
void maybe_drop(dvg_server* s, uint64_t id) {
  auto f = s->indices.find(id);
  if (f == s->indices.end() || !f->second.released || f->second.users) return;
  if (f->second.m) {
    s->to_free.emplace_back(f->second.owner, f->second.m);
    s->resident -= f->second.bytes;
  }
  s->indices.erase(f);
  s->st.resident_bytes = s->resident;
  s->cv_build.notify_all();
}

// ---- build workers -----------------------------------------------------------

// Frees released indices, each by the context that allocated it.
void free_released(std::vector<std::pair<dvg_context*, dvg_matrix*>>& frees) {
  for (auto& f : frees) {
    std::lock_guard<std::recursive_mutex> owner_lock(f.first->mu);
    dvg::free_matrix(f.first, f.second);
  }
  frees.clear();
}

void build_worker(dvg_server* s, size_t w) {
  dvg_context* ctx = s->bctxs[w];
  cudaSetDevice(s->cfg.device);
  for (;;) {
    std::vector<BuildReq> batch;
    std::vector<std::pair<dvg_context*, dvg_matrix*>> frees;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_build.wait(lk, [&] { return s->stop || !s->builds.empty() || !s->to_free.empty(); });
      frees.swap(s->to_free);
      if (s->stop && s->builds.empty() && frees.empty()) break;
      const uint64_t held = s->resident + s->reserved;
      uint64_t avail = s->cfg.hbm_budget_bytes > held ? s->cfg.hbm_budget_bytes - held : 0;
      while (!s->builds.empty() && batch.size() < s->cfg.max_batch_builds) {
        BuildReq& r = s->builds.front();
        if (r.predicted > avail) {
          if (batch.empty() && r.predicted > s->cfg.hbm_budget_bytes) {
            // can never fit the budget
            ServerIndex& ix = s->indices[r.id];
            ix.state = -1;
            ix.error = DVG_ERR_OOM;
            dvg_completion c{};
            c.request = r.id;
            c.status = DVG_ERR_OOM;
            c.kind = 1;
            c.submit_ns = r.submit_ns;
            c.start_ns = c.done_ns = now();
            complete(s, c);
            s->builds.pop_front();
            s->cv_query.notify_all();
            continue;
          }
          break;  // waits until builds in flight finish or released indices free memory
        }
        avail -= r.predicted;
        s->reserved += r.predicted;
        batch.push_back(r);
        s->builds.pop_front();
      }
      s->st.peak_reserved_bytes = std::max(s->st.peak_reserved_bytes, s->reserved + s->resident);
      if (batch.empty() && frees.empty()) {
        s->cv_build.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
    }
    // ---- GPU work, outside the server lock ----------------------------------
    free_released(frees);
    if (batch.empty()) continue;
    std::lock_guard<std::recursive_mutex> ctx_lock(ctx->mu);
    const uint64_t t_start = now();
    const size_t nb = batch.size();
    std::vector<dvg_matrix*> in(nb, nullptr), out(nb, nullptr);
    std::vector<dvg_status> status(nb, DVG_OK);
    std::vector<std::string> why(nb);
    // every request's upload checked on its own: a malformed graph fails alone
    std::vector<size_t> ok;
    for (size_t k = 0; k < nb; ++k) {
      try {
        in[k] = dvg::upload_matrix(ctx, batch[k].n, batch[k].n, batch[k].rowmap, batch[k].entries, 0);
        ok.push_back(k);
      } catch (const Error& e) {
        status[k] = e.status;
        why[k] = e.what();
      } catch (const std::exception& e) {
        status[k] = DVG_ERR_DEVICE;
        why[k] = e.what();
      }
    }
    auto build = [&](const std::vector<size_t>& members) {
      std::vector<dvg_matrix*> gi, go(members.size(), nullptr);
      std::vector<unsigned> lo, hi;
      for (size_t k : members) {
        gi.push_back(in[k]);
        lo.push_back(batch[k].dmin);
        hi.push_back(batch[k].dmax);
      }
      dvg::batch_distance_index(ctx, uint32_t(members.size()), gi.data(), lo.data(), hi.data(), go.data());
      for (size_t q = 0; q < members.size(); ++q) out[members[q]] = go[q];
    };
    size_t reruns = 0;
    if (!ok.empty()) {
      try {
        build(ok);
      } catch (const std::exception&) {
        // the batch failed as a whole: its members one by one, so a request
        // that cannot build fails alone
        for (size_t k : ok) {
          ++reruns;
          try {
            build(std::vector<size_t>{k});
          } catch (const Error& e) {
            status[k] = e.status;
            why[k] = e.what();
          } catch (const std::exception& e) {
            status[k] = DVG_ERR_DEVICE;
            why[k] = e.what();
          }
        }
      }
    }
    // the indices are read on the query context's stream from here on: the
    // last kernels that write them (the batch's split, an exact-size copy)
    // are still queued on this stream when the build returns, so wait for them
    {
      const uint64_t ts = now();
      const cudaError_t e = cudaStreamSynchronize(ctx->stream);
      ctx->stats.host_sync_ns += now() - ts;
      ctx->stats.host_syncs++;
      if (e != cudaSuccess) {
        for (size_t k = 0; k < nb; ++k) {
          if (status[k] == DVG_OK) {
            status[k] = DVG_ERR_DEVICE;
            why[k] = std::string("build batch: ") + cudaGetErrorString(e);
          }
          out[k] = nullptr;  // never published; the context is unusable after a device error
        }
      }
    }
    for (dvg_matrix* m : in)
      if (m) dvg::free_matrix(ctx, m);
    const uint64_t t_done = now();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->growth = std::max(s->growth, ctx->plan_growth);
      s->st.build_batches++;
      s->st.builds_rebuilt_alone += reruns;
      s->st.build_batch_ns_max = std::max(s->st.build_batch_ns_max, t_done - t_start);
      uint64_t alloc_ns = 0, sync_ns = 0, cap_reruns = 0;
      for (dvg_context* c : s->bctxs) {
        alloc_ns += c->stats.host_alloc_ns;
        sync_ns += c->stats.host_sync_ns;
        cap_reruns += c->stats.spgemm_reruns;
      }
      s->st.build_alloc_ns = alloc_ns;
      s->st.build_sync_ns = sync_ns;
      s->st.build_reruns = cap_reruns;
      for (size_t k = 0; k < nb; ++k) {
        ServerIndex& ix = s->indices[batch[k].id];
        s->reserved -= batch[k].predicted;
        dvg_completion c{};
        c.request = batch[k].id;
        c.kind = 1;
        c.submit_ns = batch[k].submit_ns;
        c.start_ns = t_start;
        c.done_ns = t_done;
        if (status[k] == DVG_OK && out[k]) {
          ix.m = out[k];
          ix.owner = ctx;
          ix.state = 1;
          ix.bytes = dvg::matrix_bytes(out[k]);
          s->resident += ix.bytes;
          c.status = DVG_OK;
          c.index_entries = out[k]->nentries;
          c.index_nnz = out[k]->nnz;
          s->st.builds_done++;
        } else {
          ix.state = -1;
          ix.error = status[k] == DVG_OK ? DVG_ERR_DEVICE : status[k];
          c.status = ix.error;
          s->st.builds_failed++;
          if (!why[k].empty()) dvg::record_error(why[k]);
        }
        complete(s, c);
      }
      s->st.resident_bytes = s->resident;
    }
    s->cv_query.notify_all();
    s->cv_build.notify_all();  // reserved memory came back: another worker may admit now
  }
}

// ---- query worker -------------------------------------------------------------

// Device buffers of a slot grow by doubling (stream-ordered, through the
// context's cache).  Pinned staging is only made for callers whose buffers
// are pageable, also by doubling; outgrown pinned buffers are kept until the
// server shuts down, because cudaFreeHost waits for the whole device and would
// stall the build stream.
void ensure_slot(dvg_server* s, QuerySlot& q, uint64_t npairs, bool stage_in, bool stage_out) {
  dvg_context* ctx = s->qctx;
  if (npairs > q.cap) {
    const uint64_t cap = std::max<uint64_t>({npairs, 2 * q.cap, uint64_t(1) << 16});
    if (q.d_pairs) dvg::dfree(ctx, q.d_pairs);
    if (q.d_out) dvg::dfree(ctx, q.d_out);
    q.d_pairs = nullptr;
    q.d_out = nullptr;
    q.cap = 0;
    q.d_pairs = static_cast<uint32_t*>(dvg::dalloc(ctx, cap * 8));
    q.d_out = static_cast<uint8_t*>(dvg::dalloc(ctx, cap));
    q.cap = cap;
  }
  auto grow_host = [&](void*& h, uint64_t& hcap, uint64_t bytes) {
    if (bytes <= hcap) return;
    const uint64_t want = std::max<uint64_t>({bytes, 2 * hcap, uint64_t(1) << 16});
    void* p = nullptr;
    DVG_CUDA(cudaMallocHost(&p, want));
    if (h) s->retired_host.push_back(h);
    h = p;
    hcap = want;
  };
  if (stage_in) grow_host(reinterpret_cast<void*&>(q.h_pairs), q.h_pairs_cap, npairs * 8);
  if (stage_out) grow_host(reinterpret_cast<void*&>(q.h_out), q.h_out_cap, npairs);
}

// Issues one query batch on the query context's stream.
void issue_query(dvg_server* s, QuerySlot& q, const QueryReq& r, const dvg_matrix* idx) {
  dvg_context* ctx = s->qctx;
  const bool stage_in = r.npairs && !is_pinned(r.pairs);
  q.staged_out = r.npairs && !is_pinned(r.answers);
  ensure_slot(s, q, r.npairs, stage_in, q.staged_out);
  const uint32_t* src = r.pairs;
  if (stage_in) {
    std::memcpy(q.h_pairs, r.pairs, r.npairs * 8);
    src = q.h_pairs;
  }
  uint8_t* dst = q.staged_out ? q.h_out : r.answers;
  DVG_CUDA(cudaMemsetAsync(q.d_ctl, 0, sizeof(DeviceControl), ctx->stream));
  if (r.npairs) {
    DVG_CUDA(cudaMemcpyAsync(q.d_pairs, src, r.npairs * 8, cudaMemcpyHostToDevice, ctx->stream));
    dvg::launch_query(ctx, idx, q.d_pairs, r.npairs, q.d_out, q.d_ctl);
    DVG_CUDA(cudaMemcpyAsync(dst, q.d_out, r.npairs, cudaMemcpyDeviceToHost, ctx->stream));
  }
  DVG_CUDA(cudaMemcpyAsync(q.h_ctl, q.d_ctl, sizeof(DeviceControl), cudaMemcpyDeviceToHost, ctx->stream));
  DVG_CUDA(cudaEventRecord(q.done, ctx->stream));
  ctx->stats.h2d_bytes += r.npairs * 8;
  ctx->stats.d2h_bytes += r.npairs;
}

void query_worker(dvg_server* s) {
  cudaSetDevice(s->cfg.device);
  for (;;) {
    bool busy = false;
    // completions
    for (auto& q : s->slots) {
      if (!q.busy) continue;
      const cudaError_t e = cudaEventQuery(q.done);
      if (e == cudaErrorNotReady) {
        busy = true;
        continue;
      }
      dvg_status status = DVG_OK;
      if (e != cudaSuccess) {
        status = DVG_ERR_DEVICE;
        dvg::record_error(std::string("query batch: ") + cudaGetErrorString(e));
      }
      if (status == DVG_OK && q.staged_out) std::memcpy(q.req.answers, q.h_out, q.req.npairs);
      if (status == DVG_OK && q.h_ctl->status) {
        status = DVG_ERR_DEVICE;
        dvg::record_error("query batch: the index's row pointers lie outside its entries");
      }
      const uint64_t invalid = status == DVG_OK ? q.h_ctl->invalid : 0;
      std::lock_guard<std::mutex> lk(s->mu);
      auto f = s->indices.find(q.req.index);
      if (f != s->indices.end()) f->second.users--;
      maybe_drop(s, q.req.index);
      dvg_completion c{};
      c.request = q.req.id;
      c.kind = 2;
      c.status = status == DVG_OK && invalid ? DVG_ERR_INVALID_ARG : status;
      c.submit_ns = q.req.submit_ns;
      c.start_ns = q.start_ns;
      c.done_ns = now();
      c.invalid_pairs = invalid;
      s->st.queries_done++;
      s->st.pairs_answered += q.req.npairs;
      complete(s, c);
      q.busy = false;
    }
    // new work: every waiting batch whose index is resident, in arrival order
    std::vector<std::pair<QueryReq, const dvg_matrix*>> ready;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->stop && s->queries.empty() && !busy) break;
      size_t free_slots = 0;
      for (auto& q : s->slots) free_slots += q.busy ? 0 : 1;
      for (auto it = s->queries.begin(); it != s->queries.end() && ready.size() < free_slots;) {
        auto f = s->indices.find(it->index);
        if (f == s->indices.end() || f->second.state == -1 || f->second.released) {
          dvg_completion c{};
          c.request = it->id;
          c.kind = 2;
          c.status = f == s->indices.end() || f->second.released ? DVG_ERR_INVALID_ARG : f->second.error;
          c.submit_ns = it->submit_ns;
          c.start_ns = c.done_ns = now();
          complete(s, c);
          it = s->queries.erase(it);
          continue;
        }
        if (f->second.state == 1) {
          f->second.users++;
          ready.emplace_back(*it, f->second.m);
          it = s->queries.erase(it);
          continue;
        }
        ++it;  // its index is still being built
      }
      if (ready.empty() && !busy) {
        s->cv_query.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
    }
    if (ready.empty()) {
      std::this_thread::sleep_for(std::chrono::microseconds(20));
      continue;
    }
    std::lock_guard<std::recursive_mutex> ctx_lock(s->qctx->mu);
    size_t k = 0;
    for (auto& q : s->slots) {
      if (k == ready.size()) break;
      if (q.busy) continue;
      q.req = ready[k].first;
      q.start_ns = now();
      dvg_status status = DVG_OK;
      try {
        issue_query(s, q, q.req, ready[k].second);
        q.busy = true;
      } catch (const Error& e) {
        status = e.status;
        dvg::record_error(e.what());
      }
      if (status != DVG_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        auto f = s->indices.find(q.req.index);
        if (f != s->indices.end()) f->second.users--;
        maybe_drop(s, q.req.index);
        dvg_completion c{};
        c.request = q.req.id;
        c.kind = 2;
        c.status = status;
        c.submit_ns = q.req.submit_ns;
        c.start_ns = c.done_ns = now();
        complete(s, c);
      }
      ++k;
    }
  }
}

}  // namespace

extern "C" {

dvg_status dvg_server_create(const dvg_server_config* cfg, dvg_server** out) {
  if (!cfg || !out) {
    dvg::record_error("null argument");
    return DVG_ERR_INVALID_ARG;
  }
  *out = nullptr;
  auto* s = new dvg_server();
  s->cfg = *cfg;
  if (!s->cfg.max_batch_builds) s->cfg.max_batch_builds = 64;
  if (!s->cfg.max_inflight_queries) s->cfg.max_inflight_queries = 8;
  if (!s->cfg.build_workers) s->cfg.build_workers = 2;
  dvg_status st = DVG_OK;
  for (uint32_t w = 0; w < s->cfg.build_workers && st == DVG_OK; ++w) {
    dvg_context* c = nullptr;
    st = dvg_init(cfg->device, &c);
    if (st == DVG_OK) s->bctxs.push_back(c);
  }
  if (st == DVG_OK) st = dvg_init(cfg->device, &s->qctx);
  if (st == DVG_OK) {
    try {
      // queries run on the device's highest-priority stream: when a build
      // kernel's CTAs retire, a waiting query kernel is scheduled before the
      // build's next kernel, so a query waits for one kernel, not a batch
      int prio_lo = 0, prio_hi = 0;
      DVG_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
      DVG_CUDA(cudaStreamDestroy(s->qctx->own_stream));
      s->qctx->own_stream = nullptr;
      DVG_CUDA(cudaStreamCreateWithPriority(&s->qctx->own_stream, cudaStreamNonBlocking, prio_hi));
      s->qctx->stream = s->qctx->own_stream;
      if (!s->cfg.hbm_budget_bytes) {
        size_t free_b = 0, total_b = 0;
        DVG_CUDA(cudaMemGetInfo(&free_b, &total_b));
        s->cfg.hbm_budget_bytes = uint64_t(0.8 * double(free_b));
      }
      // map device memory into the stream-ordered pool now, once: growing the
      // pool under a build batch costs about 0.2 s per GB, all of it latency
      // of the requests in the batch.  The pool keeps freed memory (release
      // threshold at maximum), so later allocations up to this size only
      // suballocate.
      {
        const uint64_t warm = std::min<uint64_t>(s->cfg.hbm_budget_bytes, uint64_t(8) << 30);
        void* p = nullptr;
        if (cudaMallocAsync(&p, warm, s->bctxs[0]->stream) == cudaSuccess) {
          DVG_CUDA(cudaFreeAsync(p, s->bctxs[0]->stream));
          DVG_CUDA(cudaStreamSynchronize(s->bctxs[0]->stream));
        } else {
          (void)cudaGetLastError();
        }
      }
      s->slots.resize(s->cfg.max_inflight_queries);
      for (auto& q : s->slots) {
        q.d_ctl = static_cast<DeviceControl*>(dvg::dalloc(s->qctx, sizeof(DeviceControl)));
        DVG_CUDA(cudaMallocHost(&q.h_ctl, sizeof(DeviceControl)));
        DVG_CUDA(cudaEventCreateWithFlags(&q.done, cudaEventDisableTiming));
      }
      s->growth = s->bctxs[0]->plan_growth;
      // batches in a request stream vary in size: no timing runs on the way
      for (dvg_context* c : s->bctxs) c->opt_autotune = 0;
      s->st.hbm_budget_bytes = s->cfg.hbm_budget_bytes;
    } catch (const Error& e) {
      dvg::record_error(e.what());
      st = e.status;
    }
  }
  if (st != DVG_OK) {
    for (auto& q : s->slots) {
      if (q.h_ctl) cudaFreeHost(q.h_ctl);
      if (q.done) cudaEventDestroy(q.done);
    }
    if (s->qctx) dvg_shutdown(s->qctx);
    for (dvg_context* c : s->bctxs) dvg_shutdown(c);
    delete s;
    return st;
  }
  for (size_t w = 0; w < s->bctxs.size(); ++w) s->tbs.emplace_back(build_worker, s, w);
  s->tq = std::thread(query_worker, s);
  *out = s;
  return DVG_OK;
}

dvg_status dvg_server_destroy(dvg_server* s) {
  if (!s) return DVG_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_build.notify_all();
  s->cv_query.notify_all();
  for (auto& t : s->tbs) t.join();
  s->tq.join();
  for (auto& kv : s->indices)
    if (kv.second.m) dvg::free_matrix(kv.second.owner, kv.second.m);
  free_released(s->to_free);
  for (auto& q : s->slots) {
    if (q.h_pairs) cudaFreeHost(q.h_pairs);
    if (q.h_out) cudaFreeHost(q.h_out);
    if (q.h_ctl) cudaFreeHost(q.h_ctl);
    if (q.done) cudaEventDestroy(q.done);
  }
  for (void* h : s->retired_host) cudaFreeHost(h);
  dvg_status a = dvg_shutdown(s->qctx), b = DVG_OK;
  for (dvg_context* c : s->bctxs) {
    const dvg_status x = dvg_shutdown(c);
    if (b == DVG_OK) b = x;
  }
  delete s;
  return a != DVG_OK ? a : b;
}

dvg_status dvg_server_submit_build(dvg_server* s, uint32_t n, const uint64_t* rowmap, const uint32_t* entries,
                                   unsigned dmin, unsigned dmax, uint64_t* request) {
  if (!s || !rowmap || !request) {
    dvg::record_error("null argument");
    return DVG_ERR_INVALID_ARG;
  }
  if (dmin > dmax || dmax == 0) {
    dvg::record_error("build: requires dmin <= dmax and dmax != 0");
    return DVG_ERR_INVALID_ARG;
  }
  const uint64_t ne = rowmap[n];
  if (ne && !entries) {
    dvg::record_error("null entries");
    return DVG_ERR_INVALID_ARG;
  }
  BuildReq r{0, n, rowmap, entries, ne, dmin, dmax, now(), 0};
  std::lock_guard<std::mutex> lk(s->mu);
  r.predicted = dvg::predict_build_bytes(s->growth, n, ne, dmin, dmax);
  r.id = s->next_id++;
  s->indices[r.id];  // state 0: building
  s->builds.push_back(r);
  s->st.builds_submitted++;
  *request = r.id;
  s->cv_build.notify_all();
  return DVG_OK;
}

dvg_status dvg_server_submit_query(dvg_server* s, uint64_t index, const uint32_t* pairs, uint64_t npairs,
                                   uint8_t* answers, uint64_t* request) {
  if (!s || !request || (npairs && (!pairs || !answers))) {
    dvg::record_error("null argument");
    return DVG_ERR_INVALID_ARG;
  }
  if (reinterpret_cast<uintptr_t>(pairs) & 7) {
    dvg::record_error("pairs must be 8-byte aligned");
    return DVG_ERR_INVALID_ARG;
  }
  QueryReq r{0, index, pairs, npairs, answers, now()};
  std::lock_guard<std::mutex> lk(s->mu);
  r.id = s->next_id++;
  s->queries.push_back(r);
  s->st.queries_submitted++;
  *request = r.id;
  s->cv_query.notify_all();
  return DVG_OK;
}

dvg_status dvg_server_poll(dvg_server* s, dvg_completion* out, uint32_t max, uint32_t* n, uint32_t wait_ms) {
  if (!s || !n || (max && !out)) return DVG_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->done.empty() && wait_ms)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
  uint32_t k = 0;
  while (k < max && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  *n = k;
  return DVG_OK;
}

dvg_status dvg_server_index_info(dvg_server* s, uint64_t index, uint32_t* nrows, uint64_t* nentries, uint64_t* nnz) {
  if (!s) return DVG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto f = s->indices.find(index);
  if (f == s->indices.end() || f->second.state != 1 || f->second.released) {
    dvg::record_error("no resident index with that id");
    return DVG_ERR_INVALID_ARG;
  }
  if (nrows) *nrows = f->second.m->nrows;
  if (nentries) *nentries = f->second.m->nentries;
  if (nnz) *nnz = f->second.m->nnz;
  return DVG_OK;
}

dvg_status dvg_server_download(dvg_server* s, uint64_t index, uint64_t* rowmap, uint32_t* entries) {
  if (!s || !rowmap) return DVG_ERR_INVALID_ARG;
  dvg_matrix* m = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto f = s->indices.find(index);
    if (f == s->indices.end() || f->second.state != 1 || f->second.released) {
      dvg::record_error("no resident index with that id");
      return DVG_ERR_INVALID_ARG;
    }
    m = f->second.m;
    f->second.users++;
  }
  const dvg_status st = dvg_matrix_download(s->qctx, m, rowmap, entries);
  std::lock_guard<std::mutex> lk(s->mu);
  auto f = s->indices.find(index);
  if (f != s->indices.end()) f->second.users--;
  maybe_drop(s, index);
  return st;
}

dvg_status dvg_server_release(dvg_server* s, uint64_t index) {
  if (!s) return DVG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto f = s->indices.find(index);
  if (f == s->indices.end() || f->second.released || f->second.state == 0) {
    dvg::record_error("no resident index with that id");
    return DVG_ERR_INVALID_ARG;
  }
  f->second.released = true;
  maybe_drop(s, index);
  return DVG_OK;
}

dvg_status dvg_server_get_stats(dvg_server* s, dvg_server_stats* out) {
  if (!s || !out) return DVG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident_bytes = s->resident;
  return DVG_OK;
}

}  // extern "C"
