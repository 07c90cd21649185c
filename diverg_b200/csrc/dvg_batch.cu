// dvg_batch.cu -- many independent graphs built in one CUDA-graph launch.
//
// A batch of adjacency matrices with their distance windows is grouped by
// window.  The graphs of a group are laid side by side as one block-diagonal
// matrix: the powers of a block-diagonal matrix, and so its distance index,
// are block-diagonal with the graphs' own indices as blocks (no range of a
// row ever leaves its block, so no two blocks' ranges meet in a row).  Every
// group is one planned build (dvg_engine.cu); the assembly kernels and all
// groups' steps are captured into one CUDA graph and launched once.  Each
// graph's index is then cut out of its group's result (rows rebased, columns
// shifted back), giving exactly what a build of that graph alone gives.
//
// The reference builds graphs one at a time (dindex.hpp:46-189 per
// component); its own combination of components (crs_matrix.hpp:1448-1518
// builds rows component by component) is the layout used here.
//
// The autotuner times the row kernel's run-list width and chunk shape on the
// first group of each (window, size class) it meets and keeps the fastest.
#include <algorithm>
#include <cstring>
#include <map>
#include <tuple>

#include "dvg_internal.h"

namespace dvg {
namespace {

struct GraphSlice {
  const uint64_t* rowmap;
  const uint32_t* entries;
  unsigned long long row_off;  // first row (and column) of the graph in the group
  unsigned long long ent_off;  // first entry of the graph in the group
};

// Index k of the slice holding position x, for offsets off(0) = 0 <= ... <= off(ng).
template <class Off>
__device__ __forceinline__ uint32_t find_slice(uint32_t ng, unsigned long long x, Off off) {
  uint32_t lo = 0, hi = ng;  // off(lo) <= x < off(hi)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off(mid) <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Block-diagonal assembly: s[0..ng] (s[ng] holds the totals).
__global__ void k_assemble(const GraphSlice* __restrict__ s, uint32_t ng, uint64_t* __restrict__ rowmap,
                           uint32_t* __restrict__ entries) {
  const unsigned long long n = s[ng].row_off, e = s[ng].ent_off;
  const unsigned long long stride = 1ull * gridDim.x * blockDim.x;
  const unsigned long long t0 = 1ull * blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 == 0) rowmap[0] = 0;
  for (unsigned long long i = t0; i < n; i += stride) {
    const uint32_t k = find_slice(ng, i, [&](uint32_t j) { return s[j].row_off; });
    rowmap[i + 1] = s[k].rowmap[i - s[k].row_off + 1] + s[k].ent_off;
  }
  for (unsigned long long x = t0; x < e; x += stride) {
    const uint32_t k = find_slice(ng, x, [&](uint32_t j) { return s[j].ent_off; });
    entries[x] = uint32_t(s[k].entries[x - s[k].ent_off] + s[k].row_off);
  }
}

// bounds[k] = rowmap[s[k].row_off] for k <= ng: where each graph's index starts.
__global__ void k_bounds(const GraphSlice* __restrict__ s, uint32_t ng, const uint64_t* __restrict__ rowmap,
                         unsigned long long* __restrict__ bounds) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= ng; k += gridDim.x * blockDim.x)
    bounds[k] = rowmap[s[k].row_off];
}

// nnz[k] += the lengths of graph k's ranges, for ranges [bounds[0], bounds[ng]) / 2
// of the group's index; warps take contiguous blocks (a graph boundary is
// rare inside one), lanes keep a running sum per graph and flush on change.
__global__ void k_graph_nnz(const unsigned long long* __restrict__ bounds, uint32_t ng,
                            const uint32_t* __restrict__ entries, unsigned long long* __restrict__ nnz) {
  const unsigned long long r0 = bounds[0] >> 1, r1 = bounds[ng] >> 1;
  const unsigned lane = threadIdx.x & 31;
  const unsigned long long warp = (1ull * blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = (1ull * gridDim.x * blockDim.x) >> 5;
  uint32_t kcur = 0xffffffffu;
  unsigned long long sum = 0;
  for (unsigned long long blk = r0 + warp * 1024; blk < r1; blk += nwarps * 1024) {
    const unsigned long long end = min(blk + 1024, r1);
    for (unsigned long long r = blk + lane; r < end; r += 32) {
      const uint32_t k = find_slice(ng, 2 * r, [&](uint32_t j) { return bounds[j]; });
      if (k != kcur) {
        if (kcur != 0xffffffffu && sum) atomicAdd(nnz + kcur, sum);
        kcur = k;
        sum = 0;
      }
      const uint2 e = reinterpret_cast<const uint2*>(entries)[r];
      sum += uint64_t(e.y) - e.x + 1;
    }
  }
  if (kcur != 0xffffffffu && sum) atomicAdd(nnz + kcur, sum);
}

struct OutSlice {
  uint64_t* rowmap;
  uint32_t* entries;
  unsigned long long row_off;
  unsigned long long ent_off;  // bounds[k]
};

// Cuts the graphs' indices out of the group's: o[0..ng] (o[ng] holds the totals).
__global__ void k_split(const OutSlice* __restrict__ o, uint32_t ng, const uint64_t* __restrict__ rowmap,
                        const uint32_t* __restrict__ entries) {
  const unsigned long long n = o[ng].row_off, e = o[ng].ent_off;
  const unsigned long long stride = 1ull * gridDim.x * blockDim.x;
  const unsigned long long t0 = 1ull * blockIdx.x * blockDim.x + threadIdx.x;
  for (unsigned long long k = t0; k < ng; k += stride) o[k].rowmap[0] = 0;
  for (unsigned long long i = t0; i < n; i += stride) {
    const uint32_t k = find_slice(ng, i, [&](uint32_t j) { return o[j].row_off; });
    o[k].rowmap[i - o[k].row_off + 1] = rowmap[i + 1] - o[k].ent_off;
  }
  for (unsigned long long x = t0; x < e; x += stride) {
    const uint32_t k = find_slice(ng, x, [&](uint32_t j) { return o[j].ent_off; });
    o[k].entries[x - o[k].ent_off] = uint32_t(entries[x] - o[k].row_off);
  }
}

unsigned grid_for(dvg_context* ctx, unsigned long long work) {
  const unsigned long long want = (work + 255) / 256;
  return unsigned(std::max<unsigned long long>(1, std::min<unsigned long long>(want, 8ull * ctx->num_sms)));
}

struct Group {
  unsigned dlo, dup;
  std::vector<uint32_t> members;   // indices into the batch
  std::vector<GraphSlice> slices;  // ng + 1
  dvg_matrix* g = nullptr;         // block-diagonal input
  dvg_matrix* t = nullptr;         // block-diagonal index
  PlannedBuild pb;
  bool planned = false;
  size_t table_off = 0;            // slices in the device table (GraphSlice units)
};

}  // namespace

// Times planned builds of `a` over the candidate kernel shapes and keeps the
// fastest per (window, size class).
TuneChoice autotune_build(dvg_context* ctx, const dvg_matrix* a, unsigned dlo, unsigned dup) {
  const int size_class = 64 - __builtin_clzll(uint64_t(a->nrows) | 1ull);
  const auto key = std::make_tuple(dlo, dup, size_class);
  auto it = ctx->tuned.find(key);
  if (it != ctx->tuned.end()) return it->second;
  const IndexPlan plan = plan_index(dlo, dup);
  TuneChoice best{int(ctx->opt_row_slot), 0};
  float best_ms = -1.f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // one build to warm the allocator cache, then every candidate once
  std::vector<TuneChoice> cands{best};
  for (int v = 0; v < 3; ++v)
    for (int64_t chunk : {int64_t(512), int64_t(1024), int64_t(2048)}) cands.push_back(TuneChoice{v, chunk});
  try {
    DVG_CUDA(cudaEventCreate(&e0));
    DVG_CUDA(cudaEventCreate(&e1));
    for (size_t c = 0; c < cands.size(); ++c) {
      PlannedBuild pb = prepare_build(ctx, plan, a, cands[c].slot_variant, cands[c].chunk_rows);
      DVG_CUDA(cudaEventRecord(e0, ctx->stream));
      try {
        launch_build(ctx, pb, false);
      } catch (...) {
        release_build(ctx, pb);
        throw;
      }
      DVG_CUDA(cudaEventRecord(e1, ctx->stream));
      dvg_matrix* t = finish_build(ctx, pb);
      if (!t) continue;  // outgrew the estimate: no timing
      free_matrix(ctx, t);
      ctx->stats.autotune_builds++;
      if (c == 0) continue;
      float ms = 0.f;
      DVG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (best_ms < 0.f || ms < best_ms) {
        best_ms = ms;
        best = cands[c];
      }
    }
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->tuned[key] = best;
  return best;
}

void batch_distance_index(dvg_context* ctx, uint32_t ngraphs, const dvg_matrix* const* graphs, const unsigned* dmin,
                          const unsigned* dmax, dvg_matrix** out) {
  for (uint32_t k = 0; k < ngraphs; ++k) out[k] = nullptr;
  // ---- validation and grouping -------------------------------------------------
  std::map<std::pair<unsigned, unsigned>, std::vector<uint32_t>> by_window;
  std::vector<uint32_t> alone;  // built one by one (non-canonical input with dmin = 0)
  for (uint32_t k = 0; k < ngraphs; ++k) {
    const dvg_matrix* a = graphs[k];
    require(a != nullptr, "batch: null graph");
    require(a->nrows == a->ncols, "batch: adjacency matrix is not square");
    require(dmin[k] <= dmax[k] && dmax[k] != 0, "batch: requires dmin <= dmax and dmax != 0");
    if ((dmin[k] == 0 && !a->canonical) || !ctx->opt_planned || ctx->opt_spgemm_mode == 1 ||
        ctx->opt_dindex_schedule != 0)
      alone.push_back(k);
    else
      by_window[{dmin[k], dmax[k]}].push_back(k);
  }
  std::vector<Group> groups;
  for (auto& kv : by_window) {
    // split a window's graphs into groups of at most 2^32 - 2 rows
    Group cur;
    unsigned long long rows = 0;
    for (uint32_t k : kv.second) {
      const uint32_t n = graphs[k]->nrows;
      if (!cur.members.empty() && rows + n > 0xFFFFFFFEull) {
        groups.push_back(std::move(cur));
        cur = Group{};
        rows = 0;
      }
      cur.dlo = kv.first.first;
      cur.dup = kv.first.second;
      cur.members.push_back(k);
      rows += n;
    }
    if (!cur.members.empty()) groups.push_back(std::move(cur));
  }
  if (groups.empty()) {
    try {
      for (uint32_t k : alone) out[k] = create_distance_index(ctx, graphs[k], dmin[k], dmax[k]);
    } catch (...) {
      for (uint32_t k = 0; k < ngraphs; ++k) {
        free_matrix(ctx, out[k]);
        out[k] = nullptr;
      }
      throw;
    }
    return;
  }
  auto cleanup = [&]() {
    for (auto& g : groups) {
      if (g.planned) release_build(ctx, g.pb);
      g.planned = false;
      free_matrix(ctx, g.g);
      free_matrix(ctx, g.t);
      g.g = g.t = nullptr;
    }
  };
  void* d_table = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  try {
    // ---- the block-diagonal inputs ---------------------------------------------
    size_t nslices = 0;
    for (auto& g : groups) {
      unsigned long long row = 0, ent = 0;
      bool canonical = true;
      for (uint32_t k : g.members) {
        g.slices.push_back(GraphSlice{graphs[k]->rowmap, graphs[k]->entries, row, ent});
        row += graphs[k]->nrows;
        ent += graphs[k]->nentries;
        canonical = canonical && graphs[k]->canonical;
      }
      g.slices.push_back(GraphSlice{nullptr, nullptr, row, ent});
      g.g = new_matrix(ctx, uint32_t(row), uint32_t(row), ent);
      g.g->canonical = canonical;
      g.table_off = nslices;
      nslices += g.slices.size();
    }
    const size_t table_bytes = std::max<size_t>(nslices, 1) * sizeof(GraphSlice);
    d_table = dalloc(ctx, table_bytes);
    {
      auto* h = static_cast<GraphSlice*>(host_stage(ctx, table_bytes));
      for (auto& g : groups) std::memcpy(h + g.table_off, g.slices.data(), g.slices.size() * sizeof(GraphSlice));
      DVG_CUDA(cudaMemcpyAsync(d_table, h, nslices * sizeof(GraphSlice), cudaMemcpyHostToDevice, ctx->stream));
      ctx->stats.h2d_bytes += nslices * sizeof(GraphSlice);
    }
    auto* table = static_cast<GraphSlice*>(d_table);
    auto assemble = [&](Group& g) {
      const uint32_t ng = uint32_t(g.members.size());
      const auto& tot = g.slices.back();
      k_assemble<<<grid_for(ctx, std::max(tot.row_off, tot.ent_off)), 256, 0, ctx->stream>>>(
          table + g.table_off, ng, g.g->rowmap, g.g->entries);
      DVG_CUDA(cudaGetLastError());
      ctx->stats.kernel_launches++;
    };
    // ---- kernel shapes: tuned on first sight of a (window, size class) -----------
    std::vector<TuneChoice> choice(groups.size(), TuneChoice{int(ctx->opt_row_slot), ctx->opt_chunk_rows});
    if (ctx->opt_autotune) {
      for (size_t i = 0; i < groups.size(); ++i) {
        const int size_class = 64 - __builtin_clzll(uint64_t(groups[i].g->nrows) | 1ull);
        if (!ctx->tuned.count(std::make_tuple(groups[i].dlo, groups[i].dup, size_class))) assemble(groups[i]);
        choice[i] = autotune_build(ctx, groups[i].g, groups[i].dlo, groups[i].dup);
      }
    }
    for (size_t i = 0; i < groups.size(); ++i) {
      Group& g = groups[i];
      g.pb = prepare_build(ctx, plan_index(g.dlo, g.dup), g.g, choice[i].slot_variant, choice[i].chunk_rows);
      g.planned = true;
    }
    // ---- one CUDA graph: every group's assembly and build ------------------------
    DVG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    try {
      for (auto& g : groups) {
        assemble(g);
        launch_build(ctx, g.pb, false);
      }
    } catch (...) {
      cudaGraph_t dropped = nullptr;
      cudaStreamEndCapture(ctx->stream, &dropped);
      if (dropped) cudaGraphDestroy(dropped);
      throw;
    }
    DVG_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
    DVG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    DVG_CUDA(cudaGraphLaunch(exec, ctx->stream));
    ctx->stats.graph_launches++;
    // ---- results ----------------------------------------------------------------
    for (auto& g : groups) {
      g.t = finish_build(ctx, g.pb);
      g.planned = false;
      if (!g.t) {  // a step outgrew its estimate: this group on the read-back path
        ctx->stats.spgemm_reruns++;
        g.t = create_distance_index(ctx, g.g, g.dlo, g.dup);
      }
      free_matrix(ctx, g.g);
      g.g = nullptr;
    }
    DVG_CUDA(cudaGraphExecDestroy(exec));
    exec = nullptr;
    DVG_CUDA(cudaGraphDestroy(graph));
    graph = nullptr;
    // where every graph's index starts in its group's, and its nnz: one
    // read-back for all
    {
      const size_t nb = std::max<size_t>(nslices, 1);
      auto* d_bounds = static_cast<unsigned long long*>(dalloc(ctx, 2 * nb * 8));
      unsigned long long* d_nnz = d_bounds + nb;
      DVG_CUDA(cudaMemsetAsync(d_nnz, 0, nb * 8, ctx->stream));
      for (auto& g : groups) {
        const uint32_t ng = uint32_t(g.members.size());
        k_bounds<<<grid_for(ctx, ng + 1), 256, 0, ctx->stream>>>(table + g.table_off, ng, g.t->rowmap,
                                                                 d_bounds + g.table_off);
        DVG_CUDA(cudaGetLastError());
        k_graph_nnz<<<grid_for(ctx, g.t->nentries / 64 + 1), 256, 0, ctx->stream>>>(
            d_bounds + g.table_off, ng, g.t->entries, d_nnz + g.table_off);
        DVG_CUDA(cudaGetLastError());
        ctx->stats.kernel_launches += 2;
      }
      auto* hb = static_cast<unsigned long long*>(host_stage(ctx, 2 * nb * 8));
      DVG_CUDA(cudaMemcpyAsync(hb, d_bounds, 2 * nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
      const uint64_t ts = now_ns();
      DVG_CUDA(cudaStreamSynchronize(ctx->stream));
      ctx->stats.host_sync_ns += now_ns() - ts;
      ctx->stats.host_syncs++;
      dfree(ctx, d_bounds);
      std::vector<unsigned long long> bounds(hb, hb + nslices), nnz(hb + nb, hb + nb + nslices);
      // the graphs' own matrices, and the table that cuts them out
      std::vector<OutSlice> outs(nslices);
      for (auto& g : groups) {
        const uint32_t ng = uint32_t(g.members.size());
        for (uint32_t j = 0; j < ng; ++j) {
          const uint32_t k = g.members[j];
          const uint64_t ne = bounds[g.table_off + j + 1] - bounds[g.table_off + j];
          dvg_matrix* m = new_matrix(ctx, graphs[k]->nrows, graphs[k]->ncols, ne);
          m->canonical = true;
          m->nnz = nnz[g.table_off + j];
          out[k] = m;
          outs[g.table_off + j] = OutSlice{m->rowmap, m->entries, g.slices[j].row_off, bounds[g.table_off + j]};
        }
        outs[g.table_off + ng] = OutSlice{nullptr, nullptr, g.slices[ng].row_off, bounds[g.table_off + ng]};
      }
      auto* ho = static_cast<OutSlice*>(host_stage(ctx, nslices * sizeof(OutSlice)));
      std::memcpy(ho, outs.data(), nslices * sizeof(OutSlice));
      auto* d_outs = static_cast<OutSlice*>(dalloc(ctx, std::max<size_t>(nslices, 1) * sizeof(OutSlice)));
      DVG_CUDA(cudaMemcpyAsync(d_outs, ho, nslices * sizeof(OutSlice), cudaMemcpyHostToDevice, ctx->stream));
      for (auto& g : groups) {
        const uint32_t ng = uint32_t(g.members.size());
        const auto& tot = outs[g.table_off + ng];
        k_split<<<grid_for(ctx, std::max(tot.row_off, tot.ent_off)), 256, 0, ctx->stream>>>(
            d_outs + g.table_off, ng, g.t->rowmap, g.t->entries);
        DVG_CUDA(cudaGetLastError());
        ctx->stats.kernel_launches++;
      }
      dfree(ctx, d_outs);
    }
    for (auto& g : groups) {
      free_matrix(ctx, g.t);
      g.t = nullptr;
    }
    dfree(ctx, d_table);
    d_table = nullptr;
    // graphs that could not join a group
    for (uint32_t k : alone) out[k] = create_distance_index(ctx, graphs[k], dmin[k], dmax[k]);
  } catch (...) {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cleanup();
    if (d_table) dfree(ctx, d_table);
    for (uint32_t k = 0; k < ngraphs; ++k) {
      free_matrix(ctx, out[k]);
      out[k] = nullptr;
    }
    throw;
  }
}

}  // namespace dvg
