// dvg_adjacency.cu -- the adjacency matrix of a sequence graph, built on the
// device in range CRS.
//
// Same result as util::range_adjacency_matrix (include/diverg/adjacency.hpp:
// 249-265 in cartoonist/diverg), which builds the Basic adjacency
// (adjacency_matrix, :170-228) and converts it with crs_matrix::append
// (crs_matrix.hpp:197-242):
//   * one row and one column per base (locus); the loci of node ids
//     lower .. upper-1 are numbered in rank order from 0 (id_to_charorder
//     minus that of `lower`);
//   * every locus but a node's last links to the next locus;
//   * a node's last locus links to the first locus of each successor, the
//     columns sorted; the Basic row becomes ranges by extending the open
//     range only with the column right after its end (col == end + 1), so a
//     repeated successor yields a repeated single-column range, as in append.
// nnz is the number of Basic entries, (loci - nodes) + edges.
//
// Kernels: edges are counted per source node and scattered into per-node
// segments (counting sort, any edge order), each node sorts its segment and
// counts its ranges, a scan gives every node's first entry, then one thread
// per locus writes the row map and the inner rows and one thread per node
// writes its last row.  All of it is streaming integer work on HBM.
#include <algorithm>
#include <vector>

#include "dvg_device.cuh"
#include "dvg_internal.h"

namespace dvg {
namespace {

constexpr int kAdjThreads = 256;

unsigned adj_grid(dvg_context* ctx, uint64_t n) {
  const uint64_t want = (n + kAdjThreads - 1) / kAdjThreads;
  const uint64_t cap = uint64_t(ctx->num_sms) * 16;
  return unsigned(std::max<uint64_t>(1, std::min(want, cap)));
}

struct AdjArgs {
  uint32_t nnodes;            // nodes of the range
  uint32_t lower, upper;      // node ids [lower, upper), 1-based
  uint64_t nedges;            // edges of the whole graph
  const uint32_t* node_len;   // [nnodes]
  const uint32_t* edges;      // [2 nedges]: (from_id, to_id)
  uint64_t* start;            // [nnodes + 1]: first locus of each node
  uint64_t* eoff;             // [nnodes + 1]: first edge slot of each node
  uint64_t* cursor;           // [nnodes]: scatter cursors
  uint32_t* cols;             // [edges of the range]: successor loci
  uint64_t* base;             // [nnodes + 1]: first entry of each node's rows
  uint64_t* c_rowmap;
  uint32_t* c_entries;
  DeviceControl* ctl;
};

// start[v + 1] = node_len[v] (scanned afterwards)
__global__ void k_adj_lengths(AdjArgs p) {
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < p.nnodes; v += uint64_t(gridDim.x) * blockDim.x)
    p.start[v + 1] = p.node_len[v];
}

// eoff[v + 1] = out-degree of node v within the range; a successor outside
// the range is an error (its column would not exist)
__global__ void k_adj_degrees(AdjArgs p) {
  for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < p.nedges; e += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t from = p.edges[2 * e], to = p.edges[2 * e + 1];
    if (from < p.lower || from >= p.upper) continue;
    if (to < p.lower || to >= p.upper) {
      atomicOr(&p.ctl->invalid, 1ull);
      continue;
    }
    atomicAdd(reinterpret_cast<unsigned long long*>(p.eoff + (from - p.lower) + 1), 1ull);
  }
}

// each edge's successor locus into its source node's segment
__global__ void k_adj_scatter(AdjArgs p) {
  for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < p.nedges; e += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t from = p.edges[2 * e], to = p.edges[2 * e + 1];
    if (from < p.lower || from >= p.upper || to < p.lower || to >= p.upper) continue;
    const uint32_t v = from - p.lower;
    const uint64_t slot = atomicAdd(reinterpret_cast<unsigned long long*>(p.cursor + v), 1ull);
    p.cols[p.eoff[v] + slot] = uint32_t(p.start[to - p.lower]);
  }
}

// Sorts a[0..n) ascending: insertion sort for short segments, heap sort
// (no scratch, n log n) for long ones.
__device__ void sort_segment(uint32_t* a, uint64_t n) {
  if (n <= 32) {
    for (uint64_t i = 1; i < n; ++i) {
      const uint32_t x = a[i];
      uint64_t j = i;
      while (j > 0 && a[j - 1] > x) {
        a[j] = a[j - 1];
        --j;
      }
      a[j] = x;
    }
    return;
  }
  auto sift = [&](uint64_t root, uint64_t end) {
    for (;;) {
      uint64_t child = 2 * root + 1;
      if (child >= end) return;
      if (child + 1 < end && a[child + 1] > a[child]) ++child;
      if (a[root] >= a[child]) return;
      const uint32_t t = a[root];
      a[root] = a[child];
      a[child] = t;
      root = child;
    }
  };
  for (uint64_t i = n / 2; i-- > 0;) sift(i, n);
  for (uint64_t end = n; end > 1; --end) {
    const uint32_t t = a[0];
    a[0] = a[end - 1];
    a[end - 1] = t;
    sift(0, end - 1);
  }
}

// Ranges of a sorted Basic row under append's rule: a column extends the
// open range only when it is the column right after the range's end.
__device__ __forceinline__ uint64_t row_ranges(const uint32_t* a, uint64_t n, bool& repeated) {
  uint64_t r = 0;
  uint32_t end = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (r && uint64_t(a[i]) == uint64_t(end) + 1) {
      ++end;
      continue;
    }
    if (r && a[i] <= end) repeated = true;
    ++r;
    end = a[i];
  }
  return r;
}

// per node: sort its successor loci, base[v + 1] = the entries of its rows
__global__ void k_adj_nodes(AdjArgs p) {
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < p.nnodes; v += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t* a = p.cols + p.eoff[v];
    const uint64_t n = p.eoff[v + 1] - p.eoff[v];
    sort_segment(a, n);
    bool repeated = false;
    const uint64_t r = row_ranges(a, n, repeated);
    if (repeated) atomicOr(&p.ctl->invalid, 16ull);
    p.base[v + 1] = 2 * (uint64_t(p.node_len[v]) - 1) + 2 * r;
  }
}

// per locus: the row map, and the single range of every row but a node's last
__global__ void k_adj_rows(AdjArgs p, uint64_t nloci) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < nloci; i += uint64_t(gridDim.x) * blockDim.x) {
    // the node holding locus i: the last v with start[v] <= i
    uint32_t lo = 0, hi = p.nnodes;  // start[lo] <= i < start[hi]
    while (hi - lo > 1) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if (p.start[mid] <= i) lo = mid;
      else hi = mid;
    }
    const uint64_t k = i - p.start[lo];
    const uint64_t len = p.node_len[lo];
    if (k + 1 < len) {
      const uint64_t at = p.base[lo] + 2 * k;
      p.c_entries[at] = uint32_t(i + 1);
      p.c_entries[at + 1] = uint32_t(i + 1);
      p.c_rowmap[i + 1] = at + 2;
    } else {
      p.c_rowmap[i + 1] = p.base[lo + 1];
    }
    if (i == 0) p.c_rowmap[0] = 0;
  }
}

// per node: the ranges of its last row
__global__ void k_adj_last_rows(AdjArgs p) {
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < p.nnodes; v += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t* a = p.cols + p.eoff[v];
    const uint64_t n = p.eoff[v + 1] - p.eoff[v];
    uint32_t* out = p.c_entries + p.base[v] + 2 * (uint64_t(p.node_len[v]) - 1);
    const uint32_t* stop = p.c_entries + p.base[v + 1];
    uint64_t w = 0;
    auto put = [&](uint32_t x) {
      if (out + w < stop) out[w] = x;
      ++w;
    };
    bool open = false;
    uint32_t end = 0;
    for (uint64_t i = 0; i < n; ++i) {
      if (open && uint64_t(a[i]) == uint64_t(end) + 1) {
        ++end;
        continue;
      }
      if (open) put(end);
      put(a[i]);
      end = a[i];
      open = true;
    }
    if (open) put(end);
    if (out + w != stop) atomicOr(&p.ctl->status, 32ull);
  }
}

}  // namespace

dvg_matrix* adjacency_from_graph(dvg_context* ctx, uint32_t nnodes, const uint32_t* node_len, uint64_t nedges,
                                 const uint32_t* edges, uint32_t lower, uint32_t upper) {
  if (upper == 0) upper = nnodes + 1;
  if (nnodes == 0 || lower < 1 || lower > nnodes || upper <= lower || upper > nnodes + 1)
    throw Error(DVG_ERR_INVALID_ARG, "adjacency: node range must satisfy 1 <= lower < upper <= nnodes + 1");
  if (!node_len || (nedges && !edges)) throw Error(DVG_ERR_INVALID_ARG, "adjacency: null argument");
  const uint32_t m = upper - lower;
  const uint32_t* lens = node_len + (lower - 1);
  uint64_t nloci = 0;
  for (uint32_t v = 0; v < m; ++v) {
    if (lens[v] == 0) throw Error(DVG_ERR_INVALID_ARG, "adjacency: a node has length 0");
    nloci += lens[v];
  }
  if (nloci > 0xFFFFFFFEull) throw Error(DVG_ERR_OVERFLOW, "adjacency: more loci than 32-bit columns hold");

  AdjArgs p{};
  p.nnodes = m;
  p.lower = lower;
  p.upper = upper;
  p.nedges = nedges;
  p.ctl = ctx->d_ctl;
  std::vector<void*> scratch;
  auto grab = [&](size_t bytes) {
    void* q = dalloc(ctx, bytes);
    scratch.push_back(q);
    return q;
  };
  dvg_matrix* out = nullptr;
  try {
    uint32_t* d_len = static_cast<uint32_t*>(grab(size_t(m) * 4));
    uint32_t* d_edges = nedges ? static_cast<uint32_t*>(grab(nedges * 8)) : nullptr;
    p.start = static_cast<uint64_t*>(grab((size_t(m) + 1) * 8));
    p.eoff = static_cast<uint64_t*>(grab((size_t(m) + 1) * 8));
    p.cursor = static_cast<uint64_t*>(grab(size_t(m) * 8));
    p.base = static_cast<uint64_t*>(grab((size_t(m) + 1) * 8));
    DVG_CUDA(cudaMemcpyAsync(d_len, lens, size_t(m) * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (nedges) DVG_CUDA(cudaMemcpyAsync(d_edges, edges, nedges * 8, cudaMemcpyHostToDevice, ctx->stream));
    ctx->stats.h2d_bytes += uint64_t(m) * 4 + nedges * 8;
    p.node_len = d_len;
    p.edges = d_edges;
    reset_control(ctx);
    DVG_CUDA(cudaMemsetAsync(p.start, 0, 8, ctx->stream));
    DVG_CUDA(cudaMemsetAsync(p.eoff, 0, (size_t(m) + 1) * 8, ctx->stream));
    DVG_CUDA(cudaMemsetAsync(p.cursor, 0, size_t(m) * 8, ctx->stream));
    DVG_CUDA(cudaMemsetAsync(p.base, 0, 8, ctx->stream));
    k_adj_lengths<<<adj_grid(ctx, m), kAdjThreads, 0, ctx->stream>>>(p);
    DVG_CUDA(cudaGetLastError());
    if (nedges) {
      k_adj_degrees<<<adj_grid(ctx, nedges), kAdjThreads, 0, ctx->stream>>>(p);
      DVG_CUDA(cudaGetLastError());
    }
    launch_rowmap_scan(ctx, p.start, m);
    launch_rowmap_scan(ctx, p.eoff, m);
    // the range's edges: one read-back sizes the segment array
    uint64_t nedges_in = 0;
    DVG_CUDA(cudaMemcpyAsync(&ctx->h_ctl[1], p.eoff + m, 8, cudaMemcpyDeviceToHost, ctx->stream));
    {
      const DeviceControl c = read_control(ctx);
      nedges_in = *reinterpret_cast<const uint64_t*>(&ctx->h_ctl[1]);
      if (c.invalid & 1) throw Error(DVG_ERR_INVALID_ARG, "adjacency: an edge leaves the node range [lower, upper)");
    }
    p.cols = static_cast<uint32_t*>(grab(std::max<uint64_t>(nedges_in, 1) * 4));
    if (nedges) {
      k_adj_scatter<<<adj_grid(ctx, nedges), kAdjThreads, 0, ctx->stream>>>(p);
      DVG_CUDA(cudaGetLastError());
    }
    k_adj_nodes<<<adj_grid(ctx, m), kAdjThreads, 0, ctx->stream>>>(p);
    DVG_CUDA(cudaGetLastError());
    launch_rowmap_scan(ctx, p.base, m);
    DVG_CUDA(cudaMemcpyAsync(&ctx->h_ctl[1], p.base + m, 8, cudaMemcpyDeviceToHost, ctx->stream));
    const DeviceControl c = read_control(ctx);
    const uint64_t nentries = *reinterpret_cast<const uint64_t*>(&ctx->h_ctl[1]);
    out = new_matrix(ctx, uint32_t(nloci), uint32_t(nloci), nentries);
    out->canonical = !(c.invalid & 16);
    out->nnz = (nloci - m) + nedges_in;
    p.c_rowmap = out->rowmap;
    p.c_entries = out->entries;
    k_adj_rows<<<adj_grid(ctx, nloci), kAdjThreads, 0, ctx->stream>>>(p, nloci);
    DVG_CUDA(cudaGetLastError());
    k_adj_last_rows<<<adj_grid(ctx, m), kAdjThreads, 0, ctx->stream>>>(p);
    DVG_CUDA(cudaGetLastError());
    ctx->stats.kernel_launches += 5 + (nedges ? 2 : 0);
    const DeviceControl done = read_control(ctx);
    if (done.status) throw Error(DVG_ERR_DEVICE, "adjacency: internal consistency check failed on the device");
  } catch (...) {
    for (void* q : scratch) dfree(ctx, q);
    if (out) free_matrix(ctx, out);
    throw;
  }
  for (void* q : scratch) dfree(ctx, q);
  return out;
}

}  // namespace dvg
