/*
 * oracle.cpp -- CPU restatement of DiVerG's range-CRS algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the timed
 * CPU baseline ("port" of the reference's host path).  It is never linked into
 * or called by the product library; only tests/, the smoke check and the CPU
 * baseline leg of bench.py load it.
 *
 * Every function restates one routine of the reference (cartoonist/diverg
 * v1.1.1); the citation next to each one names the file:line it follows.
 * The reference itself cannot be compiled here (its Kokkos, KokkosKernels,
 * gum and sdsl submodules are absent), so parity of this restatement is
 * pinned by the reference's own known-answer vectors
 * (test/src/test_hbitvector.cpp:186-234 -> :618-661) and by dense Boolean
 * brute force on the reference's GFA fixtures (see tests/).
 *
 * Matrix layout (range CRS, identical to CRSMatrix<RangeDynamic,bool,uint32_t,
 * uint64_t>, include/diverg/crs_matrix.hpp:1873-2004):
 *   rowmap  : uint64[nrows+1], counts ENTRIES (2 per range)
 *   entries : uint32[rowmap[nrows]], flattened inclusive [start,end] pairs,
 *             sorted, disjoint and non-adjacent within a row
 *   nnz     : sum of (end - start + 1)
 */
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>
#include <omp.h>

extern "C" {

typedef struct orc_mat {
  uint32_t nrows;
  uint32_t ncols;
  uint64_t nentries;
  uint64_t nnz;
  uint64_t* rowmap;   /* nrows + 1 */
  uint32_t* entries;  /* nentries */
} orc_mat;

orc_mat* orc_adjacency_range(uint32_t nnodes, const uint32_t* node_len, uint64_t nedges, const uint32_t* edges,
                             uint32_t lower, uint32_t upper);

}  // extern "C"

namespace {

struct Mat {
  uint32_t nrows = 0, ncols = 0;
  uint64_t nnz = 0;
  std::vector<uint64_t> rowmap;
  std::vector<uint32_t> entries;
};

Mat from_c(const orc_mat* m) {
  Mat r;
  r.nrows = m->nrows;
  r.ncols = m->ncols;
  r.nnz = m->nnz;
  r.rowmap.assign(m->rowmap, m->rowmap + m->nrows + 1);
  r.entries.assign(m->entries, m->entries + m->nentries);
  return r;
}

orc_mat* to_c(const Mat& m) {
  orc_mat* r = (orc_mat*)std::calloc(1, sizeof(orc_mat));
  r->nrows = m.nrows;
  r->ncols = m.ncols;
  r->nentries = m.entries.size();
  r->nnz = m.nnz;
  r->rowmap = (uint64_t*)std::malloc(sizeof(uint64_t) * (m.rowmap.size() ? m.rowmap.size() : 1));
  r->entries = (uint32_t*)std::malloc(sizeof(uint32_t) * (m.entries.size() ? m.entries.size() : 1));
  if (!m.rowmap.empty()) std::memcpy(r->rowmap, m.rowmap.data(), sizeof(uint64_t) * m.rowmap.size());
  if (!m.entries.empty()) std::memcpy(r->entries, m.entries.data(), sizeof(uint32_t) * m.entries.size());
  return r;
}

/* crs_matrix::nnz(..., RangeGroup), crs_matrix.hpp:175-189 */
uint64_t range_nnz(const std::vector<uint32_t>& e) {
  uint64_t c = 0;
  for (size_t i = 0; i + 1 < e.size(); i += 2) c += uint64_t(e[i + 1]) - e[i] + 1;
  return c;
}

/* create_range_identity_matrix, range_sparse.hpp:66-88 (entries [i,i],
 * rowmap 2(i+1)); nnz = n as in range_sparse.hpp:95-110. */
Mat identity(uint32_t n) {
  Mat r;
  r.nrows = r.ncols = n;
  r.rowmap.resize(size_t(n) + 1);
  r.entries.resize(size_t(n) * 2);
  r.rowmap[0] = 0;
  for (uint32_t i = 0; i < n; ++i) {
    r.entries[2 * size_t(i)] = i;
    r.entries[2 * size_t(i) + 1] = i;
    r.rowmap[i + 1] = 2 * (uint64_t(i) + 1);
  }
  r.nnz = n;
  return r;
}

/* Row merge of range_spadd_numeric, range_sparse.hpp:273-356: both rows are
 * walked in order of range start (ties taken from `a`), a range whose start
 * is <= hi+1 is merged into the open one, otherwise the open one is emitted.
 * After one list runs out the other is merged until its first non-merging
 * range, and the rest of it is copied verbatim. */
template <class Emit>
void spadd_row(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb, Emit emit) {
  uint64_t ai = 0, bi = 0;
  if (ai < na && bi < nb) {
    uint32_t lo, hi;
    if (a[ai] <= b[bi]) { lo = a[ai]; hi = a[ai + 1]; ai += 2; }
    else { lo = b[bi]; hi = b[bi + 1]; bi += 2; }
    while (ai < na && bi < nb) {
      uint32_t rs, re;
      if (a[ai] <= b[bi]) { rs = a[ai]; re = a[ai + 1]; ai += 2; }
      else { rs = b[bi]; re = b[bi + 1]; bi += 2; }
      if (uint64_t(rs) <= uint64_t(hi) + 1) { lo = std::min(lo, rs); hi = std::max(hi, re); continue; }
      emit(lo); emit(hi);
      lo = rs; hi = re;
    }
    while (ai < na || bi < nb) {
      uint32_t rs, re;
      if (ai == na) { rs = b[bi]; re = b[bi + 1]; bi += 2; }
      else { rs = a[ai]; re = a[ai + 1]; ai += 2; }
      if (uint64_t(rs) <= uint64_t(hi) + 1) { lo = std::min(lo, rs); hi = std::max(hi, re); continue; }
      emit(lo); emit(hi);
      lo = rs; hi = re;
      break;
    }
    emit(lo); emit(hi);
  }
  for (; ai < na; ++ai) emit(a[ai]);
  for (; bi < nb; ++bi) emit(b[bi]);
}

/* range_spadd (range_sparse.hpp:364-428) + RangeSpAdd::spadd nnz
 * (range_sparse.hpp:438-468: nnz recounted from the entries). */
Mat spadd(const Mat& A, const Mat& B) {
  Mat C;
  C.nrows = A.nrows;
  C.ncols = A.ncols;
  C.rowmap.resize(size_t(A.nrows) + 1);
  C.rowmap[0] = 0;
  C.entries.reserve(A.entries.size() + B.entries.size());
  for (uint32_t r = 0; r < A.nrows; ++r) {
    spadd_row(A.entries.data() + A.rowmap[r], A.rowmap[r + 1] - A.rowmap[r],
              B.entries.data() + B.rowmap[r], B.rowmap[r + 1] - B.rowmap[r],
              [&](uint32_t v) { C.entries.push_back(v); });
    C.rowmap[r + 1] = C.entries.size();
  }
  C.nnz = range_nnz(C.entries);
  return C;
}

/* BTree accumulator SpGEMM, range_sparse.hpp:527-572 (symbolic) and
 * :638-677 (numeric): for every range [s,f] of A's row, all B ranges of B rows
 * s..f (contiguous in B.entries) are inserted as start -> max(end) into an
 * ordered map, which is then swept merging while start <= hi+1.  The returned
 * nnz is the symbolic phase's sum of run lengths. */
Mat spgemm_btree(const Mat& A, const Mat& B, int nthreads) {
  Mat C;
  C.nrows = A.nrows;
  C.ncols = B.ncols;
  std::vector<std::vector<uint32_t>> rows(A.nrows);
  uint64_t nnz = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads) reduction(+ : nnz)
  for (int64_t row = 0; row < int64_t(A.nrows); ++row) {
    std::map<uint32_t, uint32_t> acc;
    for (uint64_t ai = A.rowmap[row]; ai < A.rowmap[row + 1]; ai += 2) {
      uint64_t bi = B.rowmap[A.entries[ai]];
      uint64_t be = B.rowmap[uint64_t(A.entries[ai + 1]) + 1];
      for (; bi < be; bi += 2) {
        auto& slot = acc[B.entries[bi]];
        slot = std::max(slot, B.entries[bi + 1]);
      }
    }
    auto& out = rows[row];
    if (!acc.empty()) {
      auto it = acc.begin();
      uint32_t lo = it->first, hi = it->second;
      for (++it; it != acc.end(); ++it) {
        if (uint64_t(it->first) <= uint64_t(hi) + 1) { lo = std::min(lo, it->first); hi = std::max(hi, it->second); continue; }
        out.push_back(lo); out.push_back(hi);
        nnz += uint64_t(hi) - lo + 1;
        lo = it->first; hi = it->second;
      }
      out.push_back(lo); out.push_back(hi);
      nnz += uint64_t(hi) - lo + 1;
    }
  }
  C.rowmap.resize(size_t(A.nrows) + 1);
  C.rowmap[0] = 0;
  for (uint32_t r = 0; r < A.nrows; ++r) C.rowmap[r + 1] = C.rowmap[r] + rows[r].size();
  C.entries.resize(C.rowmap[A.nrows]);
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t r = 0; r < int64_t(A.nrows); ++r)
    if (!rows[r].empty()) std::memcpy(C.entries.data() + C.rowmap[r], rows[r].data(), 4 * rows[r].size());
  C.nnz = nnz;
  return C;
}

/* Bitvector accumulator SpGEMM on the host: the reference's HBitVector
 * TeamSequential algorithm (range_sparse.hpp:1184-1264 symbolic, :1340-1441
 * numeric) with 64-bit bitsets as on its host backends (hbitvector.hpp:35-39).
 * Each thread owns one full-width bitvector (the reference splits it into an
 * L1 window in scratch memory and an L2 remainder; the split is a placement
 * detail with no effect on the result).  Per row: every B range of every B row
 * named by an A range is set bit-range-wise (hbitvector.hpp:1155-1233), then
 * the touched words are gathered with map01/map10 boundary masks carrying the
 * previous word's msb (hbitvector.hpp:568-597), and a run that is still open
 * after the last word is closed at that word's end (range_sparse.hpp:1435-1440).
 * Symbolic and numeric are fused here: the host has no reason to recompute.
 * This is the timed CPU baseline. */
Mat spgemm_hbv(const Mat& A, const Mat& B, int nthreads) {
  Mat C;
  C.nrows = A.nrows;
  C.ncols = B.ncols;
  const uint64_t nwords = (uint64_t(B.ncols) + 63) / 64 + 1;
  std::vector<uint64_t> counts(size_t(A.nrows) + 1, 0);
  std::vector<std::vector<uint32_t>> rows(A.nrows);
  uint64_t nnz = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : nnz)
  {
    std::vector<uint64_t> bv(nwords, 0);
#pragma omp for schedule(dynamic, 256)
    for (int64_t row = 0; row < int64_t(A.nrows); ++row) {
      uint64_t wmin = UINT64_MAX, wmax = 0;
      for (uint64_t ai = A.rowmap[row]; ai < A.rowmap[row + 1]; ai += 2) {
        uint64_t bi = B.rowmap[A.entries[ai]];
        uint64_t be = B.rowmap[uint64_t(A.entries[ai + 1]) + 1];
        for (; bi < be; bi += 2) {
          uint64_t s = B.entries[bi], f = B.entries[bi + 1];
          uint64_t ws = s >> 6, wf = f >> 6;
          wmin = std::min(wmin, ws);
          wmax = std::max(wmax, wf);
          uint64_t lo_mask = ~uint64_t(0) << (s & 63);
          uint64_t hi_mask = ~uint64_t(0) >> (63 - (f & 63));
          if (ws == wf) { bv[ws] |= lo_mask & hi_mask; continue; }
          bv[ws] |= lo_mask;
          for (uint64_t w = ws + 1; w < wf; ++w) bv[w] = ~uint64_t(0);
          bv[wf] |= hi_mask;
        }
      }
      auto& out = rows[row];
      if (wmin == UINT64_MAX) continue;
      uint64_t c = 0;
      for (uint64_t w = wmin; w <= wmax; ++w) {
        uint64_t x = bv[w];
        uint64_t prev = (x << 1) | c;
        uint64_t map01 = (x ^ prev) & x;   /* run starts  */
        uint64_t map10 = prev & ~x;        /* run ends + 1 */
        uint64_t bounds = map01 | map10;
        nnz += __builtin_popcountll(x);
        while (bounds) {
          int k = __builtin_ctzll(bounds);
          bounds &= bounds - 1;
          uint32_t pos = uint32_t(w * 64 + k);
          out.push_back((out.size() & 1) ? pos - 1 : pos);
        }
        c = x >> 63;
        bv[w] = 0;
      }
      if (c) out.push_back(uint32_t((wmax + 1) * 64 - 1));
      counts[row + 1] = out.size();
    }
  }
  C.rowmap.resize(size_t(A.nrows) + 1);
  C.rowmap[0] = 0;
  for (uint32_t r = 0; r < A.nrows; ++r) C.rowmap[r + 1] = C.rowmap[r] + counts[r + 1];
  C.entries.resize(C.rowmap[A.nrows]);
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t r = 0; r < int64_t(A.nrows); ++r)
    if (!rows[r].empty()) std::memcpy(C.entries.data() + C.rowmap[r], rows[r].data(), 4 * rows[r].size());
  C.nnz = nnz;
  return C;
}

Mat spgemm(const Mat& A, const Mat& B, int algo, int nthreads) {
  return algo == 1 ? spgemm_hbv(A, B, nthreads) : spgemm_btree(A, B, nthreads);
}

/* range_power_inplace, range_sparse.hpp:2370-2431: C starts as I (nnz =
 * ncols); for every bit of k from the lowest, C <- C*A if the bit is set,
 * then A <- A*A while bits remain.  Returns C with the last product's nnz. */
Mat power(Mat A, unsigned k, int algo, int nthreads) {
  Mat C = identity(A.ncols);
  while (true) {
    if (k & 1) C = spgemm(C, A, algo, nthreads);
    k >>= 1;
    if (k != 0) A = spgemm(A, A, algo, nthreads);
    else break;
  }
  return C;
}

}  // namespace

extern "C" {

void orc_mat_free(orc_mat* m) {
  if (!m) return;
  std::free(m->rowmap);
  std::free(m->entries);
  std::free(m);
}

orc_mat* orc_identity(uint32_t n) { return to_c(identity(n)); }

orc_mat* orc_spadd(const orc_mat* a, const orc_mat* b) { return to_c(spadd(from_c(a), from_c(b))); }

/* algo: 0 = BTree (the semantic oracle), 1 = bitvector (the CPU baseline) */
orc_mat* orc_spgemm(const orc_mat* a, const orc_mat* b, int algo, int nthreads) {
  return to_c(spgemm(from_c(a), from_c(b), algo, nthreads));
}

orc_mat* orc_power(const orc_mat* a, unsigned k, int algo, int nthreads) {
  return to_c(power(from_c(a), k, algo, nthreads));
}

/* util::create_distance_index, dindex.hpp:46-189:
 *   rai = I + A                       (dindex.hpp:122-137)
 *   rad = A^dlo        if dlo != 0    (dindex.hpp:151-157)
 *   raid = rai^(dup-dlo)              (dindex.hpp:160-164)
 *   d = rad * raid     if dlo != 0, else raid   (dindex.hpp:167-177)
 * Requires dlo <= dup and dup != 0 (dindex.hpp:66); returns NULL otherwise. */
orc_mat* orc_dindex(const orc_mat* a, unsigned dlo, unsigned dup, int algo, int nthreads) {
  if (!(dlo <= dup && dup != 0)) return nullptr;
  Mat A = from_c(a);
  Mat rai = spadd(identity(A.nrows), A);
  Mat d;
  if (dlo != 0) {
    Mat rad = power(A, dlo, algo, nthreads);
    Mat raid = power(rai, dup - dlo, algo, nthreads);
    d = spgemm(rad, raid, algo, nthreads);
  } else {
    d = power(rai, dup - dlo, algo, nthreads);
  }
  return to_c(d);
}

/* CRSMatrixBase::operator()(i,j), crs_matrix.hpp:1197-1218, through
 * crs_matrix::binary_search(..., RangeGroup), crs_matrix.hpp:149-169:
 * lower_bound of j in the row's flattened [s0,e0,s1,e1,...]; an odd landing
 * index steps back to that range's start; the answer is first != end &&
 * *first <= j.  pairs = [i0, j0, i1, j1, ...]; out[q] = 0/1. */
void orc_query(const orc_mat* m, const uint32_t* pairs, uint64_t npairs, uint8_t* out) {
  for (uint64_t q = 0; q < npairs; ++q) {
    uint32_t i = pairs[2 * q], j = pairs[2 * q + 1];
    const uint32_t* begin = m->entries + m->rowmap[i];
    const uint32_t* end = m->entries + m->rowmap[i + 1];
    const uint32_t* first = begin;
    int64_t len = end - first;
    while (len > 0) {
      int64_t half = len / 2;
      const uint32_t* middle = first + half;
      if (*middle < j) { first = middle + 1; len = len - half - 1; }
      else len = half;
    }
    if ((first - begin) % 2) --first;
    out[q] = (first != end && *first <= j) ? 1 : 0;
  }
}

/* crs_matrix::append(..., RangeGroup to, BasicGroup from), crs_matrix.hpp:
 * 197-242: per row, consecutive columns (col == pending_end + 1) extend the open
 * range, any other column closes it and opens a new one.  The nnz is the
 * Basic matrix's nnz (crs_matrix.hpp:1910-1914). */
orc_mat* orc_basic_to_range(uint32_t nrows, uint32_t ncols, const uint64_t* rowmap, const uint32_t* cols) {
  Mat r;
  r.nrows = nrows;
  r.ncols = ncols;
  r.rowmap.resize(size_t(nrows) + 1);
  r.rowmap[0] = 0;
  for (uint32_t row = 0; row < nrows; ++row) {
    bool pending = false;
    uint32_t pend = 0;
    for (uint64_t k = rowmap[row]; k < rowmap[row + 1]; ++k) {
      uint32_t col = cols[k];
      if (pending && uint64_t(col) == uint64_t(pend) + 1) { ++pend; continue; }
      if (pending) r.entries.push_back(pend);
      r.entries.push_back(col);
      pend = col;
      pending = true;
    }
    if (pending) r.entries.push_back(pend);
    r.rowmap[row + 1] = r.entries.size();
  }
  r.nnz = rowmap[nrows];
  return to_c(r);
}

/* util::adjacency_matrix, adjacency.hpp:170-228, for a graph whose nodes are
 * given in rank order with contiguous ids 1..nnodes (so id_to_charorder(id) is
 * the sum of the lengths of nodes 1..id-1, with the first node at locus 0):
 * within a node each locus links to the next one; the node's last locus links
 * to the first locus of every successor, columns sorted per row.  The Basic
 * matrix is then converted to range CRS (adjacency.hpp:249-265).
 * edges are (src_id, dst_id) pairs, ids 1-based. */
orc_mat* orc_adjacency(uint32_t nnodes, const uint32_t* node_len, uint64_t nedges, const uint32_t* edges) {
  return orc_adjacency_range(nnodes, node_len, nedges, edges, 1, 0);
}

/* The same for the nodes lower .. upper-1 (upper = 0: through the last node),
 * as adjacency_matrix(graph, lower, upper): loci numbered from the first
 * locus of node `lower` (id_to_charorder(to) - start, adjacency.hpp:205,220),
 * only the edges out of nodes in the range (for_each_node from `lower`,
 * stopping after rank upper-1, :209-226). */
orc_mat* orc_adjacency_range(uint32_t nnodes, const uint32_t* node_len, uint64_t nedges, const uint32_t* edges,
                             uint32_t lower, uint32_t upper) {
  if (upper == 0) upper = nnodes + 1;
  std::vector<uint64_t> charorder(size_t(nnodes) + 2, 0);
  for (uint32_t id = 1; id <= nnodes; ++id) charorder[id + 1] = charorder[id] + node_len[id - 1];
  std::vector<std::vector<uint32_t>> succ(size_t(nnodes) + 1);
  for (uint64_t e = 0; e < nedges; ++e) succ[edges[2 * e]].push_back(edges[2 * e + 1]);
  const uint64_t start = charorder[lower];
  const uint64_t nloci = charorder[upper] - start;
  std::vector<uint64_t> rowmap;
  std::vector<uint32_t> cols;
  rowmap.reserve(nloci + 1);
  rowmap.push_back(0);
  uint64_t cursor = 0;
  for (uint32_t id = lower; id < upper; ++id) {
    for (uint32_t off = 1; off < node_len[id - 1]; ++off) {
      cols.push_back(uint32_t(++cursor));
      rowmap.push_back(cols.size());
    }
    ++cursor;
    size_t row_begin = cols.size();
    for (uint32_t to : succ[id]) cols.push_back(uint32_t(charorder[to] - start));
    std::sort(cols.begin() + row_begin, cols.end());
    rowmap.push_back(cols.size());
  }
  return orc_basic_to_range(uint32_t(nloci), uint32_t(nloci), rowmap.data(), cols.data());
}

uint64_t orc_nnz(const orc_mat* m) {
  uint64_t c = 0;
  for (uint64_t i = 0; i + 1 < m->nentries; i += 2) c += uint64_t(m->entries[i + 1]) - m->entries[i] + 1;
  return c;
}

int orc_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
