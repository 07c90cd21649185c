// Exercises the C++ headers include/diverg/*.hpp (the reference's API over
// libdvg.so) against the CPU oracle, in the manner of the reference's
// test/src/test_dindex.cpp:177-234 (the compiled ETI entry point equals the
// templated one) and test_range_sparse.cpp (products equal an independent
// implementation).  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <sstream>
#include <stdexcept>
#include <vector>

#include <diverg/adjacency.hpp>
#include <diverg/dindex_eti.hpp>
#include <dvg_gen.h>

extern "C" {
typedef struct orc_mat {
  uint32_t nrows, ncols;
  uint64_t nentries, nnz;
  uint64_t* rowmap;
  uint32_t* entries;
} orc_mat;
orc_mat* orc_dindex(const orc_mat* a, unsigned dlo, unsigned dup, int algo, int nthreads);
orc_mat* orc_spgemm(const orc_mat* a, const orc_mat* b, int algo, int nthreads);
orc_mat* orc_spadd(const orc_mat* a, const orc_mat* b);
orc_mat* orc_power(const orc_mat* a, unsigned k, int algo, int nthreads);
orc_mat* orc_identity(uint32_t n);
void orc_mat_free(orc_mat* m);
}

using RCRS = diverg::CRSMatrix<diverg::crs_matrix::RangeDynamic, bool, uint32_t, uint64_t>;
using RCRS32 = diverg::CRSMatrix<diverg::crs_matrix::RangeDynamic, bool, uint32_t, uint32_t>;

// The part of gum's SeqGraph interface util::range_adjacency_matrix walks
// (adjacency.hpp:170-228), over a node list; ids differ from ranks
// (id = 3 rank + 7) so the rank conversion is exercised.
struct NodeGraph {
  typedef uint64_t id_type;
  typedef uint64_t rank_type;
  typedef int linktype_type;
  std::vector<uint32_t> len;                // by rank - 1
  std::vector<std::vector<uint64_t>> out;   // successor ranks, by rank - 1
  rank_type get_node_count() const { return len.size(); }
  id_type rank_to_id(rank_type r) const { return 3 * r + 7; }
  rank_type id_to_rank(id_type id) const { return (id - 7) / 3; }
  uint64_t node_length(id_type id) const { return len[id_to_rank(id) - 1]; }
  template <class F>
  void for_each_node(F f, rank_type from = 1) const {
    for (rank_type r = from; r <= len.size(); ++r)
      if (!f(r, rank_to_id(r))) return;
  }
  template <class F>
  void for_each_edges_out(id_type id, F f) const {
    for (uint64_t to : out[id_to_rank(id) - 1])
      if (!f(rank_to_id(to), 0)) return;
  }
};

static int failures = 0;
#define CHECK(cond)                                                   \
  do {                                                                \
    if (!(cond)) {                                                    \
      std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                     \
    }                                                                 \
  } while (0)

static orc_mat view(RCRS const& m) {
  orc_mat o;
  o.nrows = m.numRows();
  o.ncols = m.numCols();
  o.nentries = m.get_entries().size();
  o.nnz = m.nnz();
  o.rowmap = const_cast<uint64_t*>(m.get_rowmap().data());
  o.entries = const_cast<uint32_t*>(m.get_entries().data());
  return o;
}

static bool same(RCRS const& m, orc_mat* o) {
  bool ok = o && m.numRows() == o->nrows && m.numCols() == o->ncols && m.nnz() == o->nnz &&
            m.get_entries().size() == o->nentries;
  for (size_t i = 0; ok && i <= m.numRows(); ++i) ok = m.get_rowmap()[i] == o->rowmap[i];
  for (size_t i = 0; ok && i < o->nentries; ++i) ok = m.get_entries()[i] == o->entries[i];
  orc_mat_free(o);
  return ok;
}

int main() {
  diverg::ScopedRuntime runtime;
  dvg_graph_params gp{};
  gp.n_backbone = 60000;
  gp.snp_rate = 0.007;
  gp.indel_rate = 0.003;
  gp.ins_frac = 0.5;
  gp.indel_lmin = 1;
  gp.indel_lmax = 10;
  gp.seed = 42;
  dvg_host_matrix hm{};
  if (dvg_gen_graph_adjacency(&gp, &hm, nullptr) != 0) return 2;
  RCRS ra(hm.ncols, std::vector<uint32_t>(hm.entries, hm.entries + hm.nentries),
          std::vector<uint64_t>(hm.rowmap, hm.rowmap + hm.nrows + 1), hm.nnz);
  dvg_gen_free(&hm);
  orc_mat va = view(ra);

  // ETI entry point == templated entry point == oracle (test_dindex.cpp:177-206)
  RCRS eti = diverg::util::create_distance_index(ra, 100, 300);
  RCRS tpl = diverg::util::create_distance_index<RCRS, diverg::DefaultSparseConfiguration>(ra, 100, 300);
  CHECK(eti.get_rowmap() == tpl.get_rowmap() && eti.get_entries() == tpl.get_entries() && eti.nnz() == tpl.nnz());
  CHECK(same(eti, orc_dindex(&va, 100, 300, 1, 0)));

  // the <uint32_t, uint32_t> overload (dindex_eti.hpp:50-53, test_dindex.cpp:208-234)
  RCRS32 ra32(ra.numCols(), ra.get_entries(), std::vector<uint32_t>(ra.get_rowmap().begin(), ra.get_rowmap().end()));
  RCRS32 d32 = diverg::util::create_distance_index(ra32, 1, 3);
  RCRS d64 = diverg::util::create_distance_index(ra, 1, 3);
  CHECK(d32.nnz() == d64.nnz() && d32.get_entries() == d64.get_entries());
  for (size_t i = 0; i < d64.get_rowmap().size(); ++i) CHECK(d32.get_rowmap()[i] == d64.get_rowmap()[i]);

  // range operations
  CHECK(same(diverg::range_spgemm(ra, ra), orc_spgemm(&va, &va, 0, 0)));
  RCRS id = diverg::create_range_identity_matrix<RCRS>(ra.numRows());
  orc_mat* oid = orc_identity(ra.numRows());
  CHECK(same(diverg::range_spadd(ra, id), orc_spadd(&va, oid)));
  orc_mat_free(oid);
  CHECK(same(diverg::range_power(ra, 7), orc_power(&va, 7, 0, 0)));

  // membership, at(), serialisation
  std::mt19937_64 rng(7);
  for (int q = 0; q < 20000; ++q) {
    uint32_t i = rng() % eti.numRows(), j = i + rng() % 400;
    if (j >= eti.numCols()) continue;
    bool dense = false;
    for (uint64_t k = eti.rowMap(i); k < eti.rowMap(i + 1); k += 2)
      dense = dense || (eti.entry(k) <= j && j <= eti.entry(k + 1));
    CHECK(eti(i, j) == dense && eti.at(i, j) == dense);
  }
  bool threw = false;
  try {
    eti.at(eti.numRows(), 0);
  } catch (std::runtime_error const&) {
    threw = true;
  }
  CHECK(threw);
  std::stringstream ss;
  eti.serialize(ss);
  RCRS back;
  back.load(ss);
  CHECK(back.get_rowmap() == eti.get_rowmap() && back.get_entries() == eti.get_entries() &&
        back.nnz() == eti.nnz() && back.numCols() == eti.numCols());

  // merging two indices of one graph is their union (dindex.hpp:556-570)
  {
    RCRS near = diverg::util::create_distance_index(ra, 1, 3);
    RCRS far = diverg::util::create_distance_index(ra, 100, 300);
    RCRS merged = diverg::util::merge_distance_index<RCRS>(near, far);
    orc_mat vn = view(near), vf = view(far);
    CHECK(same(merged, orc_spadd(&vn, &vf)));
    CHECK(merged.nnz() >= far.nnz() && merged.nnz() >= near.nnz());
  }

  // adjacency of the node graph == the generator's adjacency (adjacency.hpp:249-265)
  {
    uint64_t nn = 0, ne = 0;
    uint32_t *lens = nullptr, *edges = nullptr;
    CHECK(dvg_gen_graph_nodes(&gp, &nn, &lens, &ne, &edges) == 0);
    NodeGraph g;
    g.len.assign(lens, lens + nn);
    g.out.resize(nn);
    for (uint64_t e = 0; e < ne; ++e) g.out[edges[2 * e] - 1].push_back(edges[2 * e + 1]);
    dvg_gen_free_ptr(lens);
    dvg_gen_free_ptr(edges);
    RCRS adj = diverg::util::range_adjacency_matrix<RCRS>(g);
    CHECK(adj.get_rowmap() == ra.get_rowmap() && adj.get_entries() == ra.get_entries() && adj.nnz() == ra.nnz());
    // the graph is one component: ranks [1, 3) leave an edge behind, which throws
    threw = false;
    try {
      diverg::util::range_adjacency_matrix<RCRS>(g, 1, 3);
    } catch (std::runtime_error const&) {
      threw = true;
    }
    CHECK(threw);
  }

  // invalid window: the reference aborts, the B200 path throws
  threw = false;
  try {
    diverg::util::create_distance_index(ra, 3, 2);
  } catch (std::runtime_error const&) {
    threw = true;
  }
  CHECK(threw);

  if (failures) return 1;
  std::printf("shim ok: index %u rows, %zu ranges, nnz %lu\n", eti.numRows(), eti.get_entries().size() / 2,
              (unsigned long)eti.nnz());
  return 0;
}
