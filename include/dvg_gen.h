/*
 * dvg_gen.h -- seeded synthetic workloads for the distance-index path.
 *
 * Host-only C ABI of libdvg_gen.so.  It produces, on the CPU, the inputs the
 * benchmarks and tests feed to the device path:
 *   - the range-CRS adjacency matrix of a synthetic sequence graph with the
 *     layout of diverg::util::adjacency_matrix (adjacency.hpp:170-228 in the
 *     reference): one locus per base, loci numbered in topological node order,
 *     a locus links to the next locus of its node, a node's last locus links
 *     to the first locus of each successor; rows are then converted to ranges
 *     as crs_matrix::append does (crs_matrix.hpp:197-242);
 *   - random banded range-CRS matrices (the kernel microbenchmark shape);
 *   - uniformly random Boolean matrices (the reference's test shapes,
 *     test/src/test_range_sparse.cpp:516-520).
 * Every generator is deterministic in its seed and independent of the number
 * of host threads.  Buffers are allocated with malloc and released with
 * dvg_gen_free.
 */
#ifndef DVG_GEN_H
#define DVG_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A host range-CRS matrix: rowmap[nrows+1] counts entries (two per range),
 * entries[rowmap[nrows]] holds inclusive [start,end] pairs. */
typedef struct dvg_host_matrix {
  uint32_t nrows;
  uint32_t ncols;
  uint64_t nentries;
  uint64_t nnz;
  uint64_t* rowmap;
  uint32_t* entries;
} dvg_host_matrix;

/* Bubble model of the synthetic sequence graph.  A bubble is anchored after a
 * backbone base with probability (snp_rate + indel_rate) per base; anchors
 * never overlap a previous bubble.  A bubble is structural with probability
 * sv_frac, else an SNP with probability snp_rate/(snp_rate+indel_rate), else
 * an indel.  An indel is an insertion (alt branch parallel to an empty ref)
 * with probability ins_frac, else a deletion (skip edge over ref bases).
 * Indel lengths are uniform in [indel_lmin, indel_lmax] when
 * indel_geometric_mean == 0, else geometric with that mean, capped at
 * indel_lmax.  Structural bubbles are insertions or deletions (50/50) with
 * length uniform in [sv_lmin, sv_lmax]. */
typedef struct dvg_graph_params {
  uint64_t n_backbone;
  double snp_rate;
  double indel_rate;
  double ins_frac;
  uint32_t indel_lmin;
  uint32_t indel_lmax;
  double indel_geometric_mean;
  double sv_frac;
  uint32_t sv_lmin;
  uint32_t sv_lmax;
  uint64_t seed;
} dvg_graph_params;

/* Counts of what the graph generator placed. */
typedef struct dvg_graph_stats {
  uint64_t n_loci;
  uint64_t n_snp;
  uint64_t n_ins;
  uint64_t n_del;
  uint64_t n_sv;
  uint64_t n_alt_loci;
} dvg_graph_stats;

/* Adjacency matrix (range CRS, n_loci x n_loci) of the synthetic graph.
 * Returns 0 on success, nonzero on invalid parameters or allocation failure. */
int dvg_gen_graph_adjacency(const dvg_graph_params* p, dvg_host_matrix* out, dvg_graph_stats* stats);

/* The same graph as a node/edge list with one single-base node per locus
 * (node ids are 1-based, node i+1 holds locus i): edges[2k], edges[2k+1] are
 * (from_id, to_id).  Used to cross-check the adjacency layout. */
int dvg_gen_graph_edges(const dvg_graph_params* p, uint64_t* n_nodes, uint64_t* n_edges, uint32_t** edges);

/* The same graph with its chains of bases compacted into nodes: a base
 * starts a node unless its only predecessor is the previous base and that
 * base's only successor is it.  Node ids are 1-based in base order (rank
 * order), node_len[id-1] bases each; edges[2k], edges[2k+1] = (from_id,
 * to_id) link a node's last base to a successor's first base.  The range
 * adjacency of this node graph (util::range_adjacency_matrix,
 * adjacency.hpp:249-265) is the matrix of dvg_gen_graph_adjacency.  Release
 * both arrays with dvg_gen_free_ptr. */
int dvg_gen_graph_nodes(const dvg_graph_params* p, uint64_t* n_nodes, uint32_t** node_len, uint64_t* n_edges,
                        uint32_t** edges);

/* Random banded matrix: row i holds Poisson(mean_ranges) ranges whose starts
 * are uniform in [i-half_width, i+half_width] and whose lengths are geometric
 * with mean mean_len; ranges are clipped to the band and to [0,n), sorted and
 * merged when they overlap or touch, so every row is canonical. */
int dvg_gen_banded(uint32_t n, uint32_t half_width, double mean_ranges, double mean_len, uint64_t seed,
                   dvg_host_matrix* out);

/* Uniformly random n x n Boolean matrix with exactly nnz non-zeros (distinct
 * columns per row, rows drawn uniformly), converted to range CRS. */
int dvg_gen_random(uint32_t n, uint64_t nnz, uint64_t seed, dvg_host_matrix* out);

/* Locus pairs for membership queries: a fraction in_range_frac of the pairs
 * is (i, j) with j reached from i by a walk of a uniform length in [dmin,dmax]
 * along the adjacency `adj`'s first successor range; the rest is uniform in
 * [0,n)^2.  pairs[2q], pairs[2q+1] = (i, j). */
int dvg_gen_pairs(const dvg_host_matrix* adj, uint64_t npairs, double in_range_frac, uint32_t dmin,
                  uint32_t dmax, uint64_t seed, uint32_t* pairs);

void dvg_gen_free(dvg_host_matrix* m);
void dvg_gen_free_ptr(void* p);

#ifdef __cplusplus
}
#endif

#endif /* DVG_GEN_H */
