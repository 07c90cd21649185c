/*
 * dvg.h -- C ABI of libdvg.so: DiVerG's distance-index path on one B200.
 *
 * Plain C, plain pointers and sizes.  Every entry point returns a dvg_status;
 * dvg_last_error() gives a message for the last failure of the calling thread.
 * The C++ headers under include/diverg/ wrap this ABI in the reference's own
 * API (CRSMatrix<RangeDynamic,...>, range_spgemm, create_distance_index, ...);
 * each declaration below names the reference interface (file:line in
 * cartoonist/diverg v1.1.1) it stands in for.
 *
 * Matrices are range CRS, as CRSMatrix<crs_matrix::RangeDynamic, bool,
 * uint32_t, TSize> (include/diverg/crs_matrix.hpp:1873-2004):
 *   rowmap  : TSize[nrows+1] counting ENTRIES (two per range), rowmap[0] = 0
 *   entries : uint32_t[rowmap[nrows]], inclusive [start,end] pairs, sorted
 *   nnz     : number of non-zero columns, sum of (end - start + 1)
 * A dvg_matrix lives in device memory (HBM) until dvg_matrix_free.
 *
 * Threading: calls on one context are serialised by the context; distinct
 * contexts may be used from distinct threads.  All work of a context is
 * issued on its stream; calls that return sizes or status to the host
 * synchronise that stream.
 */
#ifndef DVG_H
#define DVG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum dvg_status {
  DVG_OK = 0,
  DVG_ERR_INVALID_ARG = 1,   /* bad argument (the reference asserts / exits 134) */
  DVG_ERR_OOM = 2,           /* device or pinned host allocation failed */
  DVG_ERR_DEVICE = 3,        /* CUDA error, or no usable sm_100 device */
  DVG_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up */
  DVG_ERR_NOT_INITIALIZED = 5,
  DVG_ERR_OVERFLOW = 6       /* result does not fit the requested index type */
} dvg_status;

typedef struct dvg_context dvg_context;
typedef struct dvg_matrix dvg_matrix;

/* Counters of the work a context issued since its creation or the last
 * dvg_stats_reset. */
typedef struct dvg_stats {
  uint64_t kernel_launches;   /* kernels of this library launched */
  uint64_t spgemm_calls;      /* range SpGEMM products */
  uint64_t spadd_calls;       /* range SpAdd sums */
  uint64_t host_syncs;        /* stream synchronisations for size read-backs */
  uint64_t alg_bytes;         /* compulsory bytes: read A and B once, write C once */
  uint64_t spgemm_alg_bytes;  /* the share of alg_bytes due to SpGEMM */
  uint64_t range_ops;         /* B ranges visited by SpGEMM (work metric) */
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  /* device time of the kernels, measured with CUDA events on the context's
   * stream while the "timing" option is on (0 otherwise) */
  uint64_t spgemm_ns;           /* single-pass SpGEMM kernels (counts, offsets and runs in one pass) */
  uint64_t spgemm_levels_ns;    /* building union levels of B for long-range products */
  uint64_t scan_ns;             /* rowmap scans (SpGEMM and SpAdd) */
  uint64_t spadd_ns;            /* SpAdd passes */
  uint64_t spgemm_direct_tiles; /* SpGEMM row tiles that missed the staged path */
  uint64_t spgemm_reruns;       /* SpGEMMs re-run after an output capacity overflow */
  uint64_t spgemm_light;        /* SpGEMMs run in the thread-per-row mode */
  uint64_t spgemm_slow_rows;    /* thread-per-row rows that missed the run list (warp path) */
  uint64_t host_alloc_ns;       /* host time spent in device allocation calls */
  uint64_t host_sync_ns;        /* host time spent waiting on stream synchronisation */
  uint64_t spgemm_fused_adds;   /* products computed as D + A B in one pass */
  uint64_t graph_launches;      /* CUDA graphs launched (batched builds) */
  uint64_t autotune_builds;     /* planned builds run by the autotuner */
  uint64_t spgemm_levels;       /* union levels of B built for long-range products */
  uint64_t host_prepare_ns;     /* host time planning builds (buffers, shapes) */
  uint64_t host_launch_ns;      /* host time issuing the planned builds' work */
  uint64_t host_meminfo_ns;     /* host time querying free device memory */
  uint64_t query_ns;            /* membership-query kernels (with the "timing" option) */
  uint64_t query_pairs;         /* locus pairs answered */
} dvg_stats;

/* ---- runtime: runtime.hpp:22-53 (initialize_runtime / finalize_runtime /
 *      ScopedRuntime) and src/eti/runtime.cpp ------------------------------ */

/* Opens `device` (a CUDA ordinal), checks it is an sm_100 part and creates a
 * context with its own non-blocking stream. */
dvg_status dvg_init(int device, dvg_context** ctx);
/* Waits for the context's work, frees its scratch and destroys the stream if
 * the context owns it.  Matrices must be freed before. */
dvg_status dvg_shutdown(dvg_context* ctx);
/* Issue the context's work on a caller-owned cudaStream_t (NULL restores the
 * context's own stream). */
dvg_status dvg_set_stream(dvg_context* ctx, void* cuda_stream);
dvg_status dvg_synchronize(dvg_context* ctx);
/* Tuning knobs: "algo" (0 only: the single-pass SpGEMM kernels), "chunk_rows"
 * (fused path: 0 = automatic, else rows per output chunk, a multiple of 32 up
 * to 2048), "spgemm_mode" (fused path: 0 = automatic -- tile-staged when A's
 * ranges average more than 8 columns, else a thread per row --, 1 =
 * tile-staged rows, 2 = a thread per row), "dindex_schedule" (0 = sum of powers of A, the
 * default; 1 = the reference's squaring of A + I; both give the same index),
 * "planned_build" (1 = index builds run as a planned sequence of products with
 * pre-allocated buffers and no host round trip between them, the default; 0 =
 * one read-back per product), "plan_growth" (planned builds: the entry
 * capacity of every step as a percentage of the input's entries, 300 by
 * default and adapted after each build; a step that outgrows it makes the
 * build re-run on the read-back path), "row_slot" (thread-per-row kernel: run-list
 * entries per thread, 0 = 16, 1 = 24, the default, 2 = 32), "row_stage"
 * (thread-per-row kernel: 1 = a counted chunk's output waits in a staging
 * buffer, 16 entries a row for two chunks per CTA, while its offset resolves,
 * and is copied out one iteration later, the default; 0 = every chunk waits
 * for its offset and is written out in its own iteration), "spgemm_levels"
 * (1 = a thread-per-row product whose A ranges average 4 or more rows -- up
 * to 8 in automatic mode, which stages tiles above that -- first builds union
 * levels of B -- level k row j is the union of B's rows j .. j + 2^k - 1 --
 * and reads a couple of level rows per A range instead of its B rows, the
 * default; 0 = never), "autotune" (1 =
 * batches time the row kernel's shapes once per window and size class and
 * keep the fastest, the default; 0 = use "row_slot" and "chunk_rows"),
 * "timing" (1 =
 * time kernels with CUDA events into dvg_stats).  Every setting gives the
 * same results. */
dvg_status dvg_set_option(dvg_context* ctx, const char* key, int64_t value);
/* Device memory freed by the context's operations is kept for reuse; this
 * returns all of it to the CUDA allocator. */
dvg_status dvg_trim(dvg_context* ctx);
dvg_status dvg_get_stats(const dvg_context* ctx, dvg_stats* out);
dvg_status dvg_stats_reset(dvg_context* ctx);
const char* dvg_last_error(void);
const char* dvg_status_string(dvg_status s);

/* ---- matrices: crs_matrix_device.hpp:192-238 (entries_device_view /
 *      rowmap_device_view, H2D) and :265-290 (make_crs_matrix, D2H) -------- */

/* Copies a host range-CRS matrix to the device.  nnz may be 0, in which case
 * it is recounted (CRSMatrix ctor, crs_matrix.hpp:1894-1902). */
dvg_status dvg_matrix_upload(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint64_t* rowmap,
                             const uint32_t* entries, uint64_t nnz, dvg_matrix** out);
/* Same with a 32-bit rowmap (CRSMatrix<..., uint32_t, uint32_t>). */
dvg_status dvg_matrix_upload_u32(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint32_t* rowmap,
                                 const uint32_t* entries, uint64_t nnz, dvg_matrix** out);
/* Wraps caller-owned device arrays without copying; the arrays must outlive
 * the handle and are not freed by dvg_matrix_free. */
dvg_status dvg_matrix_wrap_device(dvg_context* ctx, uint32_t nrows, uint32_t ncols, const uint64_t* d_rowmap,
                                  const uint32_t* d_entries, uint64_t nentries, uint64_t nnz, dvg_matrix** out);
/* numRows / numCols / rowMap(numRows) / nnz (crs_matrix.hpp:1274-1369, 1980). */
dvg_status dvg_matrix_info(const dvg_matrix* m, uint32_t* nrows, uint32_t* ncols, uint64_t* nentries, uint64_t* nnz);
dvg_status dvg_matrix_device_arrays(const dvg_matrix* m, const uint64_t** d_rowmap, const uint32_t** d_entries);
/* Copies to caller buffers of nrows+1 and nentries elements. */
dvg_status dvg_matrix_download(dvg_context* ctx, const dvg_matrix* m, uint64_t* rowmap, uint32_t* entries);
dvg_status dvg_matrix_download_u32(dvg_context* ctx, const dvg_matrix* m, uint32_t* rowmap, uint32_t* entries);
dvg_status dvg_matrix_free(dvg_context* ctx, dvg_matrix* m);

/* ---- range operations: include/diverg/range_sparse.hpp ------------------- */

/* create_range_identity_matrix<RCRS>(n), range_sparse.hpp:95-110. */
dvg_status dvg_range_identity(dvg_context* ctx, uint32_t n, dvg_matrix** out);
/* range_spadd(a, b), range_sparse.hpp:470-477 (-> :364-428, :112-357). */
dvg_status dvg_range_spadd(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, dvg_matrix** c);
/* range_spgemm(a, b, config), range_sparse.hpp:2325-2332 (-> :2215-2281). */
dvg_status dvg_range_spgemm(dvg_context* ctx, const dvg_matrix* a, const dvg_matrix* b, dvg_matrix** c);
/* range_power(a, k, config), range_sparse.hpp:2362-2368 (-> :2370-2431). */
dvg_status dvg_range_power(dvg_context* ctx, const dvg_matrix* a, unsigned k, dvg_matrix** c);

/* ---- distance index: dindex.hpp:46-189, dindex_eti.hpp:44-53 ------------- */

/* create_distance_index(ra, dmin, dmax): A^dmin * (A+I)^(dmax-dmin).
 * Requires dmin <= dmax, dmax != 0 and a square `ra`. */
dvg_status dvg_create_distance_index(dvg_context* ctx, const dvg_matrix* ra, unsigned dmin, unsigned dmax,
                                     dvg_matrix** out);

/* Distance indices of `ngraphs` independent graphs in one pass (no
 * counterpart in the reference, which builds one graph per call): out[k]
 * receives exactly what dvg_create_distance_index(graphs[k], dmin[k],
 * dmax[k]) gives.  Graphs with the same window are laid side by side as one
 * block-diagonal matrix and built together; the block-diagonal assemblies and
 * the builds of all windows are captured into one CUDA graph and launched
 * once; the autotuner (option "autotune") picks the row kernel's shape on the
 * first batch of each window and size class.  On failure no output is left
 * allocated. */
dvg_status dvg_batch_distance_index(dvg_context* ctx, uint32_t ngraphs, const dvg_matrix* const* graphs,
                                    const unsigned* dmin, const unsigned* dmax, dvg_matrix** out);

/* ---- self-test of the bounded device waits
 *
 * Every device-side wait of the library (the chunk look-backs of the SpGEMM
 * kernels) gives up after a bounded number of polls, records a timeout the
 * host turns into DVG_ERR_TIMEOUT, and leaves the context usable.  This runs
 * the row kernel's look-back on a chunk whose predecessor nothing publishes,
 * with the wait bounded by spin_limit polls (0: 1 poll), and returns that
 * DVG_ERR_TIMEOUT; any other status means the bound did not hold. */
dvg_status dvg_selftest_bounded_wait(dvg_context* ctx, uint32_t spin_limit);

/* ---- the on-chip rate of a range operation
 *
 * No counterpart in the reference: a measurement for the roofline of the
 * warp-per-row SpGEMM (products with long A ranges), whose bound is on-chip
 * work, not HBM.  Times warps that OR ranges held in L1/L2 into bitmap
 * windows in shared memory and take the runs out, exactly the kernel's inner
 * work without its A / B indirection or write-out, and stores the range
 * operations a second the device sustained.  Synchronises the context's
 * stream. */
dvg_status dvg_calibrate_range_ops(dvg_context* ctx, double* ops_per_second);

/* No counterpart in the reference: a measurement for the roofline of the
 * membership query, whose pairs read rows at random.  Times independent
 * 8-byte reads at uniformly random addresses of a device buffer of `bytes`
 * (at least 8 MiB; the size of the queried index gives the same DRAM and TLB
 * behaviour), each touching one 32-byte sector, and stores the reads a second
 * the device sustained.  Synchronises the context's stream. */
dvg_status dvg_calibrate_random_reads(dvg_context* ctx, uint64_t bytes, double* reads_per_second);

/* ---- adjacency construction: util::range_adjacency_matrix
 *      (adjacency.hpp:249-265) over util::adjacency_matrix (:170-228) and the
 *      Basic->Range conversion of crs_matrix::append (crs_matrix.hpp:197-242)
 *
 * The range-CRS adjacency matrix of a sequence graph, built on the device.
 * Nodes have ids 1..nnodes in rank order; node_len[id-1] is the length of
 * node id in bases (at least 1); edges[2k], edges[2k+1] = (from_id, to_id),
 * in any order, repeats allowed.  The matrix covers the nodes lower .. upper-1
 * (upper = 0: through the last node; lower = 1 and upper = 0 is the whole
 * graph, the reference's defaults): one row and column per base, numbered in
 * rank order from the first base of node `lower`; each base links to the next
 * base of its node, a node's last base to the first base of every successor,
 * columns sorted, then rows turned into ranges as append does (a column
 * extends the open range only if it is the range's end + 1, so a repeated
 * edge gives a repeated range and a non-canonical matrix).  nnz is the number
 * of Basic entries, (bases - nodes) + edges.  Edges whose source lies outside
 * the range are ignored; an edge from inside to outside the range is
 * DVG_ERR_INVALID_ARG (the reference requires the range to be closed, its
 * components).  More than 2^32 - 2 bases is DVG_ERR_OVERFLOW. */
dvg_status dvg_adjacency_from_graph(dvg_context* ctx, uint32_t nnodes, const uint32_t* node_len, uint64_t nedges,
                                    const uint32_t* edges, uint32_t lower, uint32_t upper, dvg_matrix** out);

/* ---- range SpGEMM without device allocation -------------------------------
 * No counterpart in the reference.  Some callers of this library cannot let it
 * allocate device memory: a server that reserves the GPU's memory for resident
 * indices up front and hands out buffers from its own pool, a host runtime
 * (a JVM, a database engine) that owns every device allocation through its
 * own allocator, and latency-critical paths where cudaMalloc/cudaFree would
 * synchronise the device.  This entry point computes C = A * B exactly as
 * dvg_range_spgemm does, from caller-owned device arrays into caller-owned
 * device arrays, and allocates nothing: no cudaMalloc, no cudaFree, no
 * allocating library call.  It needs no dvg_context.
 *
 * Its scratch is a fixed array inside the library (about 1 MiB, held on every
 * GPU that loads the library until the process exits), which limits the
 * product to a_nrows <= 67,108,864; larger products are rejected with
 * DVG_ERR_INVALID_ARG.  Every call looks up that array's device address on
 * the current device.  All calls share the array: calls whose work overlaps
 * on the GPU race and must be serialised by the caller.
 *
 * The inputs are checked on the device before the product reads through
 * them; a malformed A or B (rowmap[0] != 0, a decreasing rowmap or odd row
 * length, rowmap[n] != nentries, a column >= ncols) returns
 * DVG_ERR_INVALID_ARG, names the operand and the checks in dvg_last_error(),
 * and leaves d_c_rowmap untouched.  The product always runs the tile-staged
 * kernel; dvg_range_spgemm picks the thread-per-row kernel for short-range
 * operands and is faster there.
 *
 * d_c_rowmap holds a_nrows + 1 entries; d_c_entries holds c_capacity entries.
 * On return *c_nentries and *c_nnz describe C.  If c_capacity is too small
 * the call returns DVG_ERR_OVERFLOW with c_rowmap complete and *c_nentries
 * set to the required capacity.  The call waits on `cuda_stream` twice: once
 * for the input checks and once for the product's size. */
dvg_status dvg_range_spgemm_noalloc(uint32_t a_nrows, uint32_t a_ncols, const uint64_t* d_a_rowmap,
                                    const uint32_t* d_a_entries, uint64_t a_nentries, uint32_t b_nrows,
                                    uint32_t b_ncols, const uint64_t* d_b_rowmap, const uint32_t* d_b_entries,
                                    uint64_t b_nentries, uint64_t* d_c_rowmap, uint32_t* d_c_entries,
                                    uint64_t c_capacity, uint64_t* c_nentries, uint64_t* c_nnz, void* cuda_stream);

/* ---- membership query: crs_matrix.hpp:1197-1243 (operator() / at) -------- */

/* out[q] = index(pairs[2q], pairs[2q+1]) as 0/1 for q < npairs; device
 * pointers.  Pairs outside [0,nrows) x [0,ncols) answer 0 and make the call
 * return DVG_ERR_INVALID_ARG (at() throws std::runtime_error there). */
dvg_status dvg_query_batch(dvg_context* ctx, const dvg_matrix* index, const uint32_t* d_pairs, uint64_t npairs,
                           uint8_t* d_out);
/* The same with host buffers (copies in and out on the context's stream). */
dvg_status dvg_query_batch_host(dvg_context* ctx, const dvg_matrix* index, const uint32_t* pairs, uint64_t npairs,
                                uint8_t* out);

/* ---- serving: a request loop over resident indices ------------------------
 * No counterpart in the reference, which builds one index per call and
 * answers one pair per call.  A server owns two contexts on one device: a
 * build worker admits waiting builds in arrival order while their predicted
 * device footprint fits the HBM budget next to the resident indices, and
 * builds all admitted graphs as one batch (dvg_batch_distance_index); a query
 * worker runs every query batch whose index is resident, up to
 * max_inflight_queries at once, on its own stream, concurrently with the
 * builds.  Requests that arrive while others are on the device join the next
 * batch or take the next free query slot.  Buffers passed to a request must
 * stay valid until its completion is polled; pinned host buffers are copied
 * directly, other ones through staging. */
typedef struct dvg_server dvg_server;

typedef struct dvg_server_config {
  int device;
  uint64_t hbm_budget_bytes;     /* resident indices + builds in flight; 0: 80 % of free memory */
  uint32_t max_batch_builds;     /* builds merged into one batch; 0: 64 */
  uint32_t max_inflight_queries; /* query batches on the device at once; 0: 8 */
  uint32_t build_workers;        /* build batches on the device at once, each on its own stream; 0: 2 */
} dvg_server_config;

typedef struct dvg_completion {
  uint64_t request;        /* id returned at submission */
  int32_t status;          /* dvg_status of the request */
  uint32_t kind;           /* 1: build, 2: query batch */
  uint64_t submit_ns;      /* steady-clock times: submitted, started on the device, completed */
  uint64_t start_ns;
  uint64_t done_ns;
  uint64_t index_entries;  /* builds: the index's entries and nnz */
  uint64_t index_nnz;
  uint64_t invalid_pairs;  /* query batches: pairs outside the index (answered 0) */
} dvg_completion;

typedef struct dvg_server_stats {
  uint64_t builds_submitted;
  uint64_t builds_done;
  uint64_t build_batches;
  uint64_t queries_submitted;
  uint64_t queries_done;
  uint64_t pairs_answered;
  uint64_t resident_bytes;       /* indices held in HBM */
  uint64_t peak_reserved_bytes;  /* most resident + predicted in-flight bytes seen */
  uint64_t hbm_budget_bytes;
  uint64_t build_reruns;         /* builds whose planned capacity was outgrown: re-run step by step */
  uint64_t build_batch_ns_max;   /* longest build batch, host clock */
  uint64_t build_alloc_ns;       /* build worker: host time in device allocation calls */
  uint64_t build_sync_ns;        /* build workers: host time waiting for their streams */
  uint64_t builds_failed;        /* builds completed with an error (each alone: batch-mates unaffected) */
  uint64_t builds_rebuilt_alone; /* members of a failed batch built again one by one */
} dvg_server_stats;

dvg_status dvg_server_create(const dvg_server_config* cfg, dvg_server** out);
/* Finishes every submitted request, then frees the server and its indices. */
dvg_status dvg_server_destroy(dvg_server* s);
/* Queues the index build of an n x n range-CRS graph (host arrays); the
 * request id is also the id of the index it makes. */
dvg_status dvg_server_submit_build(dvg_server* s, uint32_t n, const uint64_t* rowmap, const uint32_t* entries,
                                   unsigned dmin, unsigned dmax, uint64_t* request);
/* Queues a batch of (row, column) membership queries against index `index`
 * (a build request id); answers[q] receives 0 or 1. */
dvg_status dvg_server_submit_query(dvg_server* s, uint64_t index, const uint32_t* pairs, uint64_t npairs,
                                   uint8_t* answers, uint64_t* request);
/* Takes up to `max` completions, waiting up to wait_ms for the first. */
dvg_status dvg_server_poll(dvg_server* s, dvg_completion* out, uint32_t max, uint32_t* n, uint32_t wait_ms);
dvg_status dvg_server_index_info(dvg_server* s, uint64_t index, uint32_t* nrows, uint64_t* nentries, uint64_t* nnz);
/* Copies a resident index to host arrays (sizes from dvg_server_index_info). */
dvg_status dvg_server_download(dvg_server* s, uint64_t index, uint64_t* rowmap, uint32_t* entries);
/* Drops a resident index once the query batches on it have finished. */
dvg_status dvg_server_release(dvg_server* s, uint64_t index);
dvg_status dvg_server_get_stats(dvg_server* s, dvg_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* DVG_H */
