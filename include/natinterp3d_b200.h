/*
 * natinterp3d_b200 C ABI.
 *
 * Two shared libraries sit under the Python package:
 *   libnif_mesh.so  host-side Delaunay construction (natinterp3d's own
 *                   constructor) and export of the packed mesh arrays;
 *   libnif_cuda.so  the sm_100a query kernels.
 *
 * Every entry point returns an int status (NIF_OK or a negative code below)
 * and never aborts or exits the process.  Device pointers (d_*) are plain
 * CUDA device addresses allocated by the caller; `stream` is a cudaStream_t
 * (NULL = legacy default stream).  No entry point allocates device memory:
 * sizes are queried first (nif_dmesh_bytes, nif_query_workspace_bytes) and
 * the caller passes the buffers in.
 *
 * Citations are to natinterp3d's sources (src/natinterp3d/...).
 */
#ifndef NATINTERP3D_B200_H
#define NATINTERP3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define NIF_OK 0
#define NIF_ERR_ARG (-1)        /* invalid argument (natinterp3d: ValueError) */
#define NIF_ERR_DEGENERATE (-2) /* key set the constructor cannot triangulate */
#define NIF_ERR_NOMEM (-3)      /* host allocation failed */
#define NIF_ERR_INTERNAL (-4)   /* inconsistent mesh / internal check failed */
#define NIF_ERR_OVERFLOW (-5)   /* nnz > INT32_MAX; natinterp3d returns -1 here,
                                   natural_insertionfree.c:901-912, and Python
                                   raises OverflowError (natinterp3d_cython.pyx:86-88, 129-131) */
#define NIF_ERR_WALK (-6)       /* a point-location walk exceeded its step limit
                                   (natinterp3d's walk, delaunay.c:398-405, has none) */
#define NIF_ERR_CUDA (-7)       /* a CUDA runtime call failed */
#define NIF_ERR_CAPACITY (-8)   /* a query exceeded the large kernel's per-query limits */
#define NIF_ERR_WORKSPACE (-9)  /* a caller buffer is smaller than the queried size */
#define NIF_ERR_TOO_LARGE (-10) /* more queries than nif_interpolate_noalloc's fixed scratch holds */

/* ---- element types ----------------------------------------------------- */
#define NIF_F64 0
#define NIF_F32 1

/* ---- workspace modes --------------------------------------------------- */
#define NIF_MODE_WEIGHTS 0      /* get_weights: rows are counted (and short ones staged), then
                                   written to the CSR */
#define NIF_MODE_INTERP 1       /* interpolate: rows are reduced against values in place */

/* ======================================================================== */
/* libnif_mesh.so: host-side construction                                   */
/* ======================================================================== */

typedef struct nif_mesh nif_mesh;

/* Builds natinterp3d's Delaunay tetrahedralization of n centred keys
 * ([n][3] float64).  Replaces buildNewMeshAndVertices (natural.h:16,
 * natural.c:114-118) as called from natinterp3d_cython.pyx:64-65 and
 * :106-107.  Returns NIF_ERR_DEGENERATE where natinterp3d would exit(1)
 * (zero or non-finite extent along an axis). */
int nif_mesh_build(const double *keys_centered, int n, nif_mesh **out);

/* Releases the mesh.  Replaces freeMeshAndVertices (natural.h:18). */
void nif_mesh_free(nif_mesh *h);

/* Vertex count (n + 4 super-simplex vertices) and tet count of the mesh. */
int nif_mesh_sizes(const nif_mesh *h, int *n_vertices, int *n_tets);

/* Writes the packed mesh: vxyz [n+4][3] float64 (mesh coordinates, after the
 * constructor's perturbations, delaunay.c:513-522; super-simplex vertices at
 * rows n..n+3), tet_v [T][4] int32 (delaunay.h:60), tet_n [T][4] int32
 * (delaunay.h:64; -1 for NULL).  Tet order is the mesh's tet-list order,
 * the order natinterp3d packs tets in (natural_insertionfree.c:413-425). */
int nif_mesh_export(const nif_mesh *h, double *vxyz, int32_t *tet_v, int32_t *tet_n);

/* Degeneracy counters of the constructor (delaunay.c:106-107, 588, 649). */
int nif_mesh_degeneracies(const nif_mesh *h, int *coplanar, int *cospherical);

/* natinterp3d's own mesh object (for running natinterp3d's CPU query on the
 * same mesh when checking results). */
void *nif_mesh_native(const nif_mesh *h);

/* ======================================================================== */
/* libnif_cuda.so: device-resident mesh and query kernels                   */
/* ======================================================================== */

/* ---- GPU construction (opt-in; natinterp3d has no counterpart) ----------
 * The Delaunay tetrahedralization of n centred keys plus natinterp3d's
 * super-simplex (initSuperSimplex, delaunay.c:832-863), built on the device
 * by parallel Bowyer-Watson insertion rounds with exact predicates, in the
 * packed layout of nif_mesh_export (vxyz [n+4][3] with the super-simplex
 * vertices at rows n..n+3; tet_v, tet_n [T][4] with natinterp3d's face
 * order, delaunay.c:444-467).  For keys in general position this is the
 * same set of tets natinterp3d's constructor (buildMesh, delaunay.c:108-161)
 * produces; tet order and each tet's vertex rotation differ.  The result is
 * checked on the device with exact predicates (positive orientation,
 * neighbour symmetry, empty circumsphere across every interior face) and
 * the counts reported in *info.  Returns NIF_ERR_DEGENERATE where an exact
 * zero would decide the result (cospherical or coplanar keys that a cavity
 * meets, duplicate keys, zero extent): natinterp3d then perturbs keys
 * randomly (delaunay.c:513-522), and callers fall back to nif_mesh_build.
 * NIF_ERR_CAPACITY where an insertion's cavity exceeds 256 tets.  The tet
 * buffers hold nif_delaunay_max_tets(n) tets; *info->n_tets are written.
 * Synchronises `stream` once per insertion round. */
typedef struct {
    int64_t n_tets;             /* tets written */
    int32_t rounds;             /* insertion rounds */
    int32_t max_cavity;         /* largest cavity (tets) */
    int64_t exact_evaluations;  /* predicates the error bound could not certify */
    int32_t tet_slots;          /* slots used before compaction */
    int32_t error;              /* builder's internal error code, 0 if none */
    int64_t bad_orientation;    /* check: tets not positively oriented */
    int64_t bad_adjacency;      /* check: asymmetric neighbour entries */
    int64_t non_delaunay_faces; /* check: faces whose opposite vertex is inside */
    int64_t cospherical_faces;  /* check: ... exactly on the circumsphere */
} nif_delaunay_info;
int nif_delaunay_max_tets(int n, int *cap);
int nif_delaunay_workspace_bytes(int n, size_t *bytes);
int nif_delaunay_build(const double *d_keys, int n, void *d_ws, size_t ws_bytes, double *d_vxyz,
                       int32_t *d_tet_v, int32_t *d_tet_n, int tet_cap, void *stream,
                       nif_delaunay_info *info);

typedef struct nif_dmesh nif_dmesh;

/* Size in bytes of the device buffer that holds a resident mesh of
 * n_vertices (= keys + 4) and n_tets (at most 2^29 - 1) tets: vertices, tets, neighbours,
 * orientation and mirror flags, cached tet and face circumcentres, and the
 * tet centroids with an octree over them for the point-location seed (the
 * nearest tet centroid, which natinterp3d finds in a k-d tree built by its
 * constructor, delaunay.c:141-159).  (natinterp3d keeps the mesh as pointer-linked
 * structs, delaunay.h:44-70, and re-packs it on first query,
 * natural_insertionfree.c:397-450.) */
int nif_dmesh_bytes(int n_vertices, int n_tets, size_t *bytes);

/* Uploads a mesh: derives the resident arrays in d_buf from the packed
 * arrays written by nif_mesh_export (already copied to the device), and
 * returns a host handle.  Synchronises `stream`.  The packed input arrays
 * may be freed afterwards; d_buf must stay alive until nif_dmesh_destroy.
 * Replaces packMeshSimplices + precomputeOrientSigns
 * (natural_insertionfree.c:397-476), done once per mesh instead of per call. */
int nif_dmesh_create(const double *d_vxyz, const int32_t *d_tet_v, const int32_t *d_tet_n,
                     int n_vertices, int n_tets, void *d_buf, size_t buf_bytes, void *stream,
                     nif_dmesh **out);

/* Frees the host handle (the device buffer belongs to the caller). */
void nif_dmesh_destroy(nif_dmesh *m);

/* Tet/vertex counts, the centroid octree's size and the predicate state:
 * info = {n_vertices, n_tets, octree_nodes, octree_levels, 0, orient_uncertain,
 *         orient_flipped, predicate_mode}, where orient_uncertain counts the
 * tets whose orient3dfast sign (natural_insertionfree.c:457-476) the static
 * error bound cannot certify and orient_flipped those whose "> 0" flag the
 * exact sign changes. */
int nif_dmesh_info(const nif_dmesh *m, int64_t info[8]);

/* Geometric predicates of later query calls on this mesh.  natinterp3d uses
 * the signs of orient3dfast / inspherefast as they come (predicates.c:1687,
 * 3301; natural_insertionfree.c:461-514, delaunay.c:400) and never calls its
 * exact predicates; NIF_PRED_FAST (the default) does the same, bit for bit.
 * NIF_PRED_AUDIT gives the same results and counts, in nif_summary, the
 * evaluations whose fast value lies inside the static error bound
 * (re-evaluated exactly) and those whose decision the exact sign would
 * change.  NIF_PRED_EXACT decides every test by its exact sign (filter, then
 * expansion arithmetic); a query exactly on a face or edge then floods its
 * cavity from the lowest-id tet containing it.  A batch takes the modes its
 * meshes have when nif_batch_create runs.  (No counterpart in natinterp3d.) */
#define NIF_PRED_FAST 0
#define NIF_PRED_AUDIT 1
#define NIF_PRED_EXACT 2
int nif_dmesh_set_predicates(nif_dmesh *m, int mode);

/* Launch settings of the query kernels.  They change speed, never results:
 * every setting gives bit-identical output.  (No counterpart in natinterp3d,
 * whose query loop is OpenMP `schedule(dynamic, 64)` over Morton-sorted
 * queries, natural_insertionfree.c:856, 866-887.)
 *   blocks_per_sm  resident 4-warp blocks per SM of the shared-memory row
 *                  kernel, one warp per query: 6 (80 registers a thread) or
 *                  8 (64 registers, more spills, more warps hiding latency)
 *   bucket_shift   Morton bucket resolution of the query ordering, in bits per
 *                  axis relative to the size-based default: -2 .. 1
 *   tile           queries a warp takes per work item: 0 = a static grid
 *                  stride (one query per step), 1 .. 1024 = tiles of
 *                  consecutive bucket-ordered queries pulled from a device
 *                  counter.  For one mesh this is an upper bound: a call with
 *                  fewer than 2 x tile queries per resident warp uses smaller
 *                  tiles, or the static stride, so small calls fill the GPU
 * nif_dmesh_set_tuning applies to later query calls on the mesh (the
 * workspace size depends on bucket_shift: query nif_query_workspace_bytes
 * after setting it); nif_batch_set_tuning to later batch calls, which ignore
 * bucket_shift and need tile >= 1.  nif_interpolate_noalloc follows the
 * mesh's settings with bucket_shift capped at 0 (its fixed scratch holds the
 * default bucket count).  Defaults: {8, 0, 8} for a mesh, {8, 0, 64} for a
 * batch.
 * Out-of-range values return NIF_ERR_ARG and change nothing. */
typedef struct {
    int32_t blocks_per_sm;
    int32_t bucket_shift;
    int32_t tile;
    int32_t reserved; /* 0 */
} nif_tuning;
int nif_dmesh_set_tuning(nif_dmesh *m, const nif_tuning *t);
int nif_dmesh_get_tuning(const nif_dmesh *m, nif_tuning *t);

/* Result summary of one query call (host memory). */
typedef struct {
    int64_t nnz;            /* non-zeros of the weight matrix */
    int64_t rows_large;     /* rows that needed the large-capacity kernel */
    int64_t rows_failed;    /* rows with a non-zero status (left empty) */
    int64_t rows_outside;   /* queries outside the super-simplex (empty rows) */
    int64_t walk_steps;     /* total point-location steps */
    int32_t first_status;   /* status of a failing row, NIF_OK if none */
    int32_t rows_wide;      /* rows whose cavity exceeded a split-row record
                             * and ran in the fused row kernel (speed only) */
    /* NIF_PRED_AUDIT / NIF_PRED_EXACT meshes, over the tests natinterp3d makes
     * for these rows: walk orientation tests and cavity in-sphere tests whose
     * fast value the error bound cannot certify, and those whose decision the
     * exact sign changes.  The walk counts depend on the walk's seed tet. */
    int64_t orient_uncertain;
    int64_t orient_flipped;
    int64_t insphere_uncertain;
    int64_t insphere_flipped;
} nif_summary;

/* Device workspace bytes for M queries in the given mode
 * (NIF_MODE_WEIGHTS or NIF_MODE_INTERP). */
int nif_query_workspace_bytes(const nif_dmesh *m, int64_t M, int mode, size_t *bytes);

/* Sibson weights, step 1 of 2.  Queries are M rows of 3 coordinates
 * (query_dtype NIF_F64 or NIF_F32, C order) in the caller's frame; the key
 * centroid is subtracted on the device in float64 exactly as
 * natinterp3d.py:115 does in numpy.  Computes every row into the workspace
 * and writes d_rowptr (int32[M+1]).  Synchronises `stream` and fills
 * *summary.  Returns NIF_ERR_OVERFLOW (d_rowptr untouched) when
 * nnz > INT32_MAX.  Replaces getInsertionFreeWeightsParallel
 * (natural_insertionfree.h:81-84) up to its row-pointer pass
 * (natural_insertionfree.c:896-913). */
int nif_weights_count(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                      const double centroid[3], void *d_ws, size_t ws_bytes, int32_t *d_rowptr,
                      void *stream, nif_summary *summary);

/* Sibson weights, step 2 of 2: writes the CSR arrays d_vals (vals_dtype,
 * nnz) and d_cols (int32, nnz) for the d_rowptr of step 1.  Takes the same
 * queries, dtype, M, centroid and workspace as nif_weights_count (the queries
 * must be unchanged in between).  Rows of up to 24 entries were staged by
 * step 1 and are copied; longer rows, and rows the large-capacity kernel
 * handled, are recomputed straight into their slices, so the workspace holds
 * no more than 24 entries a row and no row is limited by a staging arena.
 * Columns of a row appear in natinterp3d's first-seen order.  If
 * d_row_totals is not NULL it receives each row's normaliser (the sum of its
 * stolen volumes, 0 for empty rows; float64 [M]), which nif_query_grad takes
 * as input.  Replaces the CSR copy of natural_insertionfree.c:915-928
 * (natinterp3d mallocs vals/cols itself, and grows per-thread arenas while
 * it computes, natural_insertionfree.c:750). */
int nif_weights_fill(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                     const double centroid[3], const void *d_ws, size_t ws_bytes,
                     const int32_t *d_rowptr, void *d_vals, int vals_dtype, int32_t *d_cols,
                     double *d_row_totals, void *stream);

/* Row counters of the last nif_interpolate / nif_query_grad call that used
 * this workspace (for calls made with summary = NULL, which do not
 * synchronise).  Synchronises `stream`. */
int nif_query_summary(const nif_dmesh *m, int64_t M, int mode, const void *d_ws, size_t ws_bytes,
                      void *stream, nif_summary *summary);

/* Interpolation without materialising the weights: out[i, :] =
 * sum_k w_ik values[k, :] for every query, accumulated in row order exactly
 * as `get_weights(Q) @ values` (natinterp3d.py:131-137, scipy csr_matvecs)
 * with weights cast to the query dtype and the product in
 * out_dtype = promote(query_dtype, values_dtype).  values is [N][D] C order.
 * If summary is non-NULL the call synchronises `stream` and fills it. */
int nif_interpolate(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                    const double centroid[3], const void *d_values, int values_dtype, int D,
                    void *d_out, int out_dtype, void *d_ws, size_t ws_bytes, void *stream,
                    nif_summary *summary);

/* ---- differentiable path (no counterpart in natinterp3d) ----------------- */

/* y[M][D] = W x with W an M-row CSR (int32 row pointers and columns) and
 * x [N][D]: each y[i, d] accumulated from zero over the row's entries in
 * stored order, in the promoted type -- what scipy's `W @ x` computes
 * (natinterp3d.py:131-137).  y_dtype must be promote(vals_dtype, x_dtype). */
int nif_spmm(int64_t M, int64_t N, const int32_t *d_rowptr, const int32_t *d_cols,
             const void *d_vals, int vals_dtype, const void *d_x, int x_dtype, int D, void *d_y,
             int y_dtype, void *stream);

/* y[N][D] = W^T x for x [M][D]: the gradient of `W @ values` with respect to
 * values.  Deterministic: a CSC is built by a stable radix sort of the
 * columns (no floating-point atomics) and each y[k, d] is accumulated from
 * zero in ascending row order.  Workspace size from nif_spmm_t_workspace_bytes. */
int nif_spmm_t_workspace_bytes(int64_t M, int64_t N, int64_t nnz, size_t *bytes);
int nif_spmm_t(int64_t M, int64_t N, int64_t nnz, const int32_t *d_rowptr, const int32_t *d_cols,
               const void *d_vals, int vals_dtype, const void *d_x, int x_dtype, int D, void *d_y,
               int y_dtype, void *d_ws, size_t ws_bytes, void *stream);

/* The same product, the columns processed in the order d_key_rank gives
 * (d_key_rank[k] = position of column k; a permutation of 0..N-1, such as a
 * spatial order of the keys, so that neighbouring keys, whose rows overlap,
 * gather their x rows while they are still in L2).  Results are identical
 * bit for bit; a d_key_rank that is not a permutation gives unspecified
 * values but no out-of-range access.  Same workspace as nif_spmm_t. */
int nif_spmm_t_ordered(int64_t M, int64_t N, int64_t nnz, const int32_t *d_rowptr,
                       const int32_t *d_cols, const void *d_vals, int vals_dtype, const void *d_x,
                       int x_dtype, int D, void *d_y, int y_dtype, const int32_t *d_key_rank,
                       void *d_ws, size_t ws_bytes, void *stream);

/* Gradient of a loss through interpolation with respect to the query
 * positions: gq[i, :] = sum_k (gout[i, :] . values[k, :]) dw_ik/dq_i, from the
 * analytic derivative of every stolen volume (the virtual-tet terms of
 * natural_insertionfree.c:681-719; all other terms are locally constant).
 * Takes the forward pass's CSR (d_rowptr, float64 d_weights) and row
 * normalisers (nif_weights_fill's d_row_totals) and recomputes each query's
 * cavity, boundary and neighbour order instead of storing them.
 * gout_dtype = promote(query, values); gq has the query dtype; rows without
 * a derivative (empty, or exactly on a data site) get zero.
 * Workspace: nif_query_workspace_bytes(NIF_MODE_INTERP). */
int nif_query_grad(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                   const double centroid[3], const int32_t *d_rowptr, const double *d_weights,
                   const double *d_row_totals, const void *d_values, int values_dtype, int D,
                   const void *d_gout, int gout_dtype, void *d_gq, void *d_ws, size_t ws_bytes,
                   void *stream, nif_summary *summary);

/* The same gradient without recomputing point location and cavities: the
 * forward keeps every row's cavity record (its cavity tets in natinterp3d's
 * visiting order, their face-circumcentre choices and boundary faces;
 * 788 bytes a row, nif_records_bytes) by calling
 * nif_weights_count_records in place of nif_weights_count, then
 * nif_weights_fill as usual; nif_query_grad_records then takes that
 * workspace (unchanged since) and the records, for the same queries, M and
 * centroid.  Meshes with natinterp3d's fast predicates only (NIF_ERR_ARG
 * otherwise; nif_query_grad serves the other modes).  d_records must be
 * 256-byte aligned.  The results equal nif_query_grad's bit for bit.  The
 * summary counts the gradient's own passes except the large-row kernel's
 * (whose rows the forward's summary reported).  (natinterp3d has no
 * counterpart.) */
int nif_records_bytes(int64_t M, size_t *bytes);
int nif_weights_count_records(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                              const double centroid[3], void *d_ws, size_t ws_bytes,
                              int32_t *d_rowptr, void *d_records, size_t records_bytes,
                              void *stream, nif_summary *summary);
int nif_query_grad_records(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                           const double centroid[3], const int32_t *d_rowptr,
                           const double *d_weights, const double *d_row_totals,
                           const void *d_values, int values_dtype, int D, const void *d_gout,
                           int gout_dtype, void *d_gq, const void *d_ws, size_t ws_bytes,
                           void *d_records, size_t records_bytes, void *stream,
                           nif_summary *summary);

/* ---- batched problems (no counterpart in natinterp3d, which needs one
 * Interpolator and one query call per key set) ------------------------------
 * A batch groups P resident meshes (each from nif_dmesh_create, all on one
 * device); d_buf (nif_batch_bytes) receives their device views.  The mesh
 * handles must outlive the batch. */
typedef struct nif_dbatch nif_dbatch;
int nif_batch_bytes(int n_problems, size_t *bytes);
int nif_batch_create(int n_problems, nif_dmesh *const *meshes, void *d_buf, size_t buf_bytes,
                     void *stream, nif_dbatch **out);
void nif_batch_destroy(nif_dbatch *b);
int nif_batch_workspace_bytes(const nif_dbatch *b, int64_t total_queries, size_t *bytes);
/* Launch settings of later batch calls (nif_tuning above). */
int nif_batch_set_tuning(nif_dbatch *b, const nif_tuning *t);
int nif_batch_get_tuning(const nif_dbatch *b, nif_tuning *t);

/* Interpolation of every problem at once.  Queries [sum M_p][3] and values
 * [sum N_p][D] are concatenated by problem; d_query_offsets and
 * d_key_offsets (int64 [P+1], device) delimit them; d_centroids (float64
 * [P][3], device) holds each problem's key centroid.  out [sum M_p][D] gets,
 * per problem, exactly what nif_interpolate returns for that problem alone.
 * The call makes no host synchronisation and reads nothing from the host,
 * so a stream capture of it replays as one CUDA graph: bucketing by
 * (problem, Morton cell), one persistent row kernel whose warps take tiles
 * of queries (64 by default, nif_batch_set_tuning) from a device work
 * counter, then the large-row kernel.
 * Read the row counters afterwards with nif_batch_summary. */
int nif_batch_interpolate(const nif_dbatch *b, const void *d_queries, int query_dtype,
                          const int64_t *d_query_offsets, const double *d_centroids,
                          const void *d_values, int values_dtype, const int64_t *d_key_offsets, int D,
                          void *d_out, int out_dtype, int64_t total_queries, void *d_ws,
                          size_t ws_bytes, void *stream);
int nif_batch_summary(const nif_dbatch *b, int64_t total_queries, const void *d_ws, size_t ws_bytes,
                      void *stream, nif_summary *summary);

/* Measurement.  While enabled, every query call records CUDA events on its
 * stream between its phases (no host synchronisation); nif_profile_read
 * waits for the last complete call and returns the device time in
 * milliseconds of {query bucketing, shared-memory row kernel, large-row
 * kernel, CSR scan or epilogue}, averaged over the calls since the last
 * enable or read (at most the last 64).  (natinterp3d has no counterpart.)
 * nif_profile_kernels then returns, for the same calls, the device time in
 * milliseconds and the launches per call of each row kernel: {k_locate,
 * k_rows_cavity, k_rows_volume, k_rows_fast, k_rows_order} (events bracket
 * each launch, at most 48 a call). */
int nif_profile_enable(int on);
int nif_profile_read(double ms[4]);
int nif_profile_kernels(double ms[5], double launches[5]);

/* Measured FP64 throughput of the current device in TFLOP/s (2 flops per
 * multiply-add pair), with fused multiply-add and with separately rounded
 * multiply and add -- the latter is the ceiling for the query kernels, which
 * never fuse.  Allocates 8 bytes of device memory for its duration. */
int nif_measure_fp64_peak(double *tflops_fused, double *tflops_separate);

/* ---- interpolation without any device allocation ------------------------
 * No counterpart in natinterp3d.  For callers that cannot hand this library a
 * workspace or let it allocate one: a process whose device memory is already
 * owned by another pool (a serving framework that reserved the GPU up front),
 * or a latency-critical loop where a device allocation could fail or quietly
 * synchronise the whole device.
 *
 * Same contract and results as nif_interpolate, minus the workspace
 * arguments: the scratch lives in a fixed static device array of
 * NIF_NOALLOC_SCRATCH_BYTES inside libnif_cuda.so, which every GPU that loads
 * the library keeps until the process exits.  At most NIF_NOALLOC_MAX_QUERIES
 * queries per call; more return NIF_ERR_TOO_LARGE (split the batch).
 * The mesh's device must be current.  The first call on each device looks up
 * the array's device address (a CUDA runtime query, made once per device);
 * make that first call before any stream capture.  That address belongs to
 * the runtime's primary context of the device: call from that context (not a
 * context the caller created with the driver API), and not after a
 * cudaDeviceReset in the same process.  All calls share the one
 * array and each call re-initialises what must start at zero, so two calls
 * that can run on the GPU at the same time (different streams, or different
 * host threads) race on it: serialise them.  Allocates no device or host
 * memory.  If summary is non-NULL the call synchronises `stream`. */
#define NIF_NOALLOC_MAX_QUERIES (1 << 20)
#define NIF_NOALLOC_SCRATCH_BYTES (20u << 20)
int nif_interpolate_noalloc(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                            const double centroid[3], const void *d_values, int values_dtype, int D,
                            void *d_out, int out_dtype, void *stream, nif_summary *summary);

#ifdef __cplusplus
}
#endif

#endif /* NATINTERP3D_B200_H */
