/*
 * merbit_b200: merge-path tiled CSR SpMV / SpMM for NVIDIA B200 (sm_100a).
 *
 * C ABI (plain pointers, sizes, int status).  All matrix, vector and
 * scratch pointers are DEVICE pointers on the current CUDA device unless
 * stated otherwise; `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  Every entry point returns a merbit_status.
 *
 * Reference interfaces replaced (paths relative to the MERBIT project root):
 *
 *   merbit_merge_coords   merge_search<SIGMA>            include/utils.cuh:5-29
 *   merbit_tile_dims      TILE<BLOCK,SIGMA> sizes         include/tile.cuh:114-115
 *   merbit_tile_build     TILE ctor + Tile_Kernel         include/tile.cuh:4-25,28-122
 *   merbit_plan_create    offset build + TILE in          include/tile.cuh:571-593
 *                         Fun_Merbit (sort is the caller's; see merbit_coo_to_csr)
 *   merbit_spmv           merbit_kernel launch            include/tile.cuh:476-561,596-603
 *                         (y = alpha*A*x; beta extends it)
 *   merbit_coo_sort       GRAPH::sort                     src/class.cu:143-177
 *   merbit_coo_to_csr     cusparseXcoo2csr in Fun_Merbit  include/tile.cuh:571-574
 *   merbit_outdegree_values  Fun_Values (loader weights)  src/class.cu:2-34
 *   merbit_pagerank_step  PARAMETER damping scaffold      include/class.cuh:119-157
 *
 * With no reference counterpart (same kernel family):
 *   merbit_spmm, merbit_batch_*   k right-hand sides; many matrices per launch
 *   merbit_plan_transpose + merbit_spmm, merbit_dval, merbit_spmm_dval
 *                         adjoints dX = A^T G and dval = G[row].X[col]
 *   merbit_plan_tune, merbit_plan_set_config   the configuration table
 *   merbit_spmv_noalloc   one SpMV that allocates nothing (+ _check, _selftest_wait)
 *   merbit_plan_check, merbit_plan_selftest_wait   device-side failure status
 *   merbit_release_cached_memory   empties the library's device memory pool
 *
 * Threading: a plan may be used from any host thread, but launches that use
 * the same plan must be ordered on the device (one stream, or ordered by
 * events): each plan owns device scratch (carry slots, a launch counter)
 * that every launch reuses.  The reference is single-stream as well
 * (include/tile.cuh:596-603).
 *
 * Devices: a plan lives on the device that was current at
 * merbit_plan_create, and its launches go to the calling thread's current
 * device, which must be that one (streams belong to a device too).
 * merbit_pagerank_step and merbit_plan_destroy switch to the plan's device
 * for the call and restore the caller's current device.
 */
#ifndef MERBIT_H
#define MERBIT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum merbit_status {
    MERBIT_OK = 0,
    MERBIT_ERR_INVALID = 1,     /* bad argument: null pointer, negative size, bad dtype/k/ld */
    MERBIT_ERR_MATRIX = 2,      /* row_ptr[0]!=0, row_ptr[nrow]!=nnz, decreasing row_ptr,
                                   or a column index outside [0,ncol) */
    MERBIT_ERR_OVERFLOW = 3,    /* nrow+nnz beyond the int32 merge-path range */
    MERBIT_ERR_CUDA = 4,        /* a CUDA runtime call failed: merbit_last_cuda_error() */
    MERBIT_ERR_TIMEOUT = 5,     /* a device-side carry wait ran out (bounded spin); the
                                   launch's output is invalid; reported by merbit_plan_check */
    MERBIT_ERR_UNSUPPORTED = 6  /* valid request the library does not implement */
} merbit_status;

typedef enum merbit_dtype {
    MERBIT_F64 = 0,  /* values f64; x, y f64; f64 accumulation (the plain form) */
    MERBIT_F32 = 1,  /* values f32; x, y f32; f32 two-sum accumulation, f64 carries */
    MERBIT_BF16 = 2  /* values bf16; x, y f32; f32 two-sum accumulation, f64 carries */
} merbit_dtype;

/* merbit_plan_create flags */
#define MERBIT_PLAN_SKIP_VALIDATE 0x1u /* trust row_ptr/col_idx (skips one pass + a sync) */
#define MERBIT_PLAN_NO_TUNE 0x2u       /* never time candidate configurations */

typedef struct merbit_plan_s* merbit_plan;

typedef struct merbit_plan_info {
    int32_t nrow, ncol, nnz;
    int32_t dtype;
    int32_t block;           /* threads per CTA of the SpMV kernel in use */
    int32_t items_per_thread;/* merge items per thread */
    int32_t tile_items;      /* merge items (row ends + nonzeros) per tile */
    int32_t num_tiles;
    int32_t vectorized;      /* 1 when 128-bit loads of col_idx/vals are used */
    int32_t kind;            /* 0: CTA-tile kernel, 1: warp-tile kernel, 3: row-group kernel */
    int32_t l1_carveout;     /* warp-tile kernel: preferred shared-memory carveout, percent
                                (0: driver default, all shared memory) */
    int32_t gather_l2_only;  /* 1: x gathers bypass L1 allocation (ld.global.cg) */
    int64_t metadata_bytes;  /* partition + carry scratch held by the plan */
    double algorithmic_bytes;/* compulsory bytes of one SpMV, y = A x */
    int32_t max_row_len;     /* longest row (nonzeros); part of the tuning signature */
} merbit_plan_info;

/* ---------------- reference-format partition (parity surface) ---------------- */

/* Merge-path coordinates at diagonals i*stride (clamped to nrow+nnz), i in
 * [0,count): d_coord_x[i] = nonzeros consumed, d_coord_y[i] = rows consumed.
 * Bit-identical to merge_search (include/utils.cuh:5-29), tie rule included. */
int merbit_merge_coords(const int32_t* d_row_ptr, int32_t nrow, int32_t nnz, int64_t stride,
                        int64_t count, int32_t* d_coord_x, int32_t* d_coord_y, void* stream);

/* TILE<BLOCK,SIGMA> sizes: lane_num = ceil((nrow+nnz)/sigma), tile_num =
 * ceil(lane_num/32) (include/tile.cuh:114-115). */
int merbit_tile_dims(int32_t nrow, int32_t nnz, int32_t sigma, int32_t* tile_num,
                     int32_t* lane_num);

/* The reference's Merbit plan, bit for bit (include/tile.cuh:28-104):
 * d_tile_x[tile_num+1], d_tile_y[tile_num+1] (MSB = "fast" tile with no row
 * end), d_lane_desc[lane_num] of 4-byte descriptors when sigma < 15 and
 * 8-byte ones otherwise.  1 <= sigma <= 42. */
int merbit_tile_build(const int32_t* d_row_ptr, int32_t nrow, int32_t nnz, int32_t sigma,
                      uint32_t* d_tile_x, uint32_t* d_tile_y, void* d_lane_desc, void* stream);

/* ---------------- plans: y = alpha*A*x + beta*y ---------------- */

/* Builds the partition and carry scratch for one CSR matrix (square or not).
 * The plan keeps the caller's device pointers (it copies nothing): they must
 * stay valid and unchanged in structure while the plan lives.  Validates the
 * structure unless MERBIT_PLAN_SKIP_VALIDATE.  Synchronizes `stream`. */
int merbit_plan_create(merbit_plan* plan, int32_t nrow, int32_t ncol, int32_t nnz,
                       const int32_t* d_row_ptr, const int32_t* d_col_idx, const void* d_vals,
                       merbit_dtype dtype, uint32_t flags, void* stream);
int merbit_plan_destroy(merbit_plan plan);
int merbit_plan_get_info(merbit_plan plan, merbit_plan_info* info);

/* Replace the value array (same structure, same dtype). */
int merbit_plan_set_values(merbit_plan plan, const void* d_vals);

/* Selects the SpMV kernel configuration by timing the candidates on this
 * matrix (`x`,`y` are scratch vectors of the plan's dtype, contents
 * overwritten): every usable configuration once (5 launches), then the
 * three fastest in three rounds of 10 launches, keeping the best time.  The
 * choice is cached per matrix signature for the process.  Not capturable
 * (it synchronizes). */
int merbit_plan_tune(merbit_plan plan, const void* d_x, void* d_y, void* stream);

/* Kernel configurations the tuner chooses from, for a dtype: kind 0 = CTA
 * tiles of block*items_per_thread merge items, kind 1 = warp tiles of
 * 32*items_per_thread items (needs 16-byte aligned row_ptr/col_idx/vals);
 * warp-tile entries also differ in the shared-memory / L1 split they launch
 * with and in the cache hint of the x gathers (merbit_plan_get_info).
 * kind 3 = row groups: items_per_thread lanes own one row (no merge-path
 * tiles; tile_items 0), for short, even rows such as stencils.
 * merbit_plan_set_config forces one (MERBIT_ERR_INVALID if the plan's
 * arrays do not allow it); it builds that tile size's partition on first
 * use, synchronizing `stream`. */
int merbit_num_configs(merbit_dtype dtype);
int merbit_config_desc(merbit_dtype dtype, int32_t idx, int32_t* kind, int32_t* block,
                       int32_t* items_per_thread);
int merbit_plan_set_config(merbit_plan plan, int32_t idx, void* stream);
/* *usable = 1 when configuration idx can run this plan (same rules). */
int merbit_plan_config_usable(merbit_plan plan, int32_t idx, int32_t* usable, void* stream);

/* y[nrow] = alpha*A*x[ncol] + beta*y.  beta == 0 never reads y. */
int merbit_spmv(merbit_plan plan, double alpha, const void* d_x, double beta, void* d_y,
                void* stream);

/* One PageRank power step in a single launch (the iteration PARAMETER's
 * damp / perrnd / maxiter scaffold, include/class.cuh:119-146; the residual
 * is RESULT::norm, include/class.cuh:157):
 *     y = damp * A x + (1 - damp) * teleport
 *     *d_residual = sum_i |y_i - x_i|   (L1, of y as stored; skipped if NULL)
 * The residual is reduced inside the SpMV launch -- per-CTA partials summed in
 * a fixed order by the launch's last CTA -- so it is deterministic and costs
 * no extra pass over y.  The plan must be square; x, teleport and y are
 * vectors of the plan's x/y type; y must not alias x (teleport may alias y).
 * A row without nonzeros gets only the teleport term; the rank of a node
 * without out-links is not redistributed (plain power step). */
int merbit_pagerank_step(merbit_plan plan, double damp, const void* d_x, const void* d_teleport,
                         void* d_y, double* d_residual, void* stream);

/* ---------------- harness front end ---------------- */

/* Sorts COO triplets in place by (major, minor) -- GRAPH::sort
 * (src/class.cu:143-177): sort(false) orders by (col, row), i.e. major =
 * col_ind.  Stable and deterministic.  d_vals may be NULL.  Synchronizes. */
int merbit_coo_sort(int32_t nnz, int32_t* d_major, int32_t* d_minor, void* d_vals,
                    merbit_dtype dtype, void* stream);
/* row_ptr[nrow+1] of sorted row indices -- cusparseXcoo2csr as used in
 * include/tile.cuh:574 (zero-based). */
int merbit_coo_to_csr(int32_t nnz, const int32_t* d_sorted_rows, int32_t nrow, int32_t* d_row_ptr,
                      void* stream);
/* values[e] = 1 / #{e' : row_ind[e'] == row_ind[e]} -- the PageRank weights
 * the reference loader writes over a Matrix Market file's values
 * (Fun_Values, src/class.cu:2-34).  Synchronizes. */
int merbit_outdegree_values(int32_t nnz, int32_t nrow, const int32_t* d_row_ind, void* d_vals,
                            merbit_dtype dtype, void* stream);

/* ---------------- adjoint (differentiation) ---------------- */

/* Builds the plan of A^T (ncol x nrow) from a plan of A: a stable sort of
 * the column indices (so every A^T row keeps A's row order and dX sums are
 * taken in a fixed order), the transposed structure and a gathered copy of
 * the values, all owned by the new plan.  dX = A^T G is then
 * merbit_spmm(tplan, ...).  The source plan must outlive nothing here: the
 * transpose owns its arrays.  Synchronizes. */
int merbit_plan_transpose(merbit_plan plan, merbit_plan* tplan, void* stream);
/* Re-gathers the transpose's values after A's values changed (same
 * structure): d_src_vals is A's value array. */
int merbit_plan_transpose_refresh(merbit_plan tplan, const void* d_src_vals, void* stream);
/* Gradient of the values: dval[e] = sum_{j<k} G[row_e, j] * X[col_e, j]
 * (row-major G [nrow x ldg], X [ncol x ldx]; dval in the x/y type: f64 for
 * f64 plans, f32 otherwise).  Each sum in a fixed order, no atomics.  The
 * first call builds the plan's nonzero-to-row map (allocates). */
int merbit_dval(merbit_plan plan, int32_t k, const void* d_g, int64_t ldg, const void* d_x,
                int64_t ldx, void* d_dval, void* stream);

/* The whole backward of Y = A X in one launch, on the transpose plan tplan
 * of A (merbit_plan_transpose): dX = A^T G (dX [ncol x lddx], overwritten)
 * and, from the G rows that product gathers anyway, dval[e] =
 * sum_{j<k} G[row_e, j] * X[col_e, j] for every nonzero e of A (in A's
 * nonzero order).  k = 1, 2, 4, 8, 16 or 32; F64 and F32 values.
 * MERBIT_ERR_UNSUPPORTED otherwise: use merbit_spmm + merbit_dval then.
 * Sums in a fixed order, no atomics. */
int merbit_spmm_dval(merbit_plan tplan, int32_t k, const void* d_g, int64_t ldg, const void* d_x,
                     int64_t ldx, void* d_dx, int64_t lddx, void* d_dval, void* stream);

/* ---------------- k right-hand sides and batches ---------------- */

/* Y[nrow x k] = alpha*A*X[ncol x k] + beta*Y, row-major with leading
 * dimensions ldx, ldy >= k (elements).  Any k >= 1 (processed in
 * power-of-two column blocks of at most 32).  The first call for a given
 * block width allocates that width's carry slots (synchronizes); later
 * calls allocate nothing and can be captured in a CUDA graph. */
int merbit_spmm(merbit_plan plan, int32_t k, double alpha, const void* d_x, int64_t ldx,
                double beta, void* d_y, int64_t ldy, void* stream);

typedef struct merbit_batch_s* merbit_batch;

typedef struct merbit_batch_info {
    int32_t count, k, dtype;
    int32_t tile_items;    /* merge items per warp tile (kernel 0; per matrix for kernel 1) */
    int32_t vector_width;  /* RHS values per lane */
    int32_t total_tiles;
    int64_t nnz;
    double algorithmic_bytes; /* sum over matrices of one SpMM's compulsory bytes */
    int32_t kernel;        /* 0: SpMM kernel (lane groups); 1: warp-tile kernel (k = 1) */
    int32_t variant;       /* kernel 1: 0 L1 gathers, all shared memory; 1 L1 gathers with a
                              72% shared-memory carveout; 2 L2-only gathers, 72% carveout;
                              5 L1 gathers, 58% carveout (these take 7, 11 or 15 items per
                              lane); 3 and 4 as 0 and 1 with stages for 15, 19 or 23 items
                              per lane; 6 and 7 as 5 and 1 with stages for 7 or 11; 8 as 6
                              with a 44% carveout; 9 as 6 with CTAs of 4 warps */
} merbit_batch_info;

/* A batch of `count` plans (same dtype) multiplied by k in {1,2,4,8,16,32}
 * right-hand sides in ONE persistent launch.  The X/Y device buffers of
 * each matrix are bound at creation (callers refill them between runs);
 * plans and buffers must outlive the batch.  Untuned, it starts from the
 * configurations that won on a 128-matrix R-MAT batch: at k = 1 the
 * warp-tile kernel (variant 6, or the cached choices of the members'
 * signatures), at k = 2 352-item staged-product tiles, at k >= 4 the odd
 * tile of k at vector width 4 (where the operands allow them).
 * Synchronizes. */
int merbit_batch_create(merbit_batch* batch, int32_t count, const merbit_plan* plans, int32_t k,
                        const void* const* d_x, const int64_t* ldx, void* const* d_y,
                        const int64_t* ldy, void* stream);
/* Y_i = alpha*A_i*X_i + beta*Y_i for every matrix of the batch: one kernel
 * launch, no allocation, no synchronization (capturable in a CUDA graph). */
int merbit_batch_spmm(merbit_batch batch, double alpha, double beta, void* stream);
/* The batch autotuner.  Times the SpMM kernel at each tile size and RHS
 * vector width and, for k = 1 on 16-byte aligned arrays, the warp-tile
 * kernel in each variant (3 launches each, then the three fastest again in
 * two rounds of 8); with the warp-tile kernel it then chooses the
 * items per lane (7, 11, 15, 19 or 23, as the variant takes) per matrix
 * signature class (mean row length and longest-row skew), largest classes
 * first, keeping whatever times fastest for the whole launch; the choices
 * are cached per matrix signature.  With the SpMM kernel at vector width 4
 * it chooses in the same way, per class, between the two tile sizes of the
 * winning size's pair (merbit_batch_set_matrix_tile).  Synchronizes. */
int merbit_batch_tune(merbit_batch batch, void* stream);
int merbit_batch_get_info(merbit_batch batch, merbit_batch_info* info);
/* The configuration of matrix `index` of the batch (the reference fixes one
 * VBLOCK/VSIGMA per build, CMakeLists.txt:4-6,22-25): the kernel (as in
 * merbit_batch_info), its merge items per tile and items per lane.  With
 * the warp-tile kernel (k = 1) each matrix has its own tile size, chosen by
 * merbit_batch_tune per matrix signature class and cached per signature
 * for later batches and plans of the process; with the SpMM kernel each
 * matrix takes one of a pair of tile sizes (merbit_batch_set_matrix_tile). */
int merbit_batch_get_matrix_config(merbit_batch batch, int32_t index, int32_t* kernel,
                                   int32_t* tile_items, int32_t* items_per_thread);
/* Selects the batch's kernel by hand (as merbit_plan_set_config does for a
 * plan): kernel 0, the SpMM kernel with `option` merge items per tile (256
 * or 512; with vector width 4 also tiles of an odd number of items per lane
 * group: 288/480 for k = 1 or 4, 272/496 for k = 8, 264/504 for k = 16,
 * 260/508 for k = 32; widest legal vector width); kernel 1, the warp-tile kernel (k = 1,
 * 16-byte aligned arrays) in variant `option` (0-9, see merbit_batch_info).
 * Synchronizes. */
int merbit_batch_set_kernel(merbit_batch batch, int32_t kernel, int32_t option, void* stream);
/* Sets the items per lane of matrix `index` -- one the kernel variant in use
 * takes (see merbit_batch_info) -- and
 * switches the batch to the warp-tile kernel (k = 1 and 16-byte aligned
 * arrays only, else MERBIT_ERR_UNSUPPORTED).  Synchronizes. */
int merbit_batch_set_matrix_config(merbit_batch batch, int32_t index, int32_t items_per_thread,
                                   void* stream);
/* Sets the merge items per tile of matrix `index` on the SpMM kernel (kernel
 * 0, vector width 4, k = 4, 8, 16 or 32): the other tile of the pair the
 * batch's tile size belongs to (256/512, or the two odd tiles of k).  One
 * launch then runs matrices of both tile sizes; merbit_batch_tune chooses
 * them per matrix signature class.  Synchronizes. */
int merbit_batch_set_matrix_tile(merbit_batch batch, int32_t index, int32_t tile_items,
                                 void* stream);
int merbit_batch_destroy(merbit_batch batch);

/* y[nrow] = alpha*A*x + beta*y without allocating any device memory -- for
 * callers that cannot allocate on the call path: hosts whose device memory
 * all belongs to their own pool allocator (a framework's caching allocator
 * that must not see a library take memory behind its back), and loops that
 * cannot afford cudaMalloc's implicit synchronization.  No counterpart in
 * the reference.
 *
 * Its scratch (tile coordinates, carry slots, launch counters) is one fixed
 * file-scope device array of about 1.3 MB, held by every GPU that loads the
 * library until the process exits.  It bounds the matrix: nrow + nnz <=
 * 58,720,256 (32,768 tiles of 1,792 merge items); larger matrices are
 * rejected with MERBIT_ERR_INVALID -- use merbit_plan_create/merbit_spmv.
 * The caller passes all arrays (device pointers, same dtype rules as a
 * plan).  The structure is not validated: it must be valid CSR.  The first
 * call on a device looks the array up, initializes it on `stream` and
 * waits for that; make that first call before any stream capture (under
 * capture it is refused with MERBIT_ERR_INVALID).  Every call reuses the
 * same array (each call rebuilds what it needs), so calls whose executions
 * overlap on the GPU -- on different streams without ordering -- race.
 * A device-side wait that runs out is recorded, not returned (the call
 * returns before the kernel runs): merbit_spmv_noalloc_check reports it,
 * and it never carries over into the results of later calls. */
int merbit_spmv_noalloc(int32_t nrow, int32_t ncol, int32_t nnz, const int32_t* d_row_ptr,
                        const int32_t* d_col_idx, const void* d_vals, merbit_dtype dtype,
                        double alpha, const void* d_x, double beta, void* d_y, void* stream);

/* Device-side status of merbit_spmv_noalloc on the current device
 * (MERBIT_ERR_TIMEOUT if a wait ran out in any call since the last check);
 * reads and clears it on `stream`, allocates nothing, synchronizes `stream`.
 * No counterpart in the reference. */
int merbit_spmv_noalloc_check(void* stream);

/* Failure-detection self-test of merbit_spmv_noalloc's scratch (no reference
 * counterpart): as merbit_plan_selftest_wait, but the time-out is recorded
 * in the no-allocation scratch of the current device, where
 * merbit_spmv_noalloc_check reports it. */
int merbit_spmv_noalloc_selftest_wait(int32_t which, int32_t wait_us, void* stream);

/* Reads and clears the plan's device-side status (MERBIT_ERR_TIMEOUT if a
 * carry wait ran out in any launch since the last check).  Synchronizes. */
int merbit_plan_check(merbit_plan plan, void* stream);

/* Failure-detection self-test (no reference counterpart): runs one bounded
 * device wait of the kind the kernels use -- which = 0 the cross-CTA carry
 * wait, 1 the shared-memory mbarrier wait of the staged copies -- on a flag
 * that nothing sets, with a limit of wait_us microseconds (1 .. 1e6).  The
 * wait runs out, records MERBIT_ERR_TIMEOUT in the plan's device status and
 * returns; merbit_plan_check then reports it.  No fault, trap or hang. */
int merbit_plan_selftest_wait(merbit_plan plan, int32_t which, int32_t wait_us, void* stream);

/* Device memory (no reference counterpart).  Every buffer the library
 * allocates comes from its own stream-ordered pool on each device, which
 * keeps up to 64 MiB of released blocks mapped so that plans can be built
 * and destroyed cheaply.  This call synchronizes the current device and
 * returns every released block of its pool to the device (blocks of live
 * plans stay). */
int merbit_release_cached_memory(void);

/* ---------------- errors ---------------- */

const char* merbit_status_string(int status);
/* Last cudaError_t seen by this thread inside the library (0 if none). */
int merbit_last_cuda_error(void);
/* Human-readable detail of this thread's last failure ("" if none). */
const char* merbit_last_error_detail(void);

#ifdef __cplusplus
}
#endif

#endif /* MERBIT_H */
