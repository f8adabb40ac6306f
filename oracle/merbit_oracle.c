/*
 * CPU oracle for the Merbit merge-path CSR SpMV path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (merbit_b200/, include/)
 * links or calls this file; tests/, the smoke check and bench.py's CPU
 * baseline leg use it as the checker and as the timed CPU restatement.
 *
 * What it restates, with the reference file:line each function follows
 * (paths relative to the MERBIT project root):
 *
 *   orc_merge_search   include/utils.cuh:5-29      diagonal search, tie rule
 *                                                   offset[mid+1] <= d-mid-1
 *   orc_tile_plan      include/tile.cuh:28-122     Tile_Kernel + TILE ctor:
 *                                                   tile_x / tile_y (MSB=fast)
 *                                                   / lane_desc bit packing
 *   orc_spmm           include/tile.cuh:476-561    y = alpha*A*X (merbit_kernel
 *                                                   computes alpha*A*x); here
 *                                                   in extended precision with
 *                                                   Neumaier summation
 *   orc_spmm_t         (adjoint of the above)       dX = A^T G
 *   orc_dval           (adjoint of the above)       dval[e] = G[row]·X[col]
 *   orc_spmv_omp_f64   include/utils.cuh:5-29 +     merge-path partitioned
 *                      include/tile.cuh:476-561     OpenMP FP64 SpMV: the CPU
 *                                                   restatement timed as the
 *                                                   reference's CPU baseline
 *                                                   (the reference ships no
 *                                                   CPU SpMV of its own)
 *
 * Parity pin: orc_merge_search is checked against the reference's own
 * host-callable merge_search (compiled from the reference sources by
 * oracle/Makefile into oracle/_ref/), and orc_tile_plan / orc_spmm against
 * fixtures produced by the reference Tile_Kernel / merbit_kernel run on a
 * B200 (tests/golden/make_golden.py).
 *
 * Value types: 0 = f64, 1 = f32, 2 = bf16 (raw uint16 bits).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { ORC_F64 = 0, ORC_F32 = 1, ORC_BF16 = 2 };

static inline long double orc_load(int type, const void* p, int64_t i) {
    switch (type) {
    case ORC_F64: return (long double)((const double*)p)[i];
    case ORC_F32: return (long double)((const float*)p)[i];
    default: {
        uint32_t bits = ((uint32_t)((const uint16_t*)p)[i]) << 16;
        float f;
        memcpy(&f, &bits, 4);
        return (long double)f;
    }
    }
}

/* include/utils.cuh:5-29.  Search range [max(d-nnz,0), min(d,nrow)];
 * go right when offset[mid+1] <= d-mid-1, so a row end at the same
 * position as a nonzero is consumed first; coord_y is clamped to nrow. */
void orc_merge_search(const int32_t* offset, int64_t nrow, int64_t nnz, int64_t diag,
                      int64_t* coord_x, int64_t* coord_y) {
    int64_t lo = diag - nnz > 0 ? diag - nnz : 0;
    int64_t hi = diag < nrow ? diag : nrow;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if ((int64_t)offset[mid + 1] <= diag - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    *coord_x = diag - lo;
    *coord_y = lo < nrow ? lo : nrow;
}

/* Coordinates at diagonals i*stride (clamped to nrow+nnz), i in [0,count). */
void orc_merge_coords(const int32_t* offset, int64_t nrow, int64_t nnz, int64_t stride,
                      int64_t count, int32_t* out_x, int32_t* out_y) {
    int64_t total = nrow + nnz;
    for (int64_t i = 0; i < count; ++i) {
        int64_t d = i * stride;
        if (d > total) d = total;
        int64_t cx, cy;
        orc_merge_search(offset, nrow, nnz, d, &cx, &cy);
        out_x[i] = (int32_t)cx;
        out_y[i] = (int32_t)cy;
    }
}

/* include/tile.cuh:114-115 */
void orc_tile_dims(int64_t nrow, int64_t nnz, int sigma, int64_t* tile_num, int64_t* lane_num) {
    *lane_num = (nrow + nnz + sigma - 1) / sigma;
    *tile_num = (*lane_num + 31) / 32;
}

/* include/tile.cuh:28-104.  One "lane" per sigma merge items, 32 lanes per
 * tile.  Each lane: merge search at gid*sigma, walk lane_nnz items setting
 * bit idx for each row end, pack (bitflag<<d1)|(dy<<d2)|dx relative to the
 * tile's first lane; d1/d2 = 18/9 for a 32-bit descriptor (sigma<15) and
 * 22/11 for a 64-bit one.  The tile's y gets MSB set when no lane's walk
 * ended on a row other than the tile's first row.  Sentinel at [tile_num].
 * lane_desc is written widened to 64 bits; a 32-bit descriptor is the low
 * half. */
void orc_tile_plan(const int32_t* offset, int64_t nrow, int64_t nnz, int sigma,
                   uint32_t* tile_x, uint32_t* tile_y, uint64_t* lane_desc) {
    int64_t tile_num, lane_num;
    orc_tile_dims(nrow, nnz, sigma, &tile_num, &lane_num);
    const int wide = sigma >= 15;
    const int d1 = wide ? 22 : 18;
    const int d2 = wide ? 11 : 9;
    const uint64_t desc_mask = wide ? ~0ull : 0xFFFFFFFFull;
    for (int64_t t = 0; t < tile_num; ++t) {
        int64_t wx = 0, wy = 0;
        int all_same = 1;
        for (int l = 0; l < 32; ++l) {
            int64_t gid = t * 32 + l;
            if (gid >= lane_num) break;
            int64_t cx, cy;
            orc_merge_search(offset, nrow, nnz, gid * sigma, &cx, &cy);
            if (l == 0) {
                wx = cx;
                wy = cy;
            }
            int64_t lane_nnz = ((gid + 1) * sigma < nnz + nrow) ? sigma : (nnz + nrow - gid * sigma);
            uint64_t dx = (uint64_t)(cx - wx), dy = (uint64_t)(cy - wy), bits = 0;
            for (int64_t idx = 0; idx < lane_nnz; ++idx) {
                if (cx < offset[cy + 1]) {
                    ++cx;
                } else {
                    bits |= 1ull << idx;
                    ++cy;
                }
            }
            lane_desc[gid] = ((bits << d1) | (dy << d2) | dx) & desc_mask;
            if (cy != wy) all_same = 0;
        }
        tile_x[t] = (uint32_t)wx;
        tile_y[t] = (uint32_t)wy | (all_same ? 0x80000000u : 0u);
    }
    tile_x[tile_num] = (uint32_t)nnz;
    tile_y[tile_num] = (uint32_t)nrow;
}

/* Neumaier-compensated accumulation in long double. */
typedef struct {
    long double s, c;
} orc_acc;

static inline void orc_add(orc_acc* a, long double v) {
    long double t = a->s + v;
    if (fabsl(a->s) >= fabsl(v))
        a->c += (a->s - t) + v;
    else
        a->c += (v - t) + a->s;
    a->s = t;
}

/* Y[i, j] = alpha * sum_k A[i,k] X[col_k, j] for j < k_rhs (row-major X with
 * leading dimension ldx, row-major Y with ldy), products in long double and
 * compensated sums: the extended-precision reference that every GPU result
 * is compared with.  yabs (optional) receives sum_k |A[i,k] X[col_k,j]|, the
 * denominator of the component-wise relative error. */
void orc_spmm(int64_t nrow, const int32_t* row_ptr, const int32_t* col, int val_type,
              const void* vals, int x_type, const void* x, int64_t k_rhs, int64_t ldx,
              double alpha, double* y, double* yabs, int64_t ldy) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nrow; ++i) {
        for (int64_t j = 0; j < k_rhs; ++j) {
            orc_acc a = {0.0L, 0.0L};
            long double aa = 0.0L;
            for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
                long double p = orc_load(val_type, vals, e) *
                                orc_load(x_type, x, (int64_t)col[e] * ldx + j);
                orc_add(&a, p);
                aa += fabsl(p);
            }
            y[i * ldy + j] = (double)((long double)alpha * (a.s + a.c));
            if (yabs) yabs[i * ldy + j] = (double)(fabsl((long double)alpha) * aa);
        }
    }
}

/* dX[c, j] = sum over entries e with col_e = c of A_e * G[row_e, j].
 * Serial over entries per column bucket (columns gathered by a counting
 * pass), long double with compensation. */
void orc_spmm_t(int64_t nrow, int64_t ncol, const int32_t* row_ptr, const int32_t* col,
                int val_type, const void* vals, int g_type, const void* g, int64_t k_rhs,
                int64_t ldg, double* dx, int64_t lddx) {
    int64_t nnz = row_ptr[nrow];
    int64_t* cnt = (int64_t*)calloc((size_t)ncol + 1, sizeof(int64_t));
    int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
    int64_t* rowof = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz > 0 ? nnz : 1));
    for (int64_t i = 0; i < nrow; ++i)
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
            cnt[col[e] + 1]++;
            rowof[e] = i;
        }
    for (int64_t c = 0; c < ncol; ++c) cnt[c + 1] += cnt[c];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ncol > 0 ? ncol : 1));
    for (int64_t c = 0; c < ncol; ++c) fill[c] = cnt[c];
    for (int64_t e = 0; e < nnz; ++e) pos[fill[col[e]]++] = e;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t c = 0; c < ncol; ++c) {
        for (int64_t j = 0; j < k_rhs; ++j) {
            orc_acc a = {0.0L, 0.0L};
            for (int64_t q = cnt[c]; q < cnt[c + 1]; ++q) {
                int64_t e = pos[q];
                orc_add(&a, orc_load(val_type, vals, e) * orc_load(g_type, g, rowof[e] * ldg + j));
            }
            dx[c * lddx + j] = (double)(a.s + a.c);
        }
    }
    free(cnt);
    free(pos);
    free(rowof);
    free(fill);
}

/* dval[e] = sum_j G[row_e, j] * X[col_e, j]. */
void orc_dval(int64_t nrow, const int32_t* row_ptr, const int32_t* col, int g_type, const void* g,
              int64_t ldg, int x_type, const void* x, int64_t ldx, int64_t k_rhs, double* dval) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nrow; ++i)
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
            orc_acc a = {0.0L, 0.0L};
            for (int64_t j = 0; j < k_rhs; ++j)
                orc_add(&a, orc_load(g_type, g, i * ldg + j) *
                                orc_load(x_type, x, (int64_t)col[e] * ldx + j));
            dval[e] = (double)(a.s + a.c);
        }
}

/* Merge-path partitioned OpenMP FP64 SpMV, y = A x.  The merge path over
 * (row ends x nonzeros) is cut into nthreads equal diagonal ranges with
 * orc_merge_search; each thread walks its range exactly as the reference's
 * lanes walk theirs (include/tile.cuh:71-82: consume a nonzero while
 * x < offset[y+1], else a row end), writing the rows it completes and
 * leaving the partial first/last rows as carries that a serial pass adds.
 * Plain double accumulation: this is the speed baseline, not the accuracy
 * reference.  Returns the number of threads used. */
int orc_spmv_omp_f64(int64_t nrow, const int32_t* row_ptr, const int32_t* col,
                     const double* vals, const double* x, double* y, int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    int64_t nnz = row_ptr[nrow];
    int64_t total = nrow + nnz;
    int64_t* carry_row = (int64_t*)malloc(sizeof(int64_t) * (size_t)nthreads);
    double* carry_val = (double*)malloc(sizeof(double) * (size_t)nthreads);
#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
        int tid = omp_get_thread_num();
        int nt = omp_get_num_threads();
#else
        int tid = 0, nt = 1;
#endif
        int64_t per = (total + nt - 1) / nt;
        int64_t d0 = (int64_t)tid * per < total ? (int64_t)tid * per : total;
        int64_t d1 = d0 + per < total ? d0 + per : total;
        int64_t xs, ys, xe, ye;
        orc_merge_search(row_ptr, nrow, nnz, d0, &xs, &ys);
        orc_merge_search(row_ptr, nrow, nnz, d1, &xe, &ye);
        double acc = 0.0;
        int64_t cx = xs;
        for (int64_t r = ys; r < ye; ++r) {
            int64_t end = row_ptr[r + 1];
            for (; cx < end; ++cx) acc += vals[cx] * x[col[cx]];
            y[r] = acc;
            acc = 0.0;
        }
        for (; cx < xe; ++cx) acc += vals[cx] * x[col[cx]];
        carry_row[tid] = ye;
        carry_val[tid] = acc;
    }
    for (int t = 0; t < nthreads - 1; ++t)
        if (carry_row[t] < nrow) y[carry_row[t]] += carry_val[t];
    free(carry_row);
    free(carry_val);
    return nthreads;
}

/* yabs[i] = sum_k |A[i,k]| |x[col_k]| in double, row-parallel: the
 * denominator of the component-wise error for large matrices, where the
 * extended-precision orc_spmm would take seconds.  Returns the threads used. */
int orc_spmv_abs_omp_f64(int64_t nrow, const int32_t* row_ptr, const int32_t* col,
                         const double* vals, const double* x, double* yabs, int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads)
    for (int64_t i = 0; i < nrow; ++i) {
        double a = 0.0;
        for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) a += fabs(vals[e]) * fabs(x[col[e]]);
        yabs[i] = a;
    }
    return nthreads;
}

/* Row-parallel OpenMP CSR SpMM in float (values f32, X/Y f32 row-major,
 * k columns, double accumulation per output): the CPU baseline of the
 * batched form.  Returns the number of threads used. */
int orc_spmm_omp_f32(int64_t nrow, const int32_t* row_ptr, const int32_t* col,
                     const float* vals, const float* x, int64_t k, float* y, int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads)
    for (int64_t i = 0; i < nrow; ++i) {
        double acc[64];
        for (int64_t j0 = 0; j0 < k; j0 += 64) {
            const int64_t kk = k - j0 < 64 ? k - j0 : 64;
            for (int64_t j = 0; j < kk; ++j) acc[j] = 0.0;
            for (int64_t e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
                const double a = vals[e];
                const float* xr = x + (int64_t)col[e] * k + j0;
                for (int64_t j = 0; j < kk; ++j) acc[j] += a * xr[j];
            }
            for (int64_t j = 0; j < kk; ++j) y[i * k + j0 + j] = (float)acc[j];
        }
    }
    return nthreads;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
