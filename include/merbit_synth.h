/*
 * Seeded synthetic CSR generators: the matrices the Merbit harness's
 * main.cu (src/main.cu:3-84) read from Matrix Market files are not
 * available, so the bench and tests build these instead.  Host code only,
 * OpenMP-parallel, and reproducible independently of the thread count: every
 * row (or edge) draws from its own counter-based stream (SplitMix64 mixing of
 * seed, stream tag and index).
 *
 * All functions return 0 on success, a negative value on invalid input
 * (or the nonzero count, for the *_rowptr / rmat sizing functions).
 * Arrays are caller-allocated; CSR rows come out with sorted, unique
 * column indices.
 */
#ifndef MERBIT_SYNTH_H
#define MERBIT_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 5-point Laplacian on an nx*ny grid, natural (row-major) ordering,
 * diagonal 4, off-diagonals -1.  row_ptr[nx*ny+1], col/vals[5*n-2*nx-2*ny]. */
int merbit_synth_laplace2d(int64_t nx, int64_t ny, int32_t* row_ptr, int32_t* col, double* vals);

/* 27-point stencil on nx*ny*nz, off-diagonals N(0,1) (stream `seed`),
 * diagonal = sum|off| + 1.  nnz = (3nx-2)(3ny-2)(3nz-2). */
int64_t merbit_synth_stencil27_nnz(int64_t nx, int64_t ny, int64_t nz);
int merbit_synth_stencil27(int64_t nx, int64_t ny, int64_t nz, uint64_t seed, int32_t* row_ptr,
                           int32_t* col, double* vals);

/* Power-law rows: length L ~ Zipf(s) on {1..cap} (capped at ncol), each row
 * empty with probability empty_frac.  Pass 1 fills row_ptr[nrow+1] and
 * returns nnz (-1 if it would not fit int32).  Pass 2 draws L unique
 * uniform columns in [0,ncol), sorted, and N(0,1) values. */
int64_t merbit_synth_zipf_rowptr(int64_t nrow, int64_t ncol, double s, int64_t cap,
                                 double empty_frac, uint64_t seed, int32_t* row_ptr);
int merbit_synth_zipf_fill(int64_t nrow, int64_t ncol, uint64_t seed, const int32_t* row_ptr,
                           int32_t* col, double* vals);

/* R-MAT (a, b, c, d = 1-a-b-c) square n*n matrix: nedges edges drawn at
 * scale ceil(log2 n), indices >= n rejected (redrawn), duplicates removed.
 * col/vals must hold nedges entries; returns the realised nnz.  Values
 * N(0,1). */
int64_t merbit_synth_rmat(int64_t n, int64_t nedges, double a, double b, double c, uint64_t seed,
                          int32_t* row_ptr, int32_t* col, double* vals);

/* Dense vectors: U[lo,hi) and N(0,1) from stream (seed, tag). */
int merbit_synth_uniform(uint64_t seed, uint64_t tag, int64_t n, double lo, double hi, double* out);
int merbit_synth_normal(uint64_t seed, uint64_t tag, int64_t n, double* out);

#ifdef __cplusplus
}
#endif

#endif /* MERBIT_SYNTH_H */
