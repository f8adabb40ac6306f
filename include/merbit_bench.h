/* Measurement support for merbit_b200 (not part of the SpMV interface, and
 * with no counterpart in the reference).
 *
 * merbit_bench_gather: sum of x[idx[i]] over i < n (n a multiple of 8 is
 * covered fully), split over 2048 * SM-count threads that each keep 8
 * gathers in flight; out[t] receives thread t's sum.  Indices outside
 * [0, nx) read x[0]; idx must be 16-byte aligned and out must hold at least
 * 2048 * SM-count doubles.  Timing one launch gives the
 * GPU's random-gather rate, the ceiling of an SpMV whose column indices are
 * random (one L1 miss per nonzero).  Does not synchronize. */
#ifndef MERBIT_BENCH_H
#define MERBIT_BENCH_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
int merbit_bench_gather(const double* d_x, int32_t nx, const int32_t* d_idx, int64_t n,
                        double* d_out, int32_t out_len, void* stream);
#ifdef __cplusplus
}
#endif
#endif
