/*
 * TEST INFRASTRUCTURE ONLY: a C-ABI harness around the reference's own
 * Merbit code, compiled by oracle/Makefile from the reference sources where
 * they lie (include path = <reference>/include) into oracle/_ref/.  It
 * contains no reference code; it only includes the reference header and
 * exposes, with plain pointers:
 *
 *   ref_merge_search   host call of merge_search<14>   include/utils.cuh:5-29
 *   ref_tile_dims      TILE ctor sizes                  include/tile.cuh:114-115
 *   ref_tile_build     Tile_Kernel<256,SIGMA> launch     include/tile.cuh:28-104,120-121
 *   ref_merbit_spmv    one merbit_kernel<V,256,14>      include/tile.cuh:476-561,596-601
 *                      launch after zeroing y and z, as Fun_Merbit does
 *                      before its loop (include/tile.cuh:597)
 *   ref_merbit_time[_sigma]  mean time of repeated launches (SIGMA 14, 20)
 *
 * Used by tests/ (GPU parity against the reference kernel), the golden
 * fixture script and bench.py's reference arm, and nothing else.
 */
#include "tile.cuh"

std::fstream FSTR;  // declared extern by the reference's inc.cuh

extern "C" {

int ref_merge_search(const int* offset, int nrow, int nnz, int diag, int* coord_x, int* coord_y) {
    merge_search<14>(offset, nrow, nnz, diag, *coord_x, *coord_y);
    return 0;
}

void ref_tile_dims(int nrow, int nnz, int sigma, int* tile_num, int* lane_num) {
    *lane_num = (nrow + nnz + sigma - 1) / sigma;
    *tile_num = (*lane_num + 31) / 32;
}

}  // extern "C"

template <unsigned SIGMA>
static int launch_tile(const int* offset, int nrow, int nnz, unsigned* tx, unsigned* ty, void* desc) {
    int tile_num, lane_num;
    ref_tile_dims(nrow, nnz, (int)SIGMA, &tile_num, &lane_num);
    int grid = (lane_num + 256) / 256;
    Tile_Kernel<256, SIGMA><<<grid, 256>>>(offset, nrow, nnz, tile_num, lane_num, tx, ty,
                                           (DescTypeT<SIGMA>*)desc);
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : (int)e;
}

extern "C" {

/* lane_desc must hold lane_num entries of 4 bytes (sigma < 15) or 8 bytes. */
int ref_tile_build(int sigma, const int* d_offset, int nrow, int nnz, unsigned* d_tile_x,
                   unsigned* d_tile_y, void* d_lane_desc) {
    switch (sigma) {
    case 7: return launch_tile<7>(d_offset, nrow, nnz, d_tile_x, d_tile_y, d_lane_desc);
    case 14: return launch_tile<14>(d_offset, nrow, nnz, d_tile_x, d_tile_y, d_lane_desc);
    case 20: return launch_tile<20>(d_offset, nrow, nnz, d_tile_x, d_tile_y, d_lane_desc);
    case 32: return launch_tile<32>(d_offset, nrow, nnz, d_tile_x, d_tile_y, d_lane_desc);
    default: return -1;
    }
}

/* y = alpha*A*x with the reference kernel at BLOCK=256, SIGMA=14, one launch.
 * dtype 0 = double, 1 = float.  d_colidx is the CSR column index array (the
 * reference calls it row_ind, include/tile.cuh:601). */
int ref_merbit_spmv(int dtype, const int* d_colidx, const void* d_vals, int nrow, int nnz,
                    const unsigned* d_tile_x, const unsigned* d_tile_y, const void* d_lane_desc,
                    double alpha, const void* d_x, void* d_y, void* d_z, void* stream) {
    int tile_num, lane_num;
    ref_tile_dims(nrow, nnz, 14, &tile_num, &lane_num);
    const int grid = (lane_num + 256 - 1) / 256;
    cudaStream_t s = (cudaStream_t)stream;
    size_t vs = dtype == 0 ? sizeof(double) : sizeof(float);
    cudaMemsetAsync(d_y, 0, vs * (size_t)nrow, s);
    cudaMemsetAsync(d_z, 0, vs * (size_t)nrow, s);
    if (dtype == 0)
        merbit_kernel<double, 256, 14><<<grid, 256, 0, s>>>(
            d_colidx, (const double*)d_vals, nrow, nnz, d_tile_x, d_tile_y,
            (const DescTypeT<14>*)d_lane_desc, tile_num, lane_num, alpha, (const double*)d_x,
            (double*)d_y, (double*)d_z);
    else
        merbit_kernel<float, 256, 14><<<grid, 256, 0, s>>>(
            d_colidx, (const float*)d_vals, nrow, nnz, d_tile_x, d_tile_y,
            (const DescTypeT<14>*)d_lane_desc, tile_num, lane_num, (float)alpha,
            (const float*)d_x, (float*)d_y, (float*)d_z);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"

template <unsigned SIGMA>
static float time_sigma(int dtype, const int* d_colidx, const void* d_vals, int nrow, int nnz,
                        const unsigned* d_tile_x, const unsigned* d_tile_y,
                        const void* d_lane_desc, const void* d_x, void* d_y, void* d_z, int reps,
                        cudaStream_t s) {
    int tile_num, lane_num;
    ref_tile_dims(nrow, nnz, (int)SIGMA, &tile_num, &lane_num);
    const int grid = (lane_num + 256 - 1) / 256;
    size_t vs = dtype == 0 ? sizeof(double) : sizeof(float);
    cudaMemsetAsync(d_y, 0, vs * (size_t)nrow, s);
    cudaMemsetAsync(d_z, 0, vs * (size_t)nrow, s);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
    for (int r = 0; r < reps; ++r) {
        if (dtype == 0)
            merbit_kernel<double, 256, SIGMA><<<grid, 256, 0, s>>>(
                d_colidx, (const double*)d_vals, nrow, nnz, d_tile_x, d_tile_y,
                (const DescTypeT<SIGMA>*)d_lane_desc, tile_num, lane_num, 1.0, (const double*)d_x,
                (double*)d_y, (double*)d_z);
        else
            merbit_kernel<float, 256, SIGMA><<<grid, 256, 0, s>>>(
                d_colidx, (const float*)d_vals, nrow, nnz, d_tile_x, d_tile_y,
                (const DescTypeT<SIGMA>*)d_lane_desc, tile_num, lane_num, 1.0f, (const float*)d_x,
                (float*)d_y, (float*)d_z);
        void* t = d_y;
        d_y = d_z;
        d_z = t;
    }
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return reps > 0 ? ms / reps : 0.f;
}

extern "C" {

/* Same kernel, launched `reps` times back to back on `stream` with the y/z
 * ping-pong of Fun_Merbit (include/tile.cuh:599-603); returns the mean
 * milliseconds per launch measured with CUDA events on that stream. */
float ref_merbit_time(int dtype, const int* d_colidx, const void* d_vals, int nrow, int nnz,
                      const unsigned* d_tile_x, const unsigned* d_tile_y, const void* d_lane_desc,
                      const void* d_x, void* d_y, void* d_z, int reps, void* stream) {
    return time_sigma<14>(dtype, d_colidx, d_vals, nrow, nnz, d_tile_x, d_tile_y, d_lane_desc,
                          d_x, d_y, d_z, reps, (cudaStream_t)stream);
}

/* As ref_merbit_time for SIGMA 14 or 20 (20: 64-bit lane descriptors,
 * include/tile.cuh:6-25); -1 for another SIGMA. */
float ref_merbit_time_sigma(int sigma, int dtype, const int* d_colidx, const void* d_vals,
                            int nrow, int nnz, const unsigned* d_tile_x, const unsigned* d_tile_y,
                            const void* d_lane_desc, const void* d_x, void* d_y, void* d_z,
                            int reps, void* stream) {
    if (sigma == 14)
        return time_sigma<14>(dtype, d_colidx, d_vals, nrow, nnz, d_tile_x, d_tile_y, d_lane_desc,
                              d_x, d_y, d_z, reps, (cudaStream_t)stream);
    if (sigma == 20)
        return time_sigma<20>(dtype, d_colidx, d_vals, nrow, nnz, d_tile_x, d_tile_y, d_lane_desc,
                              d_x, d_y, d_z, reps, (cudaStream_t)stream);
    return -1.f;
}

}  // extern "C"
