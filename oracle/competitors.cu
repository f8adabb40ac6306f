/*
 * TEST INFRASTRUCTURE ONLY: a C-ABI harness around the SpMV libraries the
 * reference benchmarks Merbit against (src/spmv.cu), compiled by
 * oracle/Makefile from the reference's vendored headers where they lie
 * (include path = <reference>/include) into oracle/_ref/.  It contains no
 * reference code: it includes the vendored CSR5 and HOLA headers and the
 * toolkit's cuSPARSE and CUB, and calls each the way src/spmv.cu does:
 *
 *   comp_cusparse_time  cusparseSpMV CSR_ALG2 / COO_ALG2    src/spmv.cu:7-121
 *   comp_cub_time       cub::DeviceSpmv::CsrMV ("MERGE")    src/spmv.cu:123-157
 *   comp_csr5_time      anonymouslibHandle asCSR5 + spmv    src/spmv.cu:336-377
 *   comp_hola_time      hola_spmv, HolaMode::Default        src/spmv.cu:379-424
 *
 * Each runs on the legacy default stream (CSR5 and HOLA take no stream),
 * warms up three times, then times `reps` back-to-back calls with CUDA
 * events and returns the mean milliseconds per call; y holds A*x afterwards.
 * FP64 only (the reference instantiates float too; the comparison runs on
 * the FP64 workloads).  Used by bench.py's reference arm and tests/, and
 * nothing else.  None of these kernels waits on another CTA: CSR5 and HOLA
 * combine rows with atomics, cuSPARSE and CUB are the toolkit's own.
 */
#include <cusparse.h>

#include <cub/device/device_spmv.cuh>
#include <stdexcept>

#include "csr5/anonymouslib_cuda.h"
#include "hola/hola.cuh"

std::fstream FSTR;  // declared extern by the reference's inc.cuh

namespace {

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~EventPair() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    float ms() {
        float v = 0.f;
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&v, a, b);
        return v;
    }
};

/* Warm up three times, then time `reps` calls of `f` on stream 0. */
template <class F>
int time_calls(F f, int reps, float* ms_per_call) {
    for (int r = 0; r < 3; ++r) f();
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return (int)e;
    EventPair ev;
    cudaEventRecord(ev.a, 0);
    for (int r = 0; r < reps; ++r) f();
    cudaEventRecord(ev.b, 0);
    float ms = ev.ms();
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    *ms_per_call = reps > 0 ? ms / reps : 0.f;
    return 0;
}

}  // namespace

extern "C" {

/* alg 0: CUSPARSE_SPMV_CSR_ALG2 on (row_ptr, col, vals), as Fun_CSRMV
 * (src/spmv.cu:32-52); alg 1: CUSPARSE_SPMV_COO_ALG2 on (row_idx, col,
 * vals) in CSR order, as Fun_COOMV (src/spmv.cu:90-111).  alpha 1, beta 0.
 * Returns 0, a cudaError_t, or 10000 + a cusparseStatus_t. */
int comp_cusparse_time(int alg, int nrow, int ncol, int nnz, const int* d_row_ptr,
                       const int* d_row_idx, const int* d_col, const double* d_vals,
                       const double* d_x, double* d_y, int reps, float* ms_per_call) {
    cusparseHandle_t h = nullptr;
    cusparseSpMatDescr_t A = nullptr;
    cusparseDnVecDescr_t X = nullptr, Y = nullptr;
    void* buf = nullptr;
    int rc = 0;
    const double alpha = 1.0, beta = 0.0;
    cusparseSpMVAlg_t a = alg == 0 ? CUSPARSE_SPMV_CSR_ALG2 : CUSPARSE_SPMV_COO_ALG2;
    size_t bytes = 0;
    cusparseStatus_t st = cusparseCreate(&h);
    if (st == CUSPARSE_STATUS_SUCCESS)
        st = alg == 0 ? cusparseCreateCsr(&A, nrow, ncol, nnz, (void*)d_row_ptr, (void*)d_col,
                                          (void*)d_vals, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                                          CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F)
                      : cusparseCreateCoo(&A, nrow, ncol, nnz, (void*)d_row_idx, (void*)d_col,
                                          (void*)d_vals, CUSPARSE_INDEX_32I,
                                          CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F);
    if (st == CUSPARSE_STATUS_SUCCESS)
        st = cusparseCreateDnVec(&X, ncol, (void*)d_x, CUDA_R_64F);
    if (st == CUSPARSE_STATUS_SUCCESS) st = cusparseCreateDnVec(&Y, nrow, (void*)d_y, CUDA_R_64F);
    if (st == CUSPARSE_STATUS_SUCCESS)
        st = cusparseSpMV_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A, X, &beta, Y,
                                     CUDA_R_64F, a, &bytes);
    if (st == CUSPARSE_STATUS_SUCCESS) {
        cudaError_t e = cudaMalloc(&buf, bytes ? bytes : 16);
        if (e != cudaSuccess) rc = (int)e;
    }
    if (st == CUSPARSE_STATUS_SUCCESS && rc == 0) {
        cusparseStatus_t call = CUSPARSE_STATUS_SUCCESS;
        rc = time_calls(
            [&] {
                cusparseStatus_t s2 = cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, &alpha, A,
                                                   X, &beta, Y, CUDA_R_64F, a, buf);
                if (s2 != CUSPARSE_STATUS_SUCCESS) call = s2;
            },
            reps, ms_per_call);
        if (rc == 0 && call != CUSPARSE_STATUS_SUCCESS) rc = 10000 + (int)call;
    }
    if (st != CUSPARSE_STATUS_SUCCESS && rc == 0) rc = 10000 + (int)st;
    if (buf) cudaFree(buf);
    if (Y) cusparseDestroyDnVec(Y);
    if (X) cusparseDestroyDnVec(X);
    if (A) cusparseDestroySpMat(A);
    if (h) cusparseDestroy(h);
    return rc;
}

/* cub::DeviceSpmv::CsrMV, the merge-based CSR SpMV the reference labels
 * MERGE (src/spmv.cu:138-147). */
int comp_cub_time(int nrow, int ncol, int nnz, const int* d_row_ptr, const int* d_col,
                  const double* d_vals, const double* d_x, double* d_y, int reps,
                  float* ms_per_call) {
    size_t bytes = 0;
    cudaError_t e = cub::DeviceSpmv::CsrMV<double>(nullptr, bytes, d_vals, d_row_ptr, d_col, d_x,
                                                   d_y, nrow, ncol, nnz);
    if (e != cudaSuccess) return (int)e;
    void* tmp = nullptr;
    e = cudaMalloc(&tmp, bytes ? bytes : 16);
    if (e != cudaSuccess) return (int)e;
    int rc = time_calls(
        [&] {
            cub::DeviceSpmv::CsrMV<double>(tmp, bytes, d_vals, d_row_ptr, d_col, d_x, d_y, nrow,
                                           ncol, nnz, (cudaStream_t)0);
        },
        reps, ms_per_call);
    cudaFree(tmp);
    return rc;
}

/* CSR5 with its auto-tuned sigma, as Fun_CSR5 (src/spmv.cu:352-368).  The
 * conversion transposes the column and value arrays in place, so the caller
 * passes copies (d_col_work, d_val_work).  Each timed call is a memset of y
 * followed by spmv, as the reference's loop does.  build_ms = asCSR5 + setX
 * (the reference's tim1); sigma_out = the sigma CSR5 chose.  Returns 0, a
 * cudaError_t, or 20000 - an anonymouslib error code. */
int comp_csr5_time(int nrow, int ncol, int nnz, const int* d_row_ptr, int* d_col_work,
                   double* d_val_work, double* d_x, double* d_y, int reps, float* build_ms,
                   float* ms_per_call, int* sigma_out) {
    anonymouslibHandle<int, unsigned int, double> A(nrow, ncol);
    A.inputCSR(nnz, const_cast<int*>(d_row_ptr), d_col_work, d_val_work);
    A.setSigma(ANONYMOUSLIB_AUTO_TUNED_SIGMA);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return (int)e;
    EventPair ev;
    cudaEventRecord(ev.a, 0);
    int err = A.asCSR5();
    if (err == ANONYMOUSLIB_SUCCESS) err = A.setX(d_x);
    cudaEventRecord(ev.b, 0);
    *build_ms = ev.ms();
    if (err != ANONYMOUSLIB_SUCCESS) return 20000 - err;
    int nnz_per_row = nrow > 0 ? nnz / nrow : 0;
    *sigma_out = nnz_per_row <= 4 ? 4 : nnz_per_row <= 32 ? nnz_per_row : nnz_per_row <= 256 ? 32 : 6;
    int call_err = ANONYMOUSLIB_SUCCESS;
    int rc = time_calls(
        [&] {
            cudaMemsetAsync(d_y, 0, sizeof(double) * (size_t)nrow, 0);
            int r = A.spmv(1.0, d_y);
            if (r != ANONYMOUSLIB_SUCCESS) call_err = r;
        },
        reps, ms_per_call);
    A.destroy();
    if (rc == 0 && call_err != ANONYMOUSLIB_SUCCESS) rc = 20000 - call_err;
    e = cudaDeviceSynchronize();
    if (rc == 0 && e != cudaSuccess) rc = (int)e;
    return rc;
}

/* HOLA in its default mode (sorted, 4 or 8 nonzeros per thread by nnz), as
 * Fun_HOLA (src/spmv.cu:394-416); build_ms = the temp-size query and its
 * allocation (the reference's tim1).  Returns 0, a cudaError_t, or 30000 when
 * hola_spmv throws. */
int comp_hola_time(int nrow, int ncol, int nnz, const int* d_row_ptr, const int* d_col,
                   double* d_vals, double* d_x, double* d_y, int reps, float* build_ms,
                   float* ms_per_call) {
    dCSR<double> m(nrow, ncol, nnz, d_vals, const_cast<int*>(d_row_ptr), const_cast<int*>(d_col));
    dDenseVector<double> v(ncol, d_x);
    dDenseVector<double> r(nrow, d_y);
    int rc = 0;
    void* tmp = nullptr;
    try {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) throw std::runtime_error("device");
        EventPair ev;
        cudaEventRecord(ev.a, 0);
        size_t req = 0;
        hola_spmv(nullptr, req, r, m, v, HolaMode::Default, false, false);
        e = cudaMalloc(&tmp, req ? req : 16);
        cudaEventRecord(ev.b, 0);
        *build_ms = ev.ms();
        if (e != cudaSuccess) {
            rc = (int)e;
            tmp = nullptr;
        } else {
            rc = time_calls([&] { hola_spmv(tmp, req, r, m, v, HolaMode::Default, false, false); },
                            reps, ms_per_call);
        }
    } catch (const std::exception&) {
        if (rc == 0) rc = 30000;
    }
    if (tmp) cudaFree(tmp);
    // the vectors wrap caller-owned buffers: keep their destructors off them
    // (a reallocation inside hola_spmv would show as a moved pointer)
    if (r.data != d_y && rc == 0) rc = 30001;
    if (r.data == d_y) r.data = nullptr;
    v.data = nullptr;
    return rc;
}

}  // extern "C"
