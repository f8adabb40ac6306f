// Front end of the reference harness: COO sort, COO -> CSR offsets and the
// loader's PageRank weights, on the GPU.
//
//   merbit_coo_sort        GRAPH::sort (src/class.cu:143-177): order the COO
//                          triplets by (major, minor); a stable radix sort
//                          of the 64-bit key major<<32|minor, then a gather
//   merbit_coo_to_csr      cusparseXcoo2csr (include/tile.cuh:574): offsets
//                          of a sorted index array
//   merbit_outdegree_values Fun_Values (src/class.cu:2-34): value = 1 /
//                          (number of entries whose row_ind equals this
//                          entry's row_ind)
#include <cub/device/device_radix_sort.cuh>

#include "merbit_internal.cuh"

namespace merbit {
namespace {

int grid_of(long long n) {
    long long g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g > 0 ? g : 1);
}

__global__ void pack_keys(const int* __restrict__ major, const int* __restrict__ minor, int n,
                          unsigned long long* __restrict__ key, int* __restrict__ idx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        key[i] = ((unsigned long long)(unsigned)major[i] << 32) | (unsigned)minor[i];
        idx[i] = i;
    }
}

__global__ void unpack_keys(const unsigned long long* __restrict__ key, int n,
                            int* __restrict__ major, int* __restrict__ minor) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        major[i] = (int)(key[i] >> 32);
        minor[i] = (int)(key[i] & 0xFFFFFFFFull);
    }
}

template <typename V>
__global__ void permute_vals(const V* __restrict__ src, const int* __restrict__ perm, int n,
                             V* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[perm[i]];
}

// offsets[r] = first position with sorted[pos] >= r, r in [0, nrow].
__global__ void offsets_kernel(const int* __restrict__ sorted, int n, int nrow,
                               int* __restrict__ offsets) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= n; j += gridDim.x * blockDim.x) {
        const int prev = j == 0 ? -1 : min(sorted[j - 1], nrow);
        const int cur = j == n ? nrow : min(sorted[j], nrow);
        for (int r = prev + 1; r <= cur; ++r) offsets[r] = j;
    }
}

// cnt[nrow] counts indices outside [0, nrow).
__global__ void count_kernel(const int* __restrict__ idx, int n, int nrow, int* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int r = idx[i];
        atomicAdd(cnt + ((unsigned)r < (unsigned)nrow ? r : nrow), 1);
    }
}

template <typename V>
__global__ void inv_count_kernel(const int* __restrict__ idx, const int* __restrict__ cnt, int n,
                                 int nrow, V* __restrict__ vals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int r = idx[i];
        vals[i] = (V)((unsigned)r < (unsigned)nrow ? 1.0 / (double)cnt[r] : 0.0);
    }
}

}  // namespace
}  // namespace merbit

using namespace merbit;

extern "C" {

int merbit_coo_sort(int32_t nnz, int32_t* d_major, int32_t* d_minor, void* d_vals,
                    merbit_dtype dtype, void* stream) {
    if (nnz < 0) return fail(MERBIT_ERR_INVALID, "coo_sort: negative nnz");
    if (nnz == 0) return MERBIT_OK;
    if (!d_major || !d_minor) return fail(MERBIT_ERR_INVALID, "coo_sort: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long *k_in = nullptr, *k_out = nullptr;
    int *i_in = nullptr, *i_out = nullptr;
    void* tmpv = nullptr;
    void* temp = nullptr;
    const size_t vs = dtype_size(dtype);
    auto done = [&](int st) {  // stream-ordered: after the sort's own work on s
        dev_free(k_in, s);
        dev_free(k_out, s);
        dev_free(i_in, s);
        dev_free(i_out, s);
        dev_free(tmpv, s);
        dev_free(temp, s);
        return st;
    };
#define TRY(call)                                              \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return done(cuda_fail(_e, #call)); \
    } while (0)
#define TRY_ALLOC(p, bytes)                              \
    do {                                                 \
        int _st = dev_alloc(&(p), (bytes), s);           \
        if (_st != MERBIT_OK) return done(_st);          \
    } while (0)
    TRY_ALLOC(k_in, 8 * (size_t)nnz);
    TRY_ALLOC(k_out, 8 * (size_t)nnz);
    TRY_ALLOC(i_in, 4 * (size_t)nnz);
    TRY_ALLOC(i_out, 4 * (size_t)nnz);
    pack_keys<<<grid_of(nnz), 256, 0, s>>>(d_major, d_minor, nnz, k_in, i_in);
    size_t tb = 0;
    TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, k_in, k_out, i_in, i_out, nnz, 0, 64, s));
    TRY_ALLOC(temp, tb);
    TRY(cub::DeviceRadixSort::SortPairs(temp, tb, k_in, k_out, i_in, i_out, nnz, 0, 64, s));
    unpack_keys<<<grid_of(nnz), 256, 0, s>>>(k_out, nnz, d_major, d_minor);
    if (d_vals) {
        TRY_ALLOC(tmpv, vs * (size_t)nnz);
        TRY(cudaMemcpyAsync(tmpv, d_vals, vs * (size_t)nnz, cudaMemcpyDeviceToDevice, s));
        if (dtype == MERBIT_F64)
            permute_vals<double><<<grid_of(nnz), 256, 0, s>>>((const double*)tmpv, i_out, nnz,
                                                              (double*)d_vals);
        else if (dtype == MERBIT_F32)
            permute_vals<float><<<grid_of(nnz), 256, 0, s>>>((const float*)tmpv, i_out, nnz,
                                                             (float*)d_vals);
        else
            permute_vals<unsigned short><<<grid_of(nnz), 256, 0, s>>>(
                (const unsigned short*)tmpv, i_out, nnz, (unsigned short*)d_vals);
    }
    TRY(cudaGetLastError());
    TRY(cudaStreamSynchronize(s));
#undef TRY
#undef TRY_ALLOC
    return done(MERBIT_OK);
}

int merbit_coo_to_csr(int32_t nnz, const int32_t* d_sorted_rows, int32_t nrow, int32_t* d_row_ptr,
                      void* stream) {
    if (nnz < 0 || nrow < 0 || !d_row_ptr || (nnz > 0 && !d_sorted_rows))
        return fail(MERBIT_ERR_INVALID, "coo_to_csr: bad arguments");
    offsets_kernel<<<grid_of((long long)nnz + 1), 256, 0, (cudaStream_t)stream>>>(
        d_sorted_rows, nnz, nrow, d_row_ptr);
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

int merbit_outdegree_values(int32_t nnz, int32_t nrow, const int32_t* d_row_ind, void* d_vals,
                            merbit_dtype dtype, void* stream) {
    if (nnz < 0 || nrow < 0 || (nnz > 0 && (!d_row_ind || !d_vals)))
        return fail(MERBIT_ERR_INVALID, "outdegree_values: bad arguments");
    if (nnz == 0) return MERBIT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int* cnt = nullptr;
    const size_t cbytes = sizeof(int) * ((size_t)nrow + 1);
    int st = dev_alloc(&cnt, cbytes, s);
    if (st != MERBIT_OK) return st;
    int bad = 0;
    cudaError_t e = cudaMemsetAsync(cnt, 0, cbytes, s);
    if (e == cudaSuccess) {
        count_kernel<<<grid_of(nnz), 256, 0, s>>>(d_row_ind, nnz, nrow, cnt);
        if (dtype == MERBIT_F64)
            inv_count_kernel<double><<<grid_of(nnz), 256, 0, s>>>(d_row_ind, cnt, nnz, nrow,
                                                                  (double*)d_vals);
        else if (dtype == MERBIT_F32)
            inv_count_kernel<float><<<grid_of(nnz), 256, 0, s>>>(d_row_ind, cnt, nnz, nrow,
                                                                 (float*)d_vals);
        else
            inv_count_kernel<__nv_bfloat16><<<grid_of(nnz), 256, 0, s>>>(
                d_row_ind, cnt, nnz, nrow, (__nv_bfloat16*)d_vals);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&bad, cnt + nrow, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dev_free(cnt, s);
    if (e != cudaSuccess) return cuda_fail(e, "outdegree_values");
    if (bad) return fail(MERBIT_ERR_MATRIX, "outdegree_values: row index outside [0, nrow)");
    return MERBIT_OK;
}

}  // extern "C"
