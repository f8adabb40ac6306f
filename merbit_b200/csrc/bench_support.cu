// Measurement support (not part of the SpMV path): the random-gather rate
// of this GPU, the ceiling that bounds an SpMV whose columns are random.
// Each thread streams K column indices (128-bit loads, evict-first) and
// gathers x at them through L1, with all K gathers in flight; the sum is
// written so the loads are not dead.  Indices outside [0, nx) read x[0].
// K = 8 at 2048 threads per SM measured the fastest on B200 among 8, 16 and
// 32 gathers per thread, 1024 or 2048 threads per SM, L1-allocating or
// L2-only loads and L1 carveouts from 28% to 100% shared (274 against 261 G
// gathers/s for K = 16), so the ceiling reported is the best rate seen.
#include "merbit_internal.cuh"

namespace merbit {
namespace {

template <int K>
__global__ void __launch_bounds__(256) gather_probe_kernel(const double* __restrict__ x, int nx,
                                                           const int* __restrict__ idx,
                                                           long long n, double* __restrict__ out) {
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long nt = (long long)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (long long b = tid * K; b + K <= n; b += nt * K) {
        int c[K];
#pragma unroll
        for (int k = 0; k < K; k += 4) {
            const int4 q = __ldcs(reinterpret_cast<const int4*>(idx + b + k));
            c[k] = q.x;
            c[k + 1] = q.y;
            c[k + 2] = q.z;
            c[k + 3] = q.w;
        }
        double v[K];
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = __ldg(x + ((unsigned)c[k] < (unsigned)nx ? c[k] : 0));
#pragma unroll
        for (int k = 0; k < K; ++k) acc += v[k];
    }
    out[tid] = acc;
}

}  // namespace
}  // namespace merbit

using namespace merbit;

extern "C" int merbit_bench_gather(const double* d_x, int32_t nx, const int32_t* d_idx, int64_t n,
                                   double* d_out, int32_t out_len, void* stream) {
    if (!d_x || !d_idx || !d_out || nx <= 0 || n < 0)
        return fail(MERBIT_ERR_INVALID, "bench_gather: bad arguments");
    if (((uintptr_t)d_idx & 15) != 0) return fail(MERBIT_ERR_INVALID, "bench_gather: idx not 16-byte aligned");
    int dev = 0, sms = 0;
    MERBIT_CUDA(cudaGetDevice(&dev));
    MERBIT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8;
    if ((long long)out_len < (long long)blocks * 256)
        return fail(MERBIT_ERR_INVALID, "bench_gather: out_len < 2048 * SM count");
    gather_probe_kernel<8><<<blocks, 256, 0, (cudaStream_t)stream>>>(d_x, nx, d_idx, n, d_out);
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}
