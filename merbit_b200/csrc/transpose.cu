// Adjoint support: the transpose plan (for dX = A^T G) and the per-nonzero
// gradient of the values (dval[e] = sum_j G[row_e, j] * X[col_e, j]).
//
// The transpose is built once per structure with a stable LSD radix sort of
// the column indices (CUB), so the entries of each transpose row keep the
// row order of A and every dX sum is taken in a fixed order: the adjoint is
// deterministic and uses no float atomics.  The transposed values are a
// gathered copy of A's values through the permutation, refreshed with
// merbit_plan_transpose_refresh when A's values change.  dX = A^T G is then
// an ordinary merge-path SpMM on the transpose plan.
#include <cub/device/device_radix_sort.cuh>

#include "merbit_internal.cuh"

namespace merbit {
namespace {

__global__ void iota_kernel(int* __restrict__ out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = i;
}

// row_of[e] = r with row_ptr[r] <= e < row_ptr[r+1] (upper bound - 1).
__global__ void row_of_kernel(const int32_t* __restrict__ row_ptr, int nrow, int nnz,
                              int* __restrict__ row_of) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
        int lo = 0, hi = nrow;  // find largest r with row_ptr[r] <= e
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(row_ptr + mid) <= e)
                lo = mid;
            else
                hi = mid;
        }
        // skip empty rows sharing the same start
        row_of[e] = lo;
    }
}

// col_ptr from the sorted column keys: col_ptr[c] = first j with key[j] >= c.
__global__ void col_ptr_kernel(const int* __restrict__ key, int nnz, int ncol,
                               int* __restrict__ col_ptr) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= nnz; j += gridDim.x * blockDim.x) {
        const int prev = j == 0 ? -1 : key[j - 1];
        const int cur = j == nnz ? ncol : key[j];
        for (int c = prev + 1; c <= cur; ++c) col_ptr[c] = j;
    }
}

template <typename V>
__global__ void gather_kernel(const V* __restrict__ src, const int* __restrict__ perm, int n,
                              V* __restrict__ dst) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        dst[j] = src[perm[j]];
}

template <typename T>
__global__ void gather_map_kernel(const int* __restrict__ src, const int* __restrict__ perm,
                                  int n, int* __restrict__ dst) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        dst[j] = src[perm[j]];
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    return (int)(g > 0 ? g : 1);
}

// dval[e] = G[row_e] . X[col_e].  Groups of LPG lanes take one nonzero, each
// lane VW consecutive RHS values per vector load (k = LPG * VW * n); a warp
// takes U * (32 / LPG) nonzeros per step and issues all their loads before
// it uses any, so each lane keeps 2U vector loads in flight.  Products of
// the stored values are exact in double and summed in a fixed order (lane
// sums, then a butterfly over the group).
template <typename Xt, int VW>
struct DvalVec;
template <>
struct DvalVec<float, 4> {
    static __device__ __forceinline__ void ld(const float* p, float (&o)[4]) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = t.x;
        o[1] = t.y;
        o[2] = t.z;
        o[3] = t.w;
    }
};
template <>
struct DvalVec<float, 2> {
    static __device__ __forceinline__ void ld(const float* p, float (&o)[2]) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        o[0] = t.x;
        o[1] = t.y;
    }
};
template <>
struct DvalVec<double, 2> {
    static __device__ __forceinline__ void ld(const double* p, double (&o)[2]) {
        const double2 t = __ldg(reinterpret_cast<const double2*>(p));
        o[0] = t.x;
        o[1] = t.y;
    }
};
template <typename Xt>
struct DvalVec<Xt, 1> {
    static __device__ __forceinline__ void ld(const Xt* p, Xt (&o)[1]) { o[0] = __ldg(p); }
};

template <typename Xt, int LPG, int VW, int U>
__global__ void __launch_bounds__(256) dval_kernel(const int32_t* __restrict__ col,
                                                   const int* __restrict__ row_of, int nnz, int k,
                                                   const Xt* __restrict__ g, long long ldg,
                                                   const Xt* __restrict__ x, long long ldx,
                                                   Xt* __restrict__ out) {
    constexpr int GPW = 32 / LPG;
    const int lane = threadIdx.x & 31;
    const int grp = lane / LPG, jl = lane % LPG;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = gw * (U * GPW); base < nnz; base += nwarps * (U * GPW)) {
        int r[U], c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long e = base + u * GPW + grp;
            r[u] = e < nnz ? __ldg(row_of + e) : -1;
            c[u] = e < nnz ? __ldg(col + e) : 0;
        }
        double acc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) acc[u] = 0.0;
        for (int j = jl * VW; j < k; j += LPG * VW) {
            Xt gv[U][VW], xv[U][VW];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (r[u] >= 0) {
                    DvalVec<Xt, VW>::ld(g + (size_t)r[u] * ldg + j, gv[u]);
                    DvalVec<Xt, VW>::ld(x + (size_t)c[u] * ldx + j, xv[u]);
                } else {
#pragma unroll
                    for (int v = 0; v < VW; ++v) gv[u][v] = xv[u][v] = (Xt)0;
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int v = 0; v < VW; ++v) acc[u] = fma((double)gv[u][v], (double)xv[u][v], acc[u]);
        }
#pragma unroll
        for (int o = LPG / 2; o > 0; o >>= 1)
#pragma unroll
            for (int u = 0; u < U; ++u) acc[u] += __shfl_xor_sync(0xFFFFFFFFu, acc[u], o);
        if (jl == 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const long long e = base + u * GPW + grp;
                if (e < nnz) out[e] = (Xt)acc[u];
            }
        }
    }
}

// Widest VW the leading dimensions and base pointers allow for this k.
template <typename Xt>
int dval_vw(int k, long long ldg, long long ldx, const void* g, const void* x) {
    const int vmax = sizeof(Xt) == 4 ? 4 : 2;
    for (int vw = vmax; vw > 1; vw >>= 1) {
        const size_t a = (size_t)vw * sizeof(Xt);
        if (k % vw == 0 && ldg % vw == 0 && ldx % vw == 0 && (uintptr_t)g % a == 0 &&
            (uintptr_t)x % a == 0)
            return vw;
    }
    return 1;
}

template <typename Xt, int VW>
int launch_dval_vw(int k, int nnz, const int32_t* col, const int* row_of, const Xt* g,
                   long long ldg, const Xt* x, long long ldx, Xt* out, cudaStream_t s) {
    // lanes per nonzero: enough to cover k in one pass when k <= 32*VW
    const int per = (k + VW - 1) / VW;
    const int grid = 148 * 8;
#define MERBIT_DVAL(L)                                                                     \
    dval_kernel<Xt, L, VW, 4><<<grid, 256, 0, s>>>(col, row_of, nnz, k, g, ldg, x, ldx, out)
    if (per <= 1)
        MERBIT_DVAL(1);
    else if (per <= 2)
        MERBIT_DVAL(2);
    else if (per <= 4)
        MERBIT_DVAL(4);
    else if (per <= 8)
        MERBIT_DVAL(8);
    else if (per <= 16)
        MERBIT_DVAL(16);
    else
        MERBIT_DVAL(32);
#undef MERBIT_DVAL
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

template <typename Xt>
int launch_dval(const merbit_plan_s* p, int k, const void* g, long long ldg, const void* x,
                long long ldx, void* out, cudaStream_t s) {
    const Xt* gg = static_cast<const Xt*>(g);
    const Xt* xx = static_cast<const Xt*>(x);
    Xt* oo = static_cast<Xt*>(out);
    const int vw = dval_vw<Xt>(k, ldg, ldx, g, x);
    if constexpr (sizeof(Xt) == 4) {
        if (vw == 4) return launch_dval_vw<Xt, 4>(k, p->nnz, p->col, p->row_of, gg, ldg, xx, ldx, oo, s);
    }
    if (vw == 2) return launch_dval_vw<Xt, 2>(k, p->nnz, p->col, p->row_of, gg, ldg, xx, ldx, oo, s);
    return launch_dval_vw<Xt, 1>(k, p->nnz, p->col, p->row_of, gg, ldg, xx, ldx, oo, s);
}

int ensure_row_of(merbit_plan_s* p, cudaStream_t s) {
    if (p->row_of || p->nnz == 0) return MERBIT_OK;
    int st = dev_alloc(&p->row_of, sizeof(int) * (size_t)p->nnz, s);
    if (st != MERBIT_OK) return st;
    row_of_kernel<<<grid_for(p->nnz), 256, 0, s>>>(p->row_ptr, p->nrow, p->nnz, p->row_of);
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

int gather_values(const void* src, int dtype, const int* perm, int n, void* dst, cudaStream_t s) {
    if (n == 0) return MERBIT_OK;
    if (dtype == MERBIT_F64)
        gather_kernel<double><<<grid_for(n), 256, 0, s>>>(static_cast<const double*>(src), perm, n,
                                                         static_cast<double*>(dst));
    else if (dtype == MERBIT_F32)
        gather_kernel<float><<<grid_for(n), 256, 0, s>>>(static_cast<const float*>(src), perm, n,
                                                        static_cast<float*>(dst));
    else
        gather_kernel<unsigned short><<<grid_for(n), 256, 0, s>>>(
            static_cast<const unsigned short*>(src), perm, n, static_cast<unsigned short*>(dst));
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

}  // namespace
}  // namespace merbit

using namespace merbit;

extern "C" {

int merbit_plan_transpose(merbit_plan plan, merbit_plan* tplan, void* stream) {
    if (!plan || !tplan) return fail(MERBIT_ERR_INVALID, "plan_transpose: null pointer");
    *tplan = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    const int nnz = plan->nnz, ncol = plan->ncol;
    int* col_ptr = nullptr;
    int* row_idx = nullptr;
    int* perm = nullptr;
    void* vals_t = nullptr;
    int* keys_out = nullptr;
    int* iota = nullptr;
    void* temp = nullptr;
    int st = MERBIT_OK;
    auto cleanup = [&]() {  // stream-ordered: after the build's work on s
        dev_free(keys_out, s);
        dev_free(iota, s);
        dev_free(temp, s);
    };
    auto bail = [&](int status) {
        cleanup();
        dev_free(col_ptr, s);
        dev_free(row_idx, s);
        dev_free(perm, s);
        dev_free(vals_t, s);
        return status;
    };
#define TRY_CUDA(call)                                                  \
    do {                                                                \
        cudaError_t _e = (call);                                        \
        if (_e != cudaSuccess) return bail(cuda_fail(_e, #call));       \
    } while (0)
#define TRY_ALLOC(p, bytes)                           \
    do {                                              \
        int _st = dev_alloc(&(p), (bytes), s);        \
        if (_st != MERBIT_OK) return bail(_st);       \
    } while (0)
    TRY_ALLOC(col_ptr, sizeof(int) * ((size_t)ncol + 1));
    const size_t nz = nnz > 0 ? (size_t)nnz : 1;
    TRY_ALLOC(row_idx, sizeof(int) * nz);
    TRY_ALLOC(perm, sizeof(int) * nz);
    TRY_ALLOC(vals_t, dtype_size(plan->dtype) * nz);
    st = ensure_row_of(plan, s);
    if (st != MERBIT_OK) return bail(st);
    if (nnz > 0) {
        TRY_ALLOC(keys_out, sizeof(int) * nz);
        TRY_ALLOC(iota, sizeof(int) * nz);
        iota_kernel<<<grid_for(nnz), 256, 0, s>>>(iota, nnz);
        int bits = 1;
        while (bits < 31 && (1ll << bits) < (long long)ncol) ++bits;
        size_t tb = 0;
        TRY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, plan->col, keys_out, iota, perm, nnz,
                                                 0, bits, s));
        TRY_ALLOC(temp, tb);
        TRY_CUDA(cub::DeviceRadixSort::SortPairs(temp, tb, plan->col, keys_out, iota, perm, nnz, 0,
                                                 bits, s));
        col_ptr_kernel<<<grid_for((long long)nnz + 1), 256, 0, s>>>(keys_out, nnz, ncol, col_ptr);
        gather_map_kernel<int><<<grid_for(nnz), 256, 0, s>>>(plan->row_of, perm, nnz, row_idx);
        TRY_CUDA(cudaGetLastError());
        st = gather_values(plan->vals, plan->dtype, perm, nnz, vals_t, s);
        if (st != MERBIT_OK) return bail(st);
    } else {
        TRY_CUDA(cudaMemsetAsync(col_ptr, 0, sizeof(int) * ((size_t)ncol + 1), s));
    }
    TRY_CUDA(cudaStreamSynchronize(s));
    cleanup();
#undef TRY_CUDA
#undef TRY_ALLOC
    merbit_plan t = nullptr;
    st = merbit_plan_create(&t, ncol, plan->nrow, nnz, col_ptr, row_idx, vals_t,
                            (merbit_dtype)plan->dtype, MERBIT_PLAN_SKIP_VALIDATE, stream);
    if (st != MERBIT_OK) {
        dev_free(col_ptr, s);
        dev_free(row_idx, s);
        dev_free(perm, s);
        dev_free(vals_t, s);
        return st;
    }
    t->owned.push_back(col_ptr);
    t->owned.push_back(row_idx);
    t->owned.push_back(perm);
    t->owned.push_back(vals_t);
    t->perm = perm;
    *tplan = t;
    return MERBIT_OK;
}

int merbit_plan_transpose_refresh(merbit_plan tplan, const void* d_src_vals, void* stream) {
    if (!tplan || !tplan->perm) return fail(MERBIT_ERR_INVALID, "transpose_refresh: not a transpose plan");
    if (tplan->nnz > 0 && !d_src_vals) return fail(MERBIT_ERR_INVALID, "transpose_refresh: vals is null");
    return gather_values(d_src_vals, tplan->dtype, tplan->perm, tplan->nnz,
                         const_cast<void*>(tplan->vals), (cudaStream_t)stream);
}

int merbit_dval(merbit_plan plan, int32_t k, const void* d_g, int64_t ldg, const void* d_x,
                int64_t ldx, void* d_dval, void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "dval: plan is null");
    if (k < 1 || ldg < k || ldx < k) return fail(MERBIT_ERR_INVALID, "dval: bad k / leading dimension");
    if (plan->nnz == 0) return MERBIT_OK;
    if (!d_g || !d_x || !d_dval) return fail(MERBIT_ERR_INVALID, "dval: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    int st = ensure_row_of(plan, s);
    if (st != MERBIT_OK) return st;
    if (plan->dtype == MERBIT_F64) return launch_dval<double>(plan, k, d_g, ldg, d_x, ldx, d_dval, s);
    return launch_dval<float>(plan, k, d_g, ldg, d_x, ldx, d_dval, s);
}

}  // extern "C"
