// Row-group CSR SpMV for sm_100a (configuration kind 3):  y = alpha*A x + beta*y.
//
// For matrices whose rows are short and even (stencils, meshes), the merge-
// path walk costs more than it saves: every item goes through shared memory
// twice and every row end through a scan.  Here a group of LPR lanes owns a
// whole row: the lanes read the row's col_idx/vals coalesced (lane j takes
// nonzeros j, j+LPR, ...), keep 4-16 gathers of x in flight, accumulate with
// the dtype's policy (F64: double; F32/BF16: TwoSum), and the group combines
// its lane sums by a fixed butterfly in double.  No row spans two groups, so
// there are no carries, no atomics and no shared memory; results are
// deterministic.  Warp w takes row blocks w, w + NW, ... of 32/LPR rows.
//
// The tuner (merbit_plan_tune) times this kernel beside the merge-path ones
// and keeps it only where it wins; long rows make it slow, never wrong.
#include <type_traits>

#include "merbit_internal.cuh"

namespace merbit {
namespace {

// finish for a launch that reduces a residual without taking part in the
// carry epochs: a counter of its own (LaunchState::pad[0]).
template <int NW>
__device__ __forceinline__ void finish_residual_only(LaunchState* st, double v, double* partials,
                                                     int idx, int nparts, double* out) {
    __shared__ double s_red[NW];
    __shared__ int s_last;
    unsigned* counter = reinterpret_cast<unsigned*>(&st->pad[0]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) t += s_red[w];
        partials[idx] = t;
        __threadfence();
        s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double t = 0.0;
    for (int i = threadIdx.x; i < nparts; i += NW * 32)
        t += __longlong_as_double((long long)ld_relaxed_u64(
            reinterpret_cast<const unsigned long long*>(partials + i)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
    if (lane == 0) s_red[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) tot += s_red[w];
        *out = tot;
        *counter = 0u;
        __threadfence();
    }
}

// STG (staged row blocks): the warp's RPW rows hold nonzeros [bs, be), one
// contiguous run.  When it fits in CAP = 32 * UNR entries the warp loads it
// coalesced (lane l takes bs + l, bs + l + 32, ...), gathers x, and stores the
// products in its shared-memory slice; each group then sums its row from
// there.  A lane sums the same nonzeros in the same order as without
// staging (j, j + LPR, ... of its row).  Every col/vals line is touched once
// per warp instead of once per unrolled step, which cuts the L1 wavefronts of
// short rows several-fold.  Blocks that do not fit take the strided path.
// Products per TwoSum step with compensated (FP32/BF16) accumulation; a
// block of 4 costs at most 4 roundings of its sum |a x|.
template <class Acc>
constexpr int kRowsBlock = std::is_same<Acc, AccTwoSum>::value ? 4 : 1;

template <int DT, int LPR, int WARPS, bool RES, bool CG, bool STG = false>
__global__ void __launch_bounds__(WARPS * 32) spmv_rows_kernel(const SpmvLaunch a) {
    using Pr = Prec<DT>;
    using V = typename Pr::V;
    using X = typename Pr::X;
    using Y = typename Pr::Y;
    using P = typename Pr::P;
    using Acc = typename Pr::Acc;
    constexpr int RPW = 32 / LPR;  // rows per warp step
    // loads in flight per lane and step: a 27-point row at 4 lanes per row
    // is one step
    constexpr int UNR = LPR <= 2 ? 16 : (LPR <= 4 ? 8 : 4);
    const int lane = threadIdx.x & 31;
    const int grp = lane / LPR, jl = lane % LPR;
    const unsigned gmask = LPR == 32 ? 0xFFFFFFFFu : (((1u << LPR) - 1u) << (grp * LPR));
    const int nw = (int)gridDim.x * WARPS;
    const int gw = (int)blockIdx.x * WARPS + (threadIdx.x >> 5);
    const int32_t* __restrict__ rp = a.row_ptr;
    const int32_t* __restrict__ col = a.col;
    const V* __restrict__ vals = static_cast<const V*>(a.vals);
    const X* __restrict__ xv = static_cast<const X*>(a.x);
    RowStore<Y, RES> out(a);
    constexpr int CAP = 32 * UNR;
    __shared__ P s_prod[STG ? WARPS : 1][STG ? CAP : 1];
    P* __restrict__ sp = s_prod[STG ? (threadIdx.x >> 5) : 0];
    for (int r0 = gw * RPW; r0 < a.nrow; r0 += nw * RPW) {
        const int r = r0 + grp;
        Acc acc;
        acc.zero();
        bool staged = false;
        if (STG) {
            int s = 0, e = 0;
            if (r < a.nrow) {
                s = __ldg(rp + r);
                e = __ldg(rp + r + 1);
            }
            const int nb_rows = min(RPW, a.nrow - r0);  // >= 1: r0 < nrow
            const int bs = __shfl_sync(0xFFFFFFFFu, s, 0);
            const int be = __shfl_sync(0xFFFFFFFFu, e, (nb_rows - 1) * LPR);
            if (be - bs <= CAP) {  // warp-uniform
                int c[UNR];
                V v[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    const int k = bs + lane + 32 * u;
                    c[u] = k < be ? __ldcs(col + k) : -1;
                    v[u] = k < be ? __ldcs(vals + k) : V(0);
                }
                X xg[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u)
                    xg[u] = c[u] >= 0 ? (CG ? __ldcg(xv + c[u]) : __ldg(xv + c[u])) : (X)0;
#pragma unroll
                for (int u = 0; u < UNR; ++u)
                    if (c[u] >= 0) sp[lane + 32 * u] = to_p(v[u]) * (P)xg[u];
                __syncwarp();
                // (clamped to the staged run, which a valid CSR never leaves)
                const int i1 = min(e, be) - bs;
                int i = max(s - bs, 0) + jl;
                if constexpr (kRowsBlock<Acc> > 1) {
                    // compensated accumulation: 4 products per TwoSum step
                    for (; i + 3 * LPR < i1; i += 4 * LPR)
                        acc.add((sp[i] + sp[i + LPR]) + (sp[i + 2 * LPR] + sp[i + 3 * LPR]));
                }
                for (; i < i1; i += LPR) acc.add(sp[i]);
                __syncwarp();  // the slice is rewritten by the next block
                staged = true;
            }
        }
        if (!staged && r < a.nrow) {
            const int s = __ldg(rp + r), e = __ldg(rp + r + 1);
            // steps of UNR * LPR nonzeros, predicated at the row end, so all
            // of a step's loads are in flight together
            for (int i = s + jl; i < e; i += UNR * LPR) {
                int c[UNR];
                V v[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u) {
                    const int k = i + u * LPR;
                    c[u] = k < e ? __ldcs(col + k) : -1;
                    v[u] = k < e ? __ldcs(vals + k) : V(0);
                }
                X xg[UNR];
#pragma unroll
                for (int u = 0; u < UNR; ++u)
                    xg[u] = c[u] >= 0 ? (CG ? __ldcg(xv + c[u]) : __ldg(xv + c[u])) : (X)0;
                if constexpr (kRowsBlock<Acc> > 1) {
                    // compensated accumulation: blocks of 4 products summed
                    // by f32 fused multiply-adds, one TwoSum per block
#pragma unroll
                    for (int u0 = 0; u0 < UNR; u0 += 4) {
                        P blk = (P)0;
#pragma unroll
                        for (int u = u0; u < u0 + 4 && u < UNR; ++u)
                            if (c[u] >= 0) blk = fmaf(to_p(v[u]), (P)xg[u], blk);
                        acc.add(blk);
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < UNR; ++u)
                        if (c[u] >= 0) acc.add(to_p(v[u]) * (P)xg[u]);
                }
            }
        }
        double t = acc.value();
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) t += __shfl_xor_sync(gmask, t, o);
        if (r < a.nrow && jl == 0) out(r, t);
    }
    if (RES)
        finish_residual_only<WARPS>(a.state, out.res, a.partials, (int)blockIdx.x, (int)gridDim.x,
                                    a.residual);
}

template <int DT, int LPR, bool RES, bool CG, bool STG>
int launch_rows_k(const SpmvLaunch& a, cudaStream_t s) {
    constexpr int WARPS = 8;
    static int grid_cap[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return fail(MERBIT_ERR_UNSUPPORTED, "spmv_rows: device ordinal >= 64");
    auto kern = spmv_rows_kernel<DT, LPR, WARPS, RES, CG, STG>;
    // per-device cache; threads that race here compute the same value
    int cap = __atomic_load_n(&grid_cap[dev], __ATOMIC_ACQUIRE);
    if (cap == 0) {
        int per_sm = 0, sms = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, 0);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy(spmv_rows)");
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cap = per_sm > 0 && sms > 0 ? per_sm * sms : 1;
        __atomic_store_n(&grid_cap[dev], cap, __ATOMIC_RELEASE);
    }
    constexpr int RPB = WARPS * (32 / LPR);  // rows per block step
    const long long need = ((long long)a.nrow + RPB - 1) / RPB;
    const int grid = (int)(need < cap ? need : cap);
    if (RES && !a.partials) return fail(MERBIT_ERR_INVALID, "spmv_rows: residual without partials");
    kern<<<grid, WARPS * 32, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? (int)MERBIT_OK : cuda_fail(e, "spmv_rows_kernel launch");
}

template <int DT, int LPR, bool STG = false>
int launch_rows_lpr(const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s) {
    if (a.residual)
        return c.cg ? launch_rows_k<DT, LPR, true, true, STG>(a, s)
                    : launch_rows_k<DT, LPR, true, false, STG>(a, s);
    return c.cg ? launch_rows_k<DT, LPR, false, true, STG>(a, s)
                : launch_rows_k<DT, LPR, false, false, STG>(a, s);
}

template <int DT>
int launch_rows_dt(const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s) {
    if (c.stg) {
        switch (c.ipt) {  // lanes per row
        case 1: return launch_rows_lpr<DT, 1, true>(c, a, s);
        case 2: return launch_rows_lpr<DT, 2, true>(c, a, s);
        case 4: return launch_rows_lpr<DT, 4, true>(c, a, s);
        case 8: return launch_rows_lpr<DT, 8, true>(c, a, s);
        }
        return fail(MERBIT_ERR_INVALID, "spmv_rows: no such configuration");
    }
    switch (c.ipt) {  // lanes per row
    case 2: return launch_rows_lpr<DT, 2>(c, a, s);
    case 4: return launch_rows_lpr<DT, 4>(c, a, s);
    case 8: return launch_rows_lpr<DT, 8>(c, a, s);
    case 16: return launch_rows_lpr<DT, 16>(c, a, s);
    case 32: return launch_rows_lpr<DT, 32>(c, a, s);
    }
    return fail(MERBIT_ERR_INVALID, "spmv_rows: no such configuration");
}

}  // namespace

int spmv_rows_launch(int dtype, const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s) {
    if (a.nrow <= 0) return MERBIT_OK;
    switch (dtype) {
    case MERBIT_F64: return launch_rows_dt<MERBIT_F64>(c, a, s);
    case MERBIT_F32: return launch_rows_dt<MERBIT_F32>(c, a, s);
    case MERBIT_BF16: return launch_rows_dt<MERBIT_BF16>(c, a, s);
    }
    return fail(MERBIT_ERR_INVALID, "spmv_rows: bad dtype");
}

}  // namespace merbit
