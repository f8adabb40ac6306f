// Batched warp-tile SpMV (k = 1 right-hand side) for sm_100a:
//   y_m = alpha * A_m x_m + beta * y_m   for every matrix m of a batch,
// in one persistent cooperative launch.
//
// The tiles of all matrices form one index space (matrix m owns global
// tiles [tile_begin_m, tile_begin_m + num_tiles_m)); global warp w takes
// tiles w, w + NW, ... in increasing order, so the matrix of a warp's tile
// only moves forward.  Each tile runs the single-matrix warp-tile walk
// (warp_tile.cuh, described in spmv_warp.cu): TMA bulk staging of the
// row_ptr window, col and vals slices on an mbarrier; all of a lane's x
// gathers in flight together in lane-contiguous order (no shared-memory bank
// conflicts); products in shared memory; a per-lane walk of an odd number of
// items (conflict-free strides); a shuffle segmented scan; coalesced row
// writes; boundary swaps and fixed-order look-backs for rows split between
// tiles.  Results are bitwise those of the single-matrix warp-tile kernel
// with the same items per lane.
//
// Per matrix: the items per lane (7, 11, 15, 19 or 23; tile = 32 x ipt
// items) is a property of the matrix's descriptor, chosen by the batch tuner
// per matrix signature.  One stage per warp is sized for the largest tile
// of the kernel variant (11, 15 or 23 items per lane), with a row_ptr window
// for a tile whose every item ends a row, so no member is restricted in
// rows per tile (R-MAT matrices have runs of empty rows).
//
// When a warp moves on to another matrix it first finishes what it holds
// of the previous one: its pending boundary swaps and its queued look-backs
// (which wait only for tiles smaller than ones this warp already processed,
// so the argument that the persistent grid cannot deadlock still holds).
#include <mutex>

#include "warp_tile.cuh"

namespace merbit {

namespace {

constexpr int kBatchWarps = 8;

// One stage for tiles of up to 32 * MAXIPT items, every item possibly a row end.
template <int DT, int MAXIPT>
using BatchSmem = WarpSmem<typename Prec<DT>::V, typename Prec<DT>::P, MAXIPT, 32 * MAXIPT + 16>;

// Tile source of a batch member: its descriptor, copied to the warp's
// shared memory when the warp reaches the matrix.
struct BatchSrc {
    const SpmmDesc* d;  // shared memory
    const SpmmLaunch& a;
    __device__ __forceinline__ int2 coord(int u) const { return d->coords[u]; }
    __device__ __forceinline__ const int32_t* row_ptr() const { return d->row_ptr; }
    __device__ __forceinline__ const int32_t* col() const { return d->col; }
    __device__ __forceinline__ const void* vals() const { return d->vals; }
    __device__ __forceinline__ const void* x() const { return d->x; }
    __device__ __forceinline__ int nrow() const { return d->nrow; }
    __device__ __forceinline__ int nnz() const { return d->nnz; }
    __device__ __forceinline__ int num_tiles() const { return d->num_tiles; }
    __device__ __forceinline__ const int2* coords() const { return d->coords; }
    __device__ __forceinline__ unsigned long long* slots() const { return a.slots; }
    __device__ __forceinline__ unsigned long long* xch() const { return a.xch; }
    __device__ __forceinline__ int nslots() const { return a.nslots; }
    __device__ __forceinline__ LaunchState* state() const { return a.state; }
    __device__ __forceinline__ int slot_base() const { return d->tile_begin; }
};

// Final store of one row of the current matrix, rounded as RowStore rounds
// it: y[r] = fma(beta, y[r], alpha * v).
template <typename Y>
struct BatchRowStore {
    Y* y;
    double alpha, beta;
    __device__ __forceinline__ void operator()(int r, double v) {
        double o = __dmul_rn(alpha, v);
        if (beta != 0.0) o = __fma_rn(beta, (double)y[r], o);
        y[r] = (Y)o;
    }
};

template <int DT, bool CG, int IPT, int MAXIPT>
using BT = WarpTile<DT, IPT, CG, BatchSmem<DT, MAXIPT>>;

// Issues (ISSUE) or processes the tile of `ipt` items per lane: a kernel
// with stages for MAXIPT takes ipt in {7, 11} (11), {7, 11, 15} (15) or
// {15, 19, 23} (23); the tuner only assigns those.
template <int DT, bool CG, int MAXIPT, bool ISSUE, int IPT, class... A>
__device__ __forceinline__ void run_ipt(A&&... args) {
    if constexpr (ISSUE)
        BT<DT, CG, IPT, MAXIPT>::issue(args...);
    else
        BT<DT, CG, IPT, MAXIPT>::process(args...);
}
template <int DT, bool CG, int MAXIPT, bool ISSUE, class... A>
__device__ __forceinline__ void dispatch_ipt(int ipt, A&&... args) {
    if constexpr (MAXIPT == 11) {
        if (ipt == 7)
            run_ipt<DT, CG, MAXIPT, ISSUE, 7>(args...);
        else
            run_ipt<DT, CG, MAXIPT, ISSUE, 11>(args...);
    } else if constexpr (MAXIPT == 15) {
        if (ipt == 7)
            run_ipt<DT, CG, MAXIPT, ISSUE, 7>(args...);
        else if (ipt == 11)
            run_ipt<DT, CG, MAXIPT, ISSUE, 11>(args...);
        else
            run_ipt<DT, CG, MAXIPT, ISSUE, 15>(args...);
    } else {
        if (ipt == 15)
            run_ipt<DT, CG, MAXIPT, ISSUE, 15>(args...);
        else if (ipt == 19)
            run_ipt<DT, CG, MAXIPT, ISSUE, 19>(args...);
        else
            run_ipt<DT, CG, MAXIPT, ISSUE, 23>(args...);
    }
}

template <int DT, int WARPS, bool CG, int CV, int MAXIPT>
__global__ void __launch_bounds__(WARPS * 32) batch_warp_kernel(const SpmmLaunch a) {
    using S = BatchSmem<DT, MAXIPT>;
    using Y = typename Prec<DT>::Y;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned s_epoch;
    __shared__ LookBack s_lbq[WARPS][kLookBackQueue];
    __shared__ SpmmDesc s_desc[WARPS];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_epoch = *(volatile unsigned*)&a.state->epoch;
    unsigned char* ws = smem + (size_t)warp * S::bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(ws + S::bar_offset);
    if (lane == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const unsigned epoch = s_epoch;
    reset_other_parity(a.slots, a.nslots, epoch);
    reset_other_parity(a.xch, a.nslots, epoch);
    const int nw = (int)gridDim.x * WARPS;
    unsigned phase = 0u;
    int nlb = 0;
    PendingSwap pa, pb;
    pa.row = pb.row = -1;
    pa.got = pb.got = kEmpty;
    pa.mine = pb.mine = 0.0;
    pa.carry = 1;
    pb.carry = 0;
    BatchRowStore<Y> out{nullptr, a.alpha, a.beta};
    const BatchSrc src{&s_desc[warp], a};
    int m = -1;  // matrix whose descriptor s_desc[warp] holds
    for (int u = (int)blockIdx.x * WARPS + warp; u < a.total_tiles; u += nw) {
        int mm = m < 0 ? 0 : m;
        while (mm + 1 < a.ndesc && a.descs[mm + 1].tile_begin <= u) ++mm;
        if (mm != m) {  // warp-uniform
            if (m >= 0) {
                resolve_swap(pa, out);
                resolve_swap(pb, out);
                drain_look_backs(src, epoch, s_lbq[warp], nlb, lane, out);
                nlb = 0;
            }
            __syncwarp();
            constexpr int kWords = (int)(sizeof(SpmmDesc) / 4);
            static_assert(sizeof(SpmmDesc) % 4 == 0 && kWords <= 32, "descriptor copy");
            if (lane < kWords)
                reinterpret_cast<int*>(&s_desc[warp])[lane] =
                    __ldg(reinterpret_cast<const int*>(a.descs + mm) + lane);
            __syncwarp();
            out.y = static_cast<Y*>(s_desc[warp].y);
            m = mm;
        }
        const int lt = u - s_desc[warp].tile_begin;
        const int ipt = s_desc[warp].ipt;  // warp-uniform
        dispatch_ipt<DT, CG, MAXIPT, true>(ipt, src, lt, ws, bar, lane);
        const bool ok = __all_sync(0xFFFFFFFFu, mbar_wait_bounded(bar, phase, a.state));
        phase ^= 1u;
        __syncwarp();
        if (ok)
            dispatch_ipt<DT, CG, MAXIPT, false>(ipt, src, lt, epoch, ws, lane, pa, pb, out,
                                                s_lbq[warp], nlb);
    }
    if (m >= 0) {
        resolve_swap(pa, out);
        resolve_swap(pb, out);
        drain_look_backs(src, epoch, s_lbq[warp], nlb, lane, out);
    }
    __syncthreads();
    if (threadIdx.x == 0) finish_launch(a.state, epoch);
}

// Persistent cooperative grid of batch_warp_kernel (all CTAs resident).
template <int DT, bool CG, int CV, int MAXIPT, int WARPS = kBatchWarps>
int launch_batch_warp(const SpmmLaunch& a, cudaStream_t s) {
    using S = BatchSmem<DT, MAXIPT>;
    constexpr size_t smem = S::bytes * WARPS;
    static int grid_cap[64] = {};
    static std::mutex mu;
    auto kern = batch_warp_kernel<DT, WARPS, CG, CV, MAXIPT>;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return fail(MERBIT_ERR_UNSUPPORTED, "batch_warp: device ordinal >= 64");
    int cap = __atomic_load_n(&grid_cap[dev], __ATOMIC_ACQUIRE);
    if (cap == 0) {
        std::lock_guard<std::mutex> lk(mu);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "batch_warp_kernel attributes");
        if (CV) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, CV);
            if (e != cudaSuccess) return cuda_fail(e, "batch_warp_kernel carveout");
        }
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy(batch_warp_kernel)");
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cap = per_sm > 0 && sms > 0 ? per_sm * sms : 1;
        __atomic_store_n(&grid_cap[dev], cap, __ATOMIC_RELEASE);
    }
    const long long need = ((long long)a.total_tiles + WARPS - 1) / WARPS;
    const int grid = (int)(need < cap ? need : cap);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(WARPS * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.numAttrs = 1;
    if (CV) {
        attr[1].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
        attr[1].val.sharedMemCarveout = (unsigned)CV;
        cfg.numAttrs = 2;
    }
    cfg.attrs = attr;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? (int)MERBIT_OK : cuda_fail(e, "batch_warp_kernel launch");
}

template <int DT>
int launch_batch_warp_dt(int variant, const SpmmLaunch& a, cudaStream_t s) {
    switch (variant) {
    case 0: return launch_batch_warp<DT, false, 0, 15>(a, s);            // L1 gathers, all shared
    case 1: return launch_batch_warp<DT, false, kCarveoutL1, 15>(a, s);  // L1 gathers, more L1
    case 2: return launch_batch_warp<DT, true, kCarveoutL1, 15>(a, s);   // L2-only gathers
    case 3: return launch_batch_warp<DT, false, 0, 23>(a, s);            // larger tiles
    case 4: return launch_batch_warp<DT, false, kCarveoutL1, 23>(a, s);
    case 5: return launch_batch_warp<DT, false, kCarveoutL1Max, 15>(a, s);  // still more L1
    case 6: return launch_batch_warp<DT, false, kCarveoutL1Max, 11>(a, s);  // smaller stages
    case 7: return launch_batch_warp<DT, false, kCarveoutL1, 11>(a, s);
    case 8: return launch_batch_warp<DT, false, kCarveoutL1Most, 11>(a, s);  // most L1
    case 9: return launch_batch_warp<DT, false, kCarveoutL1Max, 11, 4>(a, s);  // 4-warp CTAs
    }
    return fail(MERBIT_ERR_INVALID, "batch_warp: no such variant");
}

}  // namespace

int batch_warp_launch(int dtype, int variant, const SpmmLaunch& a, cudaStream_t s) {
    if (a.total_tiles <= 0) return MERBIT_OK;
    switch (dtype) {
    case MERBIT_F64: return launch_batch_warp_dt<MERBIT_F64>(variant, a, s);
    case MERBIT_F32: return launch_batch_warp_dt<MERBIT_F32>(variant, a, s);
    case MERBIT_BF16: return launch_batch_warp_dt<MERBIT_BF16>(variant, a, s);
    }
    return fail(MERBIT_ERR_INVALID, "batch_warp: bad dtype");
}

}  // namespace merbit
