// Warp-tile merge-path SpMV for sm_100a:  y = alpha * A x + beta * y.
//
// Each warp owns tiles of 32*IPT merge items (row ends + nonzeros) and runs
// each start to finish with no CTA-wide barrier:
//
//   1. lane 0 issues bulk async copies (cp.async.bulk through the TMA
//      engine, L2 evict-first) of the tile's row_ptr window (none for a
//      tile inside one row), col_idx slice and vals slice into one of the
//      warp's STAGES shared-memory stages,
//      completing on that stage's mbarrier.  Ranges are rounded out to 16
//      bytes (only the last few elements of an array, which rounding would
//      overrun, are fetched with plain loads).  With STAGES = 2 the next
//      tile's copies are issued before the current tile is processed;
//   2. lanes gather x[col] for up to IPT nonzeros each (all loads in flight
//      together) and overwrite the staged values with the products;
//   3. each lane finds its segment start by merge search in shared memory
//      (the reference's predicate, include/utils.cuh:17) and walks IPT
//      items with predicated steps, staging every row it completes except
//      its first in shared memory;
//   4. a warp segmented scan (shuffles) turns the lanes' trailing partials
//      into each lane's first-row carry-in -- the role of the reference's
//      warp_segmented_sum (include/utils.cuh:58-83), without its atomics --
//      and the warp writes the tile's completed rows to y coalesced;
//   5. rows split between tiles -- which the reference finishes with global
//      float atomicAdd on CTA-boundary rows (include/tile.cuh:363-369) --
//      are finished without float atomics:
//        * a row split between two adjacent tiles (the common case): both
//          tiles swap their partial through one 64-bit atomicExch on a
//          boundary slot; whichever arrives second adds carry + head (always
//          in that order) and writes y.  Nobody waits;
//        * a row spanning three or more tiles: every tile publishes its
//          trailing partial, and the tile where the row ends sums the
//          partials of the tiles back to the row's start in a fixed order
//          (decoupled look-back, bounded waits).
//
// Every row is written once, from sums taken in a fixed order, so results
// are deterministic.  The grid is persistent and cooperative: all CTAs are
// resident and global warp w takes tiles w, w + NW, w + 2 NW, ... (NW =
// warps in the grid).  No tile counter is needed -- a same-address atomic
// per tile serializes at a few ns each, which at ~10^5 tiles per launch
// costs more than the SpMV itself -- and the look-back cannot deadlock: the
// smallest unfinished tile has all predecessors finished.
#include <mutex>

#include "warp_tile.cuh"

namespace merbit {

// The tile source of a single-matrix launch: everything comes from the
// kernel parameter block, and local tile u is slot u.
struct SpmvSrc {
    const SpmvLaunch& a;
    __device__ __forceinline__ int2 coord(int u) const { return a.coords[u]; }
    __device__ __forceinline__ const int32_t* row_ptr() const { return a.row_ptr; }
    __device__ __forceinline__ const int32_t* col() const { return a.col; }
    __device__ __forceinline__ const void* vals() const { return a.vals; }
    __device__ __forceinline__ const void* x() const { return a.x; }
    __device__ __forceinline__ int nrow() const { return a.nrow; }
    __device__ __forceinline__ int nnz() const { return a.nnz; }
    __device__ __forceinline__ int num_tiles() const { return a.num_tiles; }
    __device__ __forceinline__ const int2* coords() const { return a.coords; }
    __device__ __forceinline__ unsigned long long* slots() const { return a.slots; }
    __device__ __forceinline__ unsigned long long* xch() const { return a.xch; }
    __device__ __forceinline__ int nslots() const { return a.nslots; }
    __device__ __forceinline__ LaunchState* state() const { return a.state; }
    __device__ __forceinline__ int slot_base() const { return 0; }
};

// CV: the shared-memory carveout the kernel is launched with (it does not
// change the code; each split gets its own function and function attribute).
// FULL: the row_ptr window holds a tile whose every item ends a row (no cap
// on rows per tile; matrices with runs of empty rows), else warp_rp_cap(IPT).
template <int DT, int IPT, bool FULL>
using SpmvWarpSmem = WarpSmem<typename Prec<DT>::V, typename Prec<DT>::P, IPT,
                              FULL ? 32 * IPT + 16 : warp_rp_cap(IPT)>;

template <int DT, int WARPS, int IPT, int STAGES, bool RES, bool CG, int CV, bool FULL>
__global__ void __launch_bounds__(WARPS * 32) spmv_warp_kernel(const SpmvLaunch a) {
    using T = WarpTile<DT, IPT, CG, SpmvWarpSmem<DT, IPT, FULL>>;
    using S = typename T::S;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned s_epoch;
    __shared__ LookBack s_lbq[WARPS][kLookBackQueue];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_epoch = *(volatile unsigned*)&a.state->epoch;
    // stage k of this warp: wbase + k * S::bytes, its barrier at bar_offset;
    // bit k of `phases` is the parity stage k waits for next
    unsigned char* wbase = smem + (size_t)warp * STAGES * S::bytes;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < STAGES; ++k)
            mbar_init(reinterpret_cast<uint64_t*>(wbase + k * S::bytes + S::bar_offset), 1);
        fence_mbar_init();
    }
    __syncthreads();
    const unsigned epoch = s_epoch;
    reset_other_parity(a.slots, a.nslots, epoch);
    reset_other_parity(a.xch, a.nslots, epoch);
    const int nw = (int)gridDim.x * WARPS;
    unsigned phases = 0u;
    RowStore<typename T::Y, RES> out(a);
    int nlb = 0;  // queued look-backs of this warp
    PendingSwap pa, pb;
    pa.row = pb.row = -1;
    pa.got = pb.got = kEmpty;
    pa.mine = pb.mine = 0.0;
    pa.carry = 1;
    pb.carry = 0;
    const SpmvSrc src{a};
    int u = (int)blockIdx.x * WARPS + warp;
    if (u < a.num_tiles)
        T::issue(src, u, wbase, reinterpret_cast<uint64_t*>(wbase + S::bar_offset), lane);
    int k = 0;
    for (; u < a.num_tiles; u += nw) {
        const int un = u + nw;
        unsigned char* cur = wbase + (size_t)k * S::bytes;
        uint64_t* cbar = reinterpret_cast<uint64_t*>(cur + S::bar_offset);
        if (STAGES == 2 && un < a.num_tiles) {
            unsigned char* nxt = wbase + (size_t)(k ^ 1) * S::bytes;
            T::issue(src, un, nxt, reinterpret_cast<uint64_t*>(nxt + S::bar_offset), lane);
        }
        const bool ok =
            __all_sync(0xFFFFFFFFu, mbar_wait_bounded(cbar, (phases >> k) & 1u, a.state));
        phases ^= 1u << k;
        __syncwarp();
        if (ok) T::process(src, u, epoch, cur, lane, pa, pb, out, s_lbq[warp], nlb);
        if (STAGES == 1) {
            if (un < a.num_tiles) T::issue(src, un, cur, cbar, lane);
        } else {
            k ^= 1;
        }
    }
    resolve_swap(pa, out);
    resolve_swap(pb, out);
    drain_look_backs(src, epoch, s_lbq[warp], nlb, lane, out);
    if (RES) {
        finish_launch_residual<WARPS>(a.state, epoch, out.res, a.partials, (int)blockIdx.x,
                                      (int)gridDim.x, a.residual);
    } else {
        __syncthreads();
        if (threadIdx.x == 0) finish_launch(a.state, epoch);
    }
}

namespace {
// Launches a persistent cooperative grid of `kern` (all CTAs resident).
// `carveout` (percent of the largest shared-memory size, 0 = the driver's
// choice) is the kernel's preferred shared-memory / L1 split: every kernel
// instantiation has one fixed split (a template parameter), set once as the
// function's attribute before the occupancy query that sizes the grid, and
// passed again with each launch.
template <typename K>
int launch_coop(K kern, int warps, size_t smem, int carveout, int* grid_cap, const SpmvLaunch& a,
                cudaStream_t s, const char* name) {
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return fail(MERBIT_ERR_UNSUPPORTED, "spmv_warp: device ordinal >= 64");
    int cap = __atomic_load_n(&grid_cap[dev], __ATOMIC_ACQUIRE);
    if (cap == 0) {
        std::lock_guard<std::mutex> lk(mu);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, name);
        if (carveout) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
            if (e != cudaSuccess) return cuda_fail(e, name);
        }
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem);
        if (e != cudaSuccess) return cuda_fail(e, name);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cap = per_sm > 0 && sms > 0 ? per_sm * sms : 1;
        __atomic_store_n(&grid_cap[dev], cap, __ATOMIC_RELEASE);
    }
    const long long need = ((long long)a.num_tiles + warps - 1) / warps;
    const int grid = (int)(need < cap ? need : cap);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(warps * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.numAttrs = 1;
    if (carveout) {
        attr[1].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
        attr[1].val.sharedMemCarveout = (unsigned)carveout;
        cfg.numAttrs = 2;
    }
    cfg.attrs = attr;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? (int)MERBIT_OK : cuda_fail(e, name);
}

template <int DT, int WARPS, int IPT, int STAGES, bool RES, bool CG, int CV, bool FULL>
int launch_warp_k(const SpmvLaunch& a, cudaStream_t s) {
    using S = SpmvWarpSmem<DT, IPT, FULL>;
    static int grid_cap[64] = {};
    if (RES && !a.partials) return fail(MERBIT_ERR_INVALID, "spmv_warp: residual without partials");
    return launch_coop(spmv_warp_kernel<DT, WARPS, IPT, STAGES, RES, CG, CV, FULL>, WARPS,
                       S::bytes * WARPS * STAGES, CV, grid_cap, a, s, "spmv_warp_kernel");
}

template <int DT, int WARPS, int IPT, int STAGES, bool CG, int CV, bool FULL = false>
int launch_warp(const SpmvLaunch& a, cudaStream_t s) {
    return a.residual ? launch_warp_k<DT, WARPS, IPT, STAGES, true, CG, CV, FULL>(a, s)
                      : launch_warp_k<DT, WARPS, IPT, STAGES, false, CG, CV, FULL>(a, s);
}

// The (warps, items per thread, gather hint, carveout) combinations of the
// configuration tables in spmv.cu.
template <int DT>
int launch_warp_dt(const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s) {
    const int warps = c.block / 32, ipt = c.ipt;
    if (c.stages != 1) return fail(MERBIT_ERR_INVALID, "spmv_warp: no such configuration");
#define MERBIT_WARP_CASE(W, I, G, C)                                                   \
    if (warps == W && ipt == I && c.cg == G && c.carveout == C && !c.stg)              \
        return launch_warp<DT, W, I, 1, G, C>(a, s);
#define MERBIT_WARP_FULL_CASE(W, I, G, C)                                              \
    if (warps == W && ipt == I && c.cg == G && c.carveout == C && c.stg)               \
        return launch_warp<DT, W, I, 1, G, C, true>(a, s);
    MERBIT_WARP_CASE(8, 15, 1, kCarveoutL1)
    MERBIT_WARP_CASE(4, 15, 1, kCarveoutL1)
    MERBIT_WARP_CASE(8, 11, 1, kCarveoutL1)
    MERBIT_WARP_CASE(4, 15, 1, kCarveoutL1Max)
    MERBIT_WARP_CASE(8, 15, 0, kCarveoutL1)
    MERBIT_WARP_CASE(8, 15, 0, 0)
    MERBIT_WARP_CASE(4, 15, 0, 0)
    MERBIT_WARP_CASE(8, 11, 0, 0)
    MERBIT_WARP_CASE(8, 7, 0, 0)
    MERBIT_WARP_CASE(4, 23, 0, 0)
    MERBIT_WARP_CASE(8, 13, 1, kCarveoutL1)
    MERBIT_WARP_FULL_CASE(8, 11, 0, kCarveoutL1Max)
    MERBIT_WARP_FULL_CASE(8, 15, 0, kCarveoutL1Max)
    MERBIT_WARP_FULL_CASE(8, 11, 1, kCarveoutL1)
#undef MERBIT_WARP_CASE
#undef MERBIT_WARP_FULL_CASE
    return fail(MERBIT_ERR_INVALID, "spmv_warp: no such configuration");
}
}  // namespace

int spmv_warp_launch(int dtype, const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s) {
    if (a.num_tiles <= 0) return MERBIT_OK;
    switch (dtype) {
    case MERBIT_F64: return launch_warp_dt<MERBIT_F64>(c, a, s);
    case MERBIT_F32: return launch_warp_dt<MERBIT_F32>(c, a, s);
    case MERBIT_BF16: return launch_warp_dt<MERBIT_BF16>(c, a, s);
    }
    return fail(MERBIT_ERR_INVALID, "spmv_warp: bad dtype");
}

}  // namespace merbit
