// Merge-path tiled CSR SpMV for sm_100a:  y = alpha * A x + beta * y.
//
// Follows the Merbit kernel's decomposition (include/tile.cuh:476-561 of the
// reference): the merge path over (row ends x nonzeros) is cut into equal
// tiles, each tile streams its slice of col_idx/vals, stages the products in
// shared memory, and threads walk fixed-length segments of the path.  It
// differs in how partial rows are combined:
//
//  * the reference sums a lane's row fragments with shared-memory atomics
//    and the rows shared by two CTAs with global float atomics (tile.cuh:
//    336, 81, 367); here every row is written exactly once, by the tile in
//    which it ends, after a deterministic segmented scan across the CTA's
//    threads and a decoupled look-back over the carries of earlier tiles,
//    so results are bit-reproducible run to run;
//  * the reference reads 4 B of descriptor per 14 merge items plus 8 B per
//    tile (tile.cuh:6-25) to avoid row_ptr; here each tile stages its window
//    of row_ptr (4 B per row, the compulsory row-pointer traffic) and every
//    thread finds its segment start with a merge search in shared memory;
//  * col_idx / vals move as 128-bit streaming loads (evict-first, leaving L2
//    to x) instead of scalar loads (tile.cuh:301-304).
//
// Tile = BLOCK * IPT merge items.  Shared memory per CTA:
//   products  (D+4) * sizeof(P)   |  row sums  D * 8  |  row_ptr window (D+1) * 4
#include "merbit_internal.cuh"

namespace merbit {

template <int BLOCK, int IPT, typename P>
struct SpmvSmem {
    static constexpr int D = BLOCK * IPT;
    static constexpr size_t prod_bytes = ((size_t)(D + 4) * sizeof(P) + 15) & ~(size_t)15;
    static constexpr size_t rows_bytes = (size_t)D * sizeof(double);
    static constexpr size_t rp_bytes = (size_t)(D + 1) * sizeof(int);
    static constexpr size_t bytes = prod_bytes + rows_bytes + rp_bytes;
};

template <int DT, int BLOCK, int IPT, bool VEC, bool RES>
__global__ void __launch_bounds__(BLOCK) spmv_tile_kernel(const SpmvLaunch a) {
    using Pr = Prec<DT>;
    using V = typename Pr::V;
    using X = typename Pr::X;
    using Y = typename Pr::Y;
    using P = typename Pr::P;
    using Acc = typename Pr::Acc;
    using S = SpmvSmem<BLOCK, IPT, P>;
    constexpr int D = S::D;
    constexpr int NW = BLOCK / 32;

    extern __shared__ __align__(16) unsigned char smem[];
    P* s_prod = reinterpret_cast<P*>(smem);
    double* s_rows = reinterpret_cast<double*>(smem + S::prod_bytes);
    int* s_rp = reinterpret_cast<int*>(smem + S::prod_bytes + S::rows_bytes);
    __shared__ int s_tile;
    __shared__ unsigned s_epoch;
    __shared__ double s_carry;
    __shared__ double s_wv[NW];
    __shared__ int s_wf[NW];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;

    if (tid == 0) draw_tile(a.state, &s_tile, &s_epoch);
    __syncthreads();
    const int t = s_tile;
    const unsigned epoch = s_epoch;
    reset_other_parity(a.slots, a.nslots, epoch);
    reset_other_parity(a.xch, a.nslots, epoch);
    if (t >= a.num_tiles) {  // launch bookkeeping out of step: report, touch nothing
        if (tid == 0) {
            atomicExch(&a.state->error, (int)MERBIT_ERR_TIMEOUT);
            finish_launch(a.state, epoch);  // the residual, if any, is not written
        }
        return;
    }

    const int2 c0 = a.coords[t];
    const int2 c1 = a.coords[t + 1];
    const int x0 = c0.x, y0 = c0.y;
    const int nz = c1.x - x0;  // nonzeros in this tile
    const int nr = c1.y - y0;  // rows that end in this tile
    const int L = nr + nz;

    // ---- stage the row_ptr window: s_rp[i] = row_ptr[y0 + i], i in [0, nr]
    for (int i = tid; i <= nr; i += BLOCK) s_rp[i] = __ldg(a.row_ptr + y0 + i);

    // ---- stage products s_prod[g - pbase] = vals[g] * x[col[g]], g in [x0, x0+nz)
    const V* __restrict__ vals = static_cast<const V*>(a.vals);
    const X* __restrict__ xv = static_cast<const X*>(a.x);
    const int* __restrict__ col = a.col;
    const int x1 = x0 + nz;
    const int pbase = VEC ? (x0 & ~3) : x0;
    if (VEC) {
        const int a0 = min((x0 + 3) & ~3, x1);
        const int a1 = max(x1 & ~3, a0);
        if (tid < a0 - x0) {
            const int g = x0 + tid;
            s_prod[g - pbase] = to_p(vals[g]) * (P)__ldg(xv + __ldg(col + g));
        } else if (tid >= 32 && tid - 32 < x1 - a1) {
            const int g = a1 + tid - 32;
            s_prod[g - pbase] = to_p(vals[g]) * (P)__ldg(xv + __ldg(col + g));
        }
        const int nch = (a1 - a0) >> 2;
        constexpr int J = (D / 4 + BLOCK - 1) / BLOCK;
        int4 cc[J];
        P vv[J][4];
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int c = tid + j * BLOCK;
            if (c < nch) {
                const int g = a0 + 4 * c;
                cc[j] = __ldcs(reinterpret_cast<const int4*>(col + g));
                ld4_stream(vals + g, vv[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int c = tid + j * BLOCK;
            if (c < nch) {
                P xg[4];
                xg[0] = (P)__ldg(xv + cc[j].x);
                xg[1] = (P)__ldg(xv + cc[j].y);
                xg[2] = (P)__ldg(xv + cc[j].z);
                xg[3] = (P)__ldg(xv + cc[j].w);
                P pr[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) pr[q] = vv[j][q] * xg[q];
                st4_shared(s_prod + (a0 + 4 * c - pbase), pr);
            }
        }
    } else {
        for (int i = tid; i < nz; i += BLOCK)
            s_prod[i] = to_p(vals[x0 + i]) * (P)__ldg(xv + __ldg(col + x0 + i));
    }
    __syncthreads();

    // ---- this thread's segment of the path: merge search in shared memory.
    // Same predicate as merge_search (include/utils.cuh:17) with the tile's
    // origin subtracted, so segment starts coincide with the global path.
    const int dl = min(tid * IPT, L);
    int lo = max(dl - nz, 0), hi = min(dl, nr);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s_rp[mid + 1] - x0 <= dl - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    int ly = lo, lx = dl - lo;
    const int pofs = x0 - pbase;

    // ---- walk IPT items: a nonzero while lx < end of row ly, else a row end
    Acc acc;
    acc.zero();
    bool has_end = false;
    int first_row = 0;
    double first_val = 0.0;
    int next_end = ly < nr ? s_rp[ly + 1] - x0 : INT_MAX;
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        if (dl + i < L) {
            if (lx >= next_end) {
                const double v = acc.value();
                if (!has_end) {
                    has_end = true;
                    first_row = ly;
                    first_val = v;
                } else {
                    s_rows[ly] = v;
                }
                acc.zero();
                ++ly;
                next_end = ly < nr ? s_rp[ly + 1] - x0 : INT_MAX;
            } else {
                acc.add(s_prod[lx + pofs]);
                ++lx;
            }
        }
    }

    // ---- CTA-wide segmented scan of (has_end, trailing partial).
    // (f1,v1) o (f2,v2) = (f1|f2, f2 ? v2 : v1+v2); fixed order, deterministic.
    int f = has_end;
    double v = acc.value();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double vv = __shfl_up_sync(0xFFFFFFFFu, v, o);
        const int ff = __shfl_up_sync(0xFFFFFFFFu, f, o);
        if (lane >= o) {
            if (!f) v = vv + v;
            f |= ff;
        }
    }
    if (lane == 31) {
        s_wf[warp] = f;
        s_wv[warp] = v;
    }
    __syncthreads();
    int pf = 0;
    double pv = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        if (w < warp) {
            if (s_wf[w]) {
                pv = s_wv[w];
                pf = 1;
            } else {
                pv = pv + s_wv[w];
            }
        }
    }
    double ev = __shfl_up_sync(0xFFFFFFFFu, v, 1);
    int ef = __shfl_up_sync(0xFFFFFFFFu, f, 1);
    if (lane == 0) {
        ev = 0.0;
        ef = 0;
    }
    const double excl = ef ? ev : pv + ev;
    (void)pf;
    if (has_end) s_rows[first_row] = excl + first_val;

    // ---- publish this tile's carry: the partial sum of its trailing row
    if (tid == BLOCK - 1) publish_carry(a.slots, a.nslots, epoch, t, f ? v : pv + v);

    // ---- decoupled look-back for the tile's first row when it began in an
    // earlier tile and ends here.  Earlier tiles are summed in a fixed order
    // (32 per step, butterfly reduction) so the result does not depend on
    // timing.
    const bool need_lb = nr > 0 && s_rp[0] < x0;
    if (need_lb && warp == 0) {
        const double total = look_back(a.coords, a.slots, a.nslots, epoch, a.state, t, s_rp[0], lane);
        if (lane == 0) s_carry = total;
    }
    __syncthreads();

    // ---- write the rows that end in this tile, coalesced
    RowStore<Y, RES> out(a);
    for (int i = tid; i < nr; i += BLOCK) {
        double r = s_rows[i];
        if (i == 0 && need_lb) r = s_carry + r;
        out(y0 + i, r);
    }

    if (RES)
        finish_launch_residual<NW>(a.state, epoch, out.res, a.partials, t, a.num_tiles,
                                   a.residual);
    else if (tid == 0)
        finish_launch(a.state, epoch);
}

// ---------------------------------------------------------------------------
// Configuration table.  kind 0 = this CTA-tile kernel (tile = block*ipt
// items), kind 1 = the warp-tile kernel of spmv_warp.cu (tile = 32*ipt items,
// block/32 warps per CTA, needs 16-byte aligned col_idx/vals), kind 3 = the
// row-group kernel of spmv_rows.cu (ipt = lanes per row, no tiles).
// ---------------------------------------------------------------------------
namespace {
// Items per thread are odd: a lane's segment then starts an odd number of
// elements after its neighbour's, which spreads the lanes of a warp over
// all shared-memory banks when they walk their segments in step.
// stages: shared-memory stages per warp of the warp-tile kernel (the kernel
// also runs 2, which measured slower: less occupancy and less L1).
// Order matters only for the default pick (the first usable entry): the
// large-L1 warp-tile entries come first because they are the better choice
// for irregular matrices; plan_tune picks per matrix.
constexpr SpmvConfig kCfgF64[] = {
    {1, 256, 15, 1, kCarveoutL1, 1}, {1, 128, 15, 1, kCarveoutL1, 1},
    {1, 256, 11, 1, kCarveoutL1, 1}, {1, 128, 15, 1, kCarveoutL1Max, 1},
    {1, 256, 15, 1, kCarveoutL1, 0}, {1, 256, 15, 1, 0, 0},
    {1, 128, 15, 1, 0, 0},           {1, 256, 11, 1, 0, 0},
    {1, 256, 7, 1, 0, 0},            {1, 128, 23, 1, 0, 0},
    {0, 256, 7, 1, 0, 0},            {0, 256, 11, 1, 0, 0},
    {0, 128, 9, 1, 0, 0},
    {3, 256, 4, 1, 0, 0},            {3, 256, 8, 1, 0, 0},
    {3, 256, 16, 1, 0, 0},           {3, 256, 32, 1, 0, 0},
    {3, 256, 8, 1, 0, 1},            {3, 256, 16, 1, 0, 1},
    {3, 256, 2, 1, 0, 0},            {3, 256, 4, 1, 0, 0, 1},
    {3, 256, 2, 1, 0, 0, 1},         {3, 256, 8, 1, 0, 0, 1},
    {3, 256, 1, 1, 0, 0, 1},
    // warp tiles added later (appended, so earlier indices stay): 13 items
    // per lane (4 CTAs of 8 warps at the 72% carveout in FP64), and tiles
    // with a row_ptr window for every item (stg = 1: no rows-per-tile cap),
    // with L1 gathers at a 58% carveout for matrices whose columns repeat
    {1, 256, 13, 1, kCarveoutL1, 1},  {1, 256, 11, 1, kCarveoutL1Max, 0, 1},
    {1, 256, 15, 1, kCarveoutL1Max, 0, 1}, {1, 256, 11, 1, kCarveoutL1, 1, 1}};
constexpr SpmvConfig kCfgF32[] = {
    {1, 256, 15, 1, kCarveoutL1, 1}, {1, 128, 15, 1, kCarveoutL1, 1},
    {1, 256, 11, 1, kCarveoutL1, 1}, {1, 128, 15, 1, kCarveoutL1Max, 1},
    {1, 256, 15, 1, kCarveoutL1, 0}, {1, 256, 15, 1, 0, 0},
    {1, 128, 15, 1, 0, 0},           {1, 256, 11, 1, 0, 0},
    {1, 256, 7, 1, 0, 0},            {1, 128, 23, 1, 0, 0},
    {0, 256, 11, 1, 0, 0},           {0, 256, 7, 1, 0, 0},
    {0, 256, 15, 1, 0, 0},
    {3, 256, 4, 1, 0, 0},            {3, 256, 8, 1, 0, 0},
    {3, 256, 16, 1, 0, 0},           {3, 256, 32, 1, 0, 0},
    {3, 256, 8, 1, 0, 1},            {3, 256, 16, 1, 0, 1},
    {3, 256, 2, 1, 0, 0},            {3, 256, 4, 1, 0, 0, 1},
    {3, 256, 2, 1, 0, 0, 1},         {3, 256, 8, 1, 0, 0, 1},
    {3, 256, 1, 1, 0, 0, 1},
    // warp tiles added later (appended, so earlier indices stay): 13 items
    // per lane (4 CTAs of 8 warps at the 72% carveout in FP64), and tiles
    // with a row_ptr window for every item (stg = 1: no rows-per-tile cap),
    // with L1 gathers at a 58% carveout for matrices whose columns repeat
    {1, 256, 13, 1, kCarveoutL1, 1},  {1, 256, 11, 1, kCarveoutL1Max, 0, 1},
    {1, 256, 15, 1, kCarveoutL1Max, 0, 1}, {1, 256, 11, 1, kCarveoutL1, 1, 1}};

template <int DT, int BLOCK, int IPT, bool VEC, bool RES>
int launch_one_k(const SpmvLaunch& a, cudaStream_t s) {
    using P = typename Prec<DT>::P;
    constexpr size_t smem = SpmvSmem<BLOCK, IPT, P>::bytes;
    // per device ordinal; threads that race here set the same attribute
    static int attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return fail(MERBIT_ERR_UNSUPPORTED, "spmv: device ordinal >= 64");
    if (!__atomic_load_n(&attr_set[dev], __ATOMIC_ACQUIRE)) {
        cudaError_t e = cudaFuncSetAttribute(spmv_tile_kernel<DT, BLOCK, IPT, VEC, RES>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(spmv)");
        __atomic_store_n(&attr_set[dev], 1, __ATOMIC_RELEASE);
    }
    spmv_tile_kernel<DT, BLOCK, IPT, VEC, RES><<<a.num_tiles, BLOCK, smem, s>>>(a);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? (int)MERBIT_OK : cuda_fail(e, "spmv_tile_kernel launch");
}

template <int DT, int BLOCK, int IPT, bool VEC>
int launch_one(const SpmvLaunch& a, cudaStream_t s) {
    if (a.residual && !a.partials) return fail(MERBIT_ERR_INVALID, "spmv: residual without partials");
    return a.residual ? launch_one_k<DT, BLOCK, IPT, VEC, true>(a, s)
                      : launch_one_k<DT, BLOCK, IPT, VEC, false>(a, s);
}

template <int DT, int BLOCK, int IPT>
int launch_vec(bool vec, const SpmvLaunch& a, cudaStream_t s) {
    return vec ? launch_one<DT, BLOCK, IPT, true>(a, s) : launch_one<DT, BLOCK, IPT, false>(a, s);
}

template <int DT>
int launch_cta(int block, int ipt, bool vec, const SpmvLaunch& a, cudaStream_t s) {
    if (block == 256 && ipt == 7) return launch_vec<DT, 256, 7>(vec, a, s);
    if (block == 256 && ipt == 11) return launch_vec<DT, 256, 11>(vec, a, s);
    if (block == 128 && ipt == 9) return launch_vec<DT, 128, 9>(vec, a, s);
    if (block == 256 && ipt == 5) return launch_vec<DT, 256, 5>(vec, a, s);
    if (block == 256 && ipt == 15) return launch_vec<DT, 256, 15>(vec, a, s);
    if (block == 128 && ipt == 11) return launch_vec<DT, 128, 11>(vec, a, s);
    return fail(MERBIT_ERR_INVALID, "spmv: no such configuration");
}
}  // namespace

int spmv_num_configs(int dtype) {
    return dtype == MERBIT_F64 ? (int)(sizeof(kCfgF64) / sizeof(kCfgF64[0]))
                               : (int)(sizeof(kCfgF32) / sizeof(kCfgF32[0]));
}

SpmvConfig spmv_config(int dtype, int idx) {
    return dtype == MERBIT_F64 ? kCfgF64[idx] : kCfgF32[idx];
}

// kind 3 has no merge-path tiles (0: no partition to build)
int spmv_tile_items(const SpmvConfig& c) {
    return c.kind == 3 ? 0 : c.kind == 1 ? 32 * c.ipt : c.block * c.ipt;
}

bool spmv_config_allowed(const SpmvConfig& c, bool vec) { return vec || c.kind == 0 || c.kind == 3; }

int spmv_config_row_cap(const SpmvConfig& c) {
    // warp tiles with stg = 1 stage a row_ptr window for every item of the tile
    return c.kind == 1 && !c.stg ? warp_rp_cap(c.ipt) - 8 : INT_MAX;
}


int spmv_warp_launch(int dtype, const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s);
int spmv_rows_launch(int dtype, const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s);

int spmv_launch(int dtype, int cfg, bool vec, const SpmvLaunch& a, cudaStream_t s) {
    const SpmvConfig c = spmv_config(dtype, cfg);
    if (c.kind == 3) return spmv_rows_launch(dtype, c, a, s);  // no tiles
    if (a.num_tiles <= 0) return MERBIT_OK;
    if (!spmv_config_allowed(c, vec)) return fail(MERBIT_ERR_INVALID, "spmv: config needs aligned arrays");
    if (c.kind != 0) return spmv_warp_launch(dtype, c, a, s);
    switch (dtype) {
    case MERBIT_F64: return launch_cta<MERBIT_F64>(c.block, c.ipt, vec, a, s);
    case MERBIT_F32: return launch_cta<MERBIT_F32>(c.block, c.ipt, vec, a, s);
    case MERBIT_BF16: return launch_cta<MERBIT_BF16>(c.block, c.ipt, vec, a, s);
    }
    return fail(MERBIT_ERR_INVALID, "spmv: bad dtype");
}

}  // namespace merbit
