// Warp-tile merge-path SpMV for sm_100a:  y = alpha * A x + beta * y.
//
// Each warp owns tiles of 32*IPT merge items (row ends + nonzeros) and runs
// each start to finish with no CTA-wide barrier:
//
//   1. lane 0 issues bulk async copies (cp.async.bulk through the TMA
//      engine, L2 evict-first) of the tile's row_ptr window, col_idx slice
//      and vals slice into one of the warp's STAGES shared-memory stages,
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

#include "merbit_internal.cuh"

namespace merbit {

constexpr size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// One stage of a warp: row_ptr window (warp_rp_cap entries: the plan only
// runs this configuration when no tile ends more rows than fit), col slice
// and value slice (W + rounding), one mbarrier.  Completed rows are staged
// for the coalesced write in whichever slice is dead after the products are
// formed: the col slice when products overwrite the values, the value slice
// when they overwrite the columns (bf16); rows beyond OUTCAP go straight to y.
template <typename V, typename P, int IPT>
struct WarpSmem {
    static constexpr int W = 32 * IPT;
    static constexpr int CAP = W + 32;  // slice + rounding on both sides
    static constexpr size_t rp_bytes = align16((size_t)warp_rp_cap(IPT) * 4);
    static constexpr size_t col_bytes = align16((size_t)CAP * 4);
    static constexpr size_t val_bytes = align16((size_t)CAP * sizeof(V));
    static constexpr bool prod_in_val = sizeof(P) == sizeof(V);
    static constexpr size_t out_offset = prod_in_val ? rp_bytes : rp_bytes + col_bytes;
    static constexpr int OUTCAP_ = (int)((prod_in_val ? col_bytes : val_bytes) / 8);
    static constexpr int OUTCAP = OUTCAP_ < 256 ? OUTCAP_ : 256;
    static constexpr size_t bar_offset = rp_bytes + col_bytes + val_bytes;
    static constexpr size_t bytes = bar_offset + 16;
};

// Bytes the bulk part of stage_range moves for [s, e) of an n-element array
// with G elements per 16 bytes.
__device__ __forceinline__ unsigned bulk_bytes(int s, int e, int n, int G, int esz) {
    if (e <= s) return 0u;
    const int base = s & ~(G - 1), lim = n & ~(G - 1);
    const int b_end = min((e + G - 1) & ~(G - 1), lim);
    return b_end > base ? (unsigned)(b_end - base) * (unsigned)esz : 0u;
}

// Copies global elements [s, e) of an array of n elements into stage
// memory at index (g - floor(s)).  The bulk part covers [floor(s),
// min(ceil(e), floor(n))) in 16-byte granules; elements beyond floor(n)
// (only at the end of the array) are loaded by lanes.
template <typename T>
__device__ __forceinline__ void stage_range(T* dst, const T* src, int s, int e, int n,
                                            uint64_t* bar, uint64_t pol, int lane) {
    constexpr int G = 16 / (int)sizeof(T);
    if (e <= s) return;
    const int base = s & ~(G - 1);
    const int lim = n & ~(G - 1);
    const int b_end = min((e + G - 1) & ~(G - 1), lim);
    if (b_end > base && lane == 0)
        bulk_g2s(dst, src + base, (unsigned)(b_end - base) * (unsigned)sizeof(T), bar, pol);
    const int p0 = max(b_end, s);
    if (lane < e - p0) dst[p0 + lane - base] = src[p0 + lane];
}

// Boundary slot swap: deposits `mine` in slot t and returns what was there
// (kEmpty if this side arrived first).
__device__ __forceinline__ unsigned long long swap_boundary(unsigned long long* xch, int nslots,
                                                            unsigned epoch, int t, double mine) {
    unsigned long long b = (unsigned long long)__double_as_longlong(mine);
    if (b == kEmpty) b = 0x7FF8000000000000ull;
    return atomicExch(xch + (size_t)(epoch & 1u) * nslots + t, b);
}

// A boundary swap whose result is read one tile later, so the atomic's
// round trip overlaps the next tile instead of stalling the warp.
struct PendingSwap {
    unsigned long long got;  // what the swap returned (kEmpty: other side not there yet)
    double mine;
    int row;      // -1: nothing pending
    int carry;    // 1: `mine` is the carry (earlier tile), 0: the head (later tile)
};

template <class RS>
__device__ __forceinline__ void resolve_swap(PendingSwap& p, RS& out) {
    if (p.row >= 0 && p.got != kEmpty) {
        const double other = __longlong_as_double((long long)p.got);
        // always carry + head, whichever side finishes the row
        out(p.row, p.carry ? p.mine + other : other + p.mine);
    }
    p.row = -1;
}

// A row that began two or more tiles before the tile that completes it:
// its carry-in is the sum of the carries of the tiles in between, which run
// on other warps at about the same time.  Its look-back is queued and taken
// later (when the queue is full, else after the warp's last tile), so the
// warp does not wait for those tiles while it still has tiles to process.
struct LookBack {
    double head;  // the completing tile's part of the row
    int row, u, rs;
};
constexpr int kLookBackQueue = 8;

template <class RS>
__device__ __forceinline__ void drain_look_backs(const SpmvLaunch& a, unsigned epoch,
                                                 const LookBack* q, int n, int lane, RS& out) {
    for (int i = 0; i < n; ++i) {
        const LookBack e = q[i];
        const double total = look_back(a.coords, a.slots, a.nslots, epoch, a.state, e.u, e.rs, lane);
        if (lane == 0) out(e.row, total + e.head);
    }
    __syncwarp();
}

// x gather: through L1 (ld.global.nc), or, CG, cached in L2 only (no L1
// line is allocated, which leaves L1 to other gathers in flight; better when
// x has no reuse within an SM).
template <bool CG, typename T>
__device__ __forceinline__ T gather_x(const T* p) {
    return CG ? __ldcg(p) : __ldg(p);
}

template <int DT, int IPT, bool CG = false>
struct WarpTile {
    using Pr = Prec<DT>;
    using V = typename Pr::V;
    using X = typename Pr::X;
    using Y = typename Pr::Y;
    using P = typename Pr::P;
    using Acc = typename Pr::Acc;
    using S = WarpSmem<V, P, IPT>;
    static constexpr int GV = 16 / (int)sizeof(V);
    static constexpr int kOutCap = S::OUTCAP;

    // Issues the copies of tile u into stage `ws`; lane 0 arms the barrier
    // with the byte count before any copy is issued.
    static __device__ __forceinline__ void issue(const SpmvLaunch& a, int u, unsigned char* ws,
                                                 uint64_t* bar, int lane) {
        const int2 c0 = a.coords[u];
        const int2 c1 = a.coords[u + 1];
        int* s_rp = reinterpret_cast<int*>(ws);
        int* s_col = reinterpret_cast<int*>(ws + S::rp_bytes);
        V* s_val = reinterpret_cast<V*>(ws + S::rp_bytes + S::col_bytes);
        const V* vals = static_cast<const V*>(a.vals);
        const int nrp = a.nrow + 1;
        const unsigned tot = bulk_bytes(c0.y, c1.y + 1, nrp, 4, 4) +
                             bulk_bytes(c0.x, c1.x, a.nnz, 4, 4) +
                             bulk_bytes(c0.x, c1.x, a.nnz, GV, (int)sizeof(V));
        __syncwarp();
        if (lane == 0) {
            // order this warp's earlier generic accesses of the stage before
            // the async-proxy writes that are about to overwrite it
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive_expect_tx(bar, tot);
        }
        const uint64_t pol = l2_evict_first_policy();
        stage_range<int>(s_rp, a.row_ptr, c0.y, c1.y + 1, nrp, bar, pol, lane);
        stage_range<int>(s_col, a.col, c0.x, c1.x, a.nnz, bar, pol, lane);
        stage_range<V>(s_val, vals, c0.x, c1.x, a.nnz, bar, pol, lane);
    }

    // Processes tile u from stage `ws` (its copies complete).
    template <class RS>
    static __device__ __forceinline__ void process(const SpmvLaunch& a, int u, unsigned epoch,
                                                   unsigned char* ws, int lane,
                                                   PendingSwap& pa, PendingSwap& pb, RS& out,
                                                   LookBack* lbq, int& nlb) {
        const int* s_rp = reinterpret_cast<const int*>(ws);
        const int* s_col = reinterpret_cast<const int*>(ws + S::rp_bytes);
        const V* s_val = reinterpret_cast<const V*>(ws + S::rp_bytes + S::col_bytes);
        double* s_out = reinterpret_cast<double*>(ws + S::out_offset);

        const int2 c0 = a.coords[u];
        const int2 c1 = a.coords[u + 1];
        const int prev_x = u > 0 ? a.coords[u - 1].x : 0;
        const int x0 = c0.x, y0 = c0.y, x1 = c1.x, y1 = c1.y;
        const int nz = x1 - x0, nr = y1 - y0, L = nz + nr;
        const int rp_base = y0 & ~3, col_base = x0 & ~3, val_base = x0 & ~(GV - 1);
        const int rpo0 = y0 - rp_base;  // staged index of row_ptr[y0]

        // ---- tile inside one row (no row ends: the common case for long rows
        // of power-law matrices, the reference's fast_track,
        // include/tile.cuh:267-290): the tile's partial is just the sum of
        // its products -- lane sums in a fixed order, then a butterfly.
        if (nr == 0) {
            const X* __restrict__ xv = static_cast<const X*>(a.x);
            X xg[IPT];
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int i = lane + 32 * j;
                xg[j] = i < nz ? gather_x<CG>(xv + s_col[x0 + i - col_base]) : (X)0;
            }
            Acc acc;
            acc.zero();
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int i = lane + 32 * j;
                if (i < nz) acc.add(to_p(s_val[x0 + i - val_base]) * (P)xg[j]);
            }
            double v = acc.value();
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            resolve_swap(pa, out);
            resolve_swap(pb, out);
            if (lane == 31) {
                publish_carry(a.slots, a.nslots, epoch, u, v);
                // the row may have begun in this tile and end in the next
                const int rs1 = s_rp[rpo0];
                if (y1 < a.nrow && u + 1 < a.num_tiles && rs1 >= x0 && rs1 < x1) {
                    pa.got = swap_boundary(a.xch, a.nslots, epoch, u + 1, v);
                    pa.mine = v;
                    pa.row = y1;
                    pa.carry = 1;
                }
            }
            return;
        }

        // ---- products, in place of the staged values (or of col when the
        // product is wider than a value)
        P* s_prod;
        int pbase;
        if (sizeof(P) == sizeof(V)) {
            s_prod = reinterpret_cast<P*>(ws + S::rp_bytes + S::col_bytes);
            pbase = val_base;
        } else {
            s_prod = reinterpret_cast<P*>(ws + S::rp_bytes);
            pbase = col_base;
        }
        {
            const X* __restrict__ xv = static_cast<const X*>(a.x);
            int cidx[IPT];
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int i = lane + 32 * j;
                cidx[j] = i < nz ? s_col[x0 + i - col_base] : 0;
            }
            X xg[IPT];
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int i = lane + 32 * j;
                xg[j] = i < nz ? gather_x<CG>(xv + cidx[j]) : (X)0;
            }
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int i = lane + 32 * j;
                if (i < nz) {
                    const int g = x0 + i;
                    s_prod[g - pbase] = to_p(s_val[g - val_base]) * (P)xg[j];
                }
            }
        }
        __syncwarp();

        // ---- this lane's segment: merge search in the staged row_ptr window
        const int rpo = y0 - rp_base;
        const int pofs = x0 - pbase;
        const int dl = min(lane * IPT, L);
        int lo = max(dl - nz, 0), hi = min(dl, nr);
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s_rp[rpo + mid + 1] - x0 <= dl - mid - 1)
                lo = mid + 1;
            else
                hi = mid;
        }
        int ly = lo, lx = dl - lo;

        // ---- walk IPT items: predicated steps, completed rows staged
        Acc acc;
        acc.zero();
        int first_row = -1;
        double first_val = 0.0;
        int next_end = ly < nr ? s_rp[rpo + ly + 1] - x0 : INT_MAX;
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const bool valid = dl + i < L;
            const bool is_end = valid && lx >= next_end;
            const P p = (valid && !is_end) ? s_prod[pofs + lx] : (P)0;
            if (is_end) {
                const double v = acc.value();
                if (first_row < 0) {
                    first_row = ly;
                    first_val = v;
                } else if (ly < kOutCap) {
                    s_out[ly] = v;
                } else {
                    out(y0 + ly, v);
                }
                acc.zero();
                ++ly;
                next_end = ly < nr ? s_rp[rpo + ly + 1] - x0 : INT_MAX;
            }
            acc.add(p);
            lx += (valid && !is_end) ? 1 : 0;
        }

        // ---- warp segmented scan of (has_end, trailing partial)
        int f = first_row >= 0;
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
        double ev = __shfl_up_sync(0xFFFFFFFFu, v, 1);
        if (lane == 0) ev = 0.0;
        const int rs = s_rp[rpo];           // start of row y0
        const bool need_lb = nr > 0 && rs < x0;
        const double rv = ev + first_val;   // this lane's first completed row
        const bool holds_first = first_row == 0 && need_lb;
        if (first_row >= 0 && !holds_first) {
            if (first_row < kOutCap)
                s_out[first_row] = rv;
            else
                out(y0 + first_row, rv);
        }

        // ---- trailing partial of row y1: published for long-row look-backs,
        // swapped with tile u+1 when row y1 began in this tile
        resolve_swap(pa, out);  // the previous tile's swaps
        resolve_swap(pb, out);
        if (lane == 31) {
            publish_carry(a.slots, a.nslots, epoch, u, v);
            if (y1 < a.nrow && u + 1 < a.num_tiles) {
                const int rs1 = s_rp[rpo + nr];  // start of row y1
                if (rs1 >= x0 && rs1 < x1) {
                    pa.got = swap_boundary(a.xch, a.nslots, epoch, u + 1, v);
                    pa.mine = v;
                    pa.row = y1;
                    pa.carry = 1;
                }
            }
        }
        __syncwarp();

        // ---- coalesced write of the staged rows (row 0 of a split row is
        // finished below)
        const int nst = min(nr, kOutCap);
        for (int r = lane; r < nst; r += 32)
            if (!(r == 0 && need_lb)) out(y0 + r, s_out[r]);

        // ---- row y0 when it began in an earlier tile
        if (need_lb) {
            if (prev_x <= rs) {
                // began in tile u-1: swap with it, the later side writes
                if (holds_first) {
                    pb.got = swap_boundary(a.xch, a.nslots, epoch, u, rv);
                    pb.mine = rv;
                    pb.row = y0;
                    pb.carry = 0;
                }
            } else {
                if (nlb == kLookBackQueue) {  // warp-uniform
                    drain_look_backs(a, epoch, lbq, nlb, lane, out);
                    nlb = 0;
                }
                if (holds_first) {
                    LookBack e;
                    e.head = rv;
                    e.row = y0;
                    e.u = u;
                    e.rs = rs;
                    lbq[nlb] = e;
                }
                ++nlb;
                __syncwarp();
            }
        }
    }
};

// CV: the shared-memory carveout the kernel is launched with (it does not
// change the code; each split gets its own function and function attribute).
template <int DT, int WARPS, int IPT, int STAGES, bool RES, bool CG, int CV>
__global__ void __launch_bounds__(WARPS * 32) spmv_warp_kernel(const SpmvLaunch a) {
    using T = WarpTile<DT, IPT, CG>;
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
    int u = (int)blockIdx.x * WARPS + warp;
    if (u < a.num_tiles)
        T::issue(a, u, wbase, reinterpret_cast<uint64_t*>(wbase + S::bar_offset), lane);
    int k = 0;
    for (; u < a.num_tiles; u += nw) {
        const int un = u + nw;
        unsigned char* cur = wbase + (size_t)k * S::bytes;
        uint64_t* cbar = reinterpret_cast<uint64_t*>(cur + S::bar_offset);
        if (STAGES == 2 && un < a.num_tiles) {
            unsigned char* nxt = wbase + (size_t)(k ^ 1) * S::bytes;
            T::issue(a, un, nxt, reinterpret_cast<uint64_t*>(nxt + S::bar_offset), lane);
        }
        const bool ok =
            __all_sync(0xFFFFFFFFu, mbar_wait_bounded(cbar, (phases >> k) & 1u, a.state));
        phases ^= 1u << k;
        __syncwarp();
        if (ok) T::process(a, u, epoch, cur, lane, pa, pb, out, s_lbq[warp], nlb);
        if (STAGES == 1) {
            if (un < a.num_tiles) T::issue(a, un, cur, cbar, lane);
        } else {
            k ^= 1;
        }
    }
    resolve_swap(pa, out);
    resolve_swap(pb, out);
    drain_look_backs(a, epoch, s_lbq[warp], nlb, lane, out);
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

template <int DT, int WARPS, int IPT, int STAGES, bool RES, bool CG, int CV>
int launch_warp_k(const SpmvLaunch& a, cudaStream_t s) {
    using S = typename WarpTile<DT, IPT, CG>::S;
    static int grid_cap[64] = {};
    if (RES && !a.partials) return fail(MERBIT_ERR_INVALID, "spmv_warp: residual without partials");
    return launch_coop(spmv_warp_kernel<DT, WARPS, IPT, STAGES, RES, CG, CV>, WARPS,
                       S::bytes * WARPS * STAGES, CV, grid_cap, a, s, "spmv_warp_kernel");
}

template <int DT, int WARPS, int IPT, int STAGES, bool CG, int CV>
int launch_warp(const SpmvLaunch& a, cudaStream_t s) {
    return a.residual ? launch_warp_k<DT, WARPS, IPT, STAGES, true, CG, CV>(a, s)
                      : launch_warp_k<DT, WARPS, IPT, STAGES, false, CG, CV>(a, s);
}

// The (warps, items per thread, gather hint, carveout) combinations of the
// configuration tables in spmv.cu.
template <int DT>
int launch_warp_dt(const SpmvConfig& c, const SpmvLaunch& a, cudaStream_t s) {
    const int warps = c.block / 32, ipt = c.ipt;
    if (c.stages != 1) return fail(MERBIT_ERR_INVALID, "spmv_warp: no such configuration");
#define MERBIT_WARP_CASE(W, I, G, C)                                                   \
    if (warps == W && ipt == I && c.cg == G && c.carveout == C)                        \
        return launch_warp<DT, W, I, 1, G, C>(a, s);
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
#undef MERBIT_WARP_CASE
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
