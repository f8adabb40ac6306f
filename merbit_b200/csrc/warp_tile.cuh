// Warp-tile merge-path machinery shared by the SpMV kernel (spmv_warp.cu)
// and the batched k = 1 kernel (batch_warp.cu): stage layout, TMA bulk
// staging, boundary swaps, the look-back queue and the per-tile walk
// (WarpTile).  The description of the algorithm is at the top of
// spmv_warp.cu.
//
// A WarpTile reads its matrix through a source object Src with
//   coord(u)        merge-path coordinates of local tile u (int2)
//   row_ptr(), col(), vals(), x(), nrow(), nnz(), num_tiles()
//   slots(), xch(), nslots(), state()   the launch's slot arrays and state
//   slot_base()     slot index of local tile 0
// so that one tile walk serves a single matrix and the matrices of a batch.
#pragma once

#include <type_traits>

#include "merbit_internal.cuh"

namespace merbit {

constexpr size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Products per TwoSum step with compensated (FP32/BF16) accumulation: on a
// single-row tile a block of 4 is summed by f32 fused multiply-adds, on the
// walk the products of 4 steps are summed in f32; either way a block costs
// at most 4 roundings of its sum |a x| and is then added exactly.
template <class Acc>
constexpr int kWarpBlockSum = std::is_same<Acc, AccTwoSum>::value ? 4 : 1;

// One stage of a warp: row_ptr window (RP entries; warp_rp_cap(IPT) by
// default -- the plan only runs such a configuration when no tile ends more
// rows than fit), col slice and value slice (W + rounding), one mbarrier.
// Completed rows are staged for the coalesced write in whichever slice is
// dead after the products are formed: the col slice when products
// overwrite the values, the value slice when they overwrite the columns
// (bf16); rows beyond OUTCAP go straight to y.  W is the largest tile the
// stage holds (a batch sizes one stage for the largest items per lane of
// its matrices).
template <typename V, typename P, int IPT, int RP = warp_rp_cap(IPT)>
struct WarpSmem {
    static constexpr int W = 32 * IPT;
    static constexpr int CAP = W + 32;  // slice + rounding on both sides
    static constexpr size_t rp_bytes = align16((size_t)RP * 4);
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

template <class Src, class RS>
__device__ __forceinline__ void drain_look_backs(const Src& src, unsigned epoch,
                                                 const LookBack* q, int n, int lane, RS& out) {
    for (int i = 0; i < n; ++i) {
        const LookBack e = q[i];
        const double total = look_back(src.coords(), src.slots(), src.nslots(), epoch, src.state(),
                                       e.u, e.rs, lane, src.slot_base());
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

// One warp tile of IPT items per lane.  Src is where the tile's matrix comes
// from: its arrays, its partition (local tile indices u), the carry / swap
// slot arrays of the launch and the slot of its local tile 0 (slot_base);
// SS the stage layout (the default, or one sized for a batch's largest IPT).
template <int DT, int IPT, bool CG = false,
          class SS = WarpSmem<typename Prec<DT>::V, typename Prec<DT>::P, IPT>>
struct WarpTile {
    using Pr = Prec<DT>;
    using V = typename Pr::V;
    using X = typename Pr::X;
    using Y = typename Pr::Y;
    using P = typename Pr::P;
    using Acc = typename Pr::Acc;
    using S = SS;
    static_assert(32 * IPT <= S::W, "stage smaller than the tile");
    static constexpr int GV = 16 / (int)sizeof(V);
    static constexpr int kOutCap = S::OUTCAP;
    // single-row tiles with compensated (TwoSum) accumulation: products
    // enter in blocks of this many, fused in f32 (1: one TwoSum each)
    static constexpr int kBlockSum = kWarpBlockSum<Acc>;

    // Issues the copies of tile u into stage `ws`; lane 0 arms the barrier
    // with the byte count before any copy is issued.
    template <class Src>
    static __device__ __forceinline__ void issue(const Src& src, int u, unsigned char* ws,
                                                 uint64_t* bar, int lane) {
        const int2 c0 = src.coord(u);
        const int2 c1 = src.coord(u + 1);
        int* s_rp = reinterpret_cast<int*>(ws);
        int* s_col = reinterpret_cast<int*>(ws + S::rp_bytes);
        V* s_val = reinterpret_cast<V*>(ws + S::rp_bytes + S::col_bytes);
        const V* vals = static_cast<const V*>(src.vals());
        const int nnz = src.nnz();
        const int nrp = src.nrow() + 1;
        // a tile inside one row stages no row_ptr window (process reads its
        // one entry, row_ptr[y0], from global memory)
        const bool single = c0.y == c1.y;
        const unsigned tot = (single ? 0u : bulk_bytes(c0.y, c1.y + 1, nrp, 4, 4)) +
                             bulk_bytes(c0.x, c1.x, nnz, 4, 4) +
                             bulk_bytes(c0.x, c1.x, nnz, GV, (int)sizeof(V));
        __syncwarp();
        if (lane == 0) {
            // order this warp's earlier generic accesses of the stage before
            // the async-proxy writes that are about to overwrite it
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive_expect_tx(bar, tot);
        }
        const uint64_t pol = l2_evict_first_policy();
        if (!single) stage_range<int>(s_rp, src.row_ptr(), c0.y, c1.y + 1, nrp, bar, pol, lane);
        stage_range<int>(s_col, src.col(), c0.x, c1.x, nnz, bar, pol, lane);
        stage_range<V>(s_val, vals, c0.x, c1.x, nnz, bar, pol, lane);
    }

    // Processes tile u from stage `ws` (its copies complete).
    template <class Src, class RS>
    static __device__ __forceinline__ void process(const Src& src, int u, unsigned epoch,
                                                   unsigned char* ws, int lane,
                                                   PendingSwap& pa, PendingSwap& pb, RS& out,
                                                   LookBack* lbq, int& nlb) {
        const int* s_rp = reinterpret_cast<const int*>(ws);
        const int* s_col = reinterpret_cast<const int*>(ws + S::rp_bytes);
        const V* s_val = reinterpret_cast<const V*>(ws + S::rp_bytes + S::col_bytes);
        double* s_out = reinterpret_cast<double*>(ws + S::out_offset);

        const int2 c0 = src.coord(u);
        const int2 c1 = src.coord(u + 1);
        const int prev_x = u > 0 ? src.coord(u - 1).x : 0;
        const int x0 = c0.x, y0 = c0.y, x1 = c1.x, y1 = c1.y;
        const int nz = x1 - x0, nr = y1 - y0, L = nz + nr;
        const int rp_base = y0 & ~3, col_base = x0 & ~3, val_base = x0 & ~(GV - 1);

        // ---- tile inside one row (no row ends: the common case for long rows
        // of power-law matrices, the reference's fast_track,
        // include/tile.cuh:267-290): the tile's partial is just the sum of
        // its products -- lane sums in a fixed order, then a butterfly.
        if (nr == 0) {
            // start of row y0 (not staged for a single-row tile), loaded now
            // so that it arrives while the gathers are in flight
            const int rs1 = lane == 31 ? __ldg(src.row_ptr() + y0) : 0;
            const X* __restrict__ xv = static_cast<const X*>(src.x());
            X xg[IPT];
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int i = lane + 32 * j;
                xg[j] = i < nz ? gather_x<CG>(xv + s_col[x0 + i - col_base]) : (X)0;
            }
            Acc acc;
            acc.zero();
            if constexpr (kBlockSum > 1) {
                // blocks of kBlockSum products summed by fused multiply-adds,
                // each block added to (s, c) by TwoSum
#pragma unroll
                for (int j0 = 0; j0 < IPT; j0 += kBlockSum) {
                    P blk = (P)0;
#pragma unroll
                    for (int j = j0; j < j0 + kBlockSum && j < IPT; ++j) {
                        const int i = lane + 32 * j;
                        if (i < nz) blk = fmaf(to_p(s_val[x0 + i - val_base]), (P)xg[j], blk);
                    }
                    acc.add(blk);
                }
            } else {
#pragma unroll
                for (int j = 0; j < IPT; ++j) {
                    const int i = lane + 32 * j;
                    if (i < nz) acc.add(to_p(s_val[x0 + i - val_base]) * (P)xg[j]);
                }
            }
            double v = acc.value();
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            resolve_swap(pa, out);
            resolve_swap(pb, out);
            if (lane == 31) {
                publish_carry(src.slots(), src.nslots(), epoch, src.slot_base() + u, v);
                // the row may have begun in this tile and end in the next
                if (y1 < src.nrow() && u + 1 < src.num_tiles() && rs1 >= x0 && rs1 < x1) {
                    pa.got = swap_boundary(src.xch(), src.nslots(), epoch, src.slot_base() + u + 1, v);
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
            const X* __restrict__ xv = static_cast<const X*>(src.x());
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
        // (compensated accumulation: the products of every kBlockSum steps
        // are summed in f32 and added by one TwoSum; a row end adds the
        // open block's sum in double)
        Acc acc;
        acc.zero();
        P blk = (P)0;
        int first_row = -1;
        double first_val = 0.0;
        int next_end = ly < nr ? s_rp[rpo + ly + 1] - x0 : INT_MAX;
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const bool valid = dl + i < L;
            const bool is_end = valid && lx >= next_end;
            const P p = (valid && !is_end) ? s_prod[pofs + lx] : (P)0;
            if (is_end) {
                const double v = kBlockSum > 1 ? acc.value() + (double)blk : acc.value();
                blk = (P)0;
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
            if constexpr (kBlockSum > 1) {
                blk += p;
                if (i % kBlockSum == kBlockSum - 1) {
                    acc.add(blk);
                    blk = (P)0;
                }
            } else {
                acc.add(p);
            }
            lx += (valid && !is_end) ? 1 : 0;
        }

        // ---- warp segmented scan of (has_end, trailing partial)
        int f = first_row >= 0;
        double v = kBlockSum > 1 ? acc.value() + (double)blk : acc.value();
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
            publish_carry(src.slots(), src.nslots(), epoch, src.slot_base() + u, v);
            if (y1 < src.nrow() && u + 1 < src.num_tiles()) {
                const int rs1 = s_rp[rpo + nr];  // start of row y1
                if (rs1 >= x0 && rs1 < x1) {
                    pa.got = swap_boundary(src.xch(), src.nslots(), epoch, src.slot_base() + u + 1, v);
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
                    pb.got = swap_boundary(src.xch(), src.nslots(), epoch, src.slot_base() + u, rv);
                    pb.mine = rv;
                    pb.row = y0;
                    pb.carry = 0;
                }
            } else {
                if (nlb == kLookBackQueue) {  // warp-uniform
                    drain_look_backs(src, epoch, lbq, nlb, lane, out);
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

}  // namespace merbit
