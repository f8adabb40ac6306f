// Merge-path SpMM for sm_100a:  Y = alpha * A X + beta * Y  with K
// right-hand sides (row-major X [ncol x ldx], Y [nrow x ldy]), for one
// matrix or a batch of matrices in one persistent launch.
//
// The merge path of each matrix is cut into warp tiles of ITEMS merge
// items, as for the SpMV (spmv_warp.cu): lane 0 stages the tile's row_ptr
// window, col_idx slice and vals slice with cp.async.bulk on an mbarrier.
// Inside the warp, lanes form groups of K/VW lanes (VW = RHS values per
// lane: 1, 2 or 4); each group walks its own segment of ITEMS/G merge items
// (G groups per warp), lane j of a group owning RHS columns
// [j*VW, j*VW + VW).  The x rows of the next CH nonzeros are gathered while
// the current CH are accumulated, so gathers overlap the walk.  A row that
// ends inside a segment is written directly (coalesced across the group's
// lanes); the group segmented scan (shuffles with stride K/VW) finishes the
// rows split between groups, and rows split between tiles are finished
// per RHS column exactly as in the SpMV: two-tile rows by an atomicExch
// swap of the partials (the later side writes carry + head), longer rows by
// a fixed-order look-back over published per-tile partials.  No float
// atomics: results are bitwise reproducible.
//
// Batches: the tiles of all matrices form one index space; matrix m owns
// tiles [tile_begin_m, tile_begin_m + num_tiles_m).  Warps of the
// persistent cooperative grid take tiles round-robin, so one launch covers
// the whole batch, and the launch can be captured in a CUDA graph and
// replayed (carry slots are per launch parity, as in the SpMV).
//
// Fused backward (DV, merbit_spmm_dval): run on the transpose plan of A, the
// walk also forms dL/dval for each nonzero from the G row it has just
// gathered and the current row of X, and stores it through the transpose
// permutation (staged by TMA with the tile's col and vals).
#include <type_traits>

#include "merbit_internal.cuh"

namespace merbit {

namespace {

constexpr size_t a16(size_t b) { return (b + 15) & ~(size_t)15; }

template <int VW>
__device__ __forceinline__ void ld_vec(const float* p, float (&o)[VW]) {
    if (VW == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = t.x;
        o[1] = t.y;
        o[2] = t.z;
        o[3] = t.w;
    } else if (VW == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        o[0] = t.x;
        o[1] = t.y;
    } else {
        o[0] = __ldg(p);
    }
}
template <int VW>
__device__ __forceinline__ void ld_vec(const double* p, double (&o)[VW]) {
    if (VW >= 2) {
#pragma unroll
        for (int q = 0; q < VW; q += 2) {
            const double2 t = __ldg(reinterpret_cast<const double2*>(p) + q / 2);
            o[q] = t.x;
            o[q + 1] = t.y;
        }
    } else {
        o[0] = __ldg(p);
    }
}

template <typename Y>
__device__ __forceinline__ void st_row(Y* __restrict__ y, size_t off, double v, double alpha,
                                       double beta) {
    double o = alpha * v;
    if (beta != 0.0) o += beta * (double)y[off];
    y[off] = (Y)o;
}

__device__ __forceinline__ unsigned long long dbits(double v) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return b == kEmpty ? 0x7FF8000000000000ull : b;
}

}  // namespace

// The VW accumulators of one lane.  Generic: one Acc per column.
template <class Acc, int VW, typename P, typename X>
struct AccRow {
    static constexpr bool kPairs = false;
    Acc a[VW];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int v = 0; v < VW; ++v) a[v].zero();
    }
    __device__ __forceinline__ void add(P av, const X (&x)[VW]) {
#pragma unroll
        for (int v = 0; v < VW; ++v) a[v].add(av * (P)x[v]);
    }
    __device__ __forceinline__ double value(int v) const { return a[v].value(); }
    __device__ __forceinline__ void add_pair(P a0, const X (&x0)[VW], P a1, const X (&x1)[VW]) {
        add(a0, x0);
        add(a1, x1);
    }
    // products formed beforehand (one per column)
    __device__ __forceinline__ void add_p(const P (&p)[VW]) {
#pragma unroll
        for (int v = 0; v < VW; ++v) a[v].add(p[v]);
    }
};

// TwoSum accumulators of an even number of columns, two columns per packed
// f32x2 instruction (sm_100).  Every operation rounds as the scalar TwoSum of
// AccTwoSum does (products rounded, then s + p with its exact error added
// to c), so the results are bit-identical to the scalar form with half the
// instructions.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
template <int VW>
struct AccRow<AccTwoSum, VW, float, float> {
    static_assert(VW % 2 == 0, "packed TwoSum needs an even width");
    // two products of one row may enter as their fused sum: the pair's
    // rounding (one unit of |a0 x0| + |a1 x1|) replaces the product's
    static constexpr bool kPairs = true;
    unsigned long long s[VW / 2], c[VW / 2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int h = 0; h < VW / 2; ++h) s[h] = c[h] = 0ull;  // +0.0f, +0.0f
    }
    __device__ __forceinline__ void add(float av, const float (&x)[VW]) {
        const unsigned long long a2 = f2_pack(av, av);
#pragma unroll
        for (int h = 0; h < VW / 2; ++h) sum(h, f2_mul(a2, f2_pack(x[2 * h], x[2 * h + 1])));
    }
    __device__ __forceinline__ void add_pair(float a0, const float (&x0)[VW], float a1,
                                             const float (&x1)[VW]) {
        const unsigned long long b0 = f2_pack(a0, a0), b1 = f2_pack(a1, a1);
#pragma unroll
        for (int h = 0; h < VW / 2; ++h) {
            const unsigned long long p0 = f2_mul(b0, f2_pack(x0[2 * h], x0[2 * h + 1]));
            sum(h, f2_fma(b1, f2_pack(x1[2 * h], x1[2 * h + 1]), p0));
        }
    }
    __device__ __forceinline__ void add_p(const float (&p)[VW]) {
#pragma unroll
        for (int h = 0; h < VW / 2; ++h) sum(h, f2_pack(p[2 * h], p[2 * h + 1]));
    }
    // TwoSum of p into (s[h], c[h])
    __device__ __forceinline__ void sum(int h, unsigned long long p) {
        const unsigned long long t = f2_add(s[h], p);
        const unsigned long long bp = f2_sub(t, s[h]);
        const unsigned long long e = f2_add(f2_sub(s[h], f2_sub(t, bp)), f2_sub(p, bp));
        s[h] = t;
        c[h] = f2_add(c[h], e);
    }
    __device__ __forceinline__ double value(int v) const {
        float s0, s1, c0, c1;
        f2_unpack(s[v / 2], s0, s1);
        f2_unpack(c[v / 2], c0, c1);
        return (v & 1) ? (double)s1 + (double)c1 : (double)s0 + (double)c0;
    }
};
template <>
struct AccRow<AccTwoSum, 1, float, float> {
    static constexpr bool kPairs = false;
    AccTwoSum a;
    __device__ __forceinline__ void zero() { a.zero(); }
    __device__ __forceinline__ void add(float av, const float (&x)[1]) { a.add(av * x[0]); }
    __device__ __forceinline__ double value(int) const { return a.value(); }
    __device__ __forceinline__ void add_pair(float a0, const float (&x0)[1], float a1,
                                             const float (&x1)[1]) {
        add(a0, x0);
        add(a1, x1);
    }
    __device__ __forceinline__ void add_p(const float (&p)[1]) { a.add(p[0]); }
};

// DV: also form dL/dval for each nonzero (SpmmLaunch::dv_*), from the x row
// the walk gathers anyway and the current row of dv_x.
template <int DT, int K, int VW, int ITEMS, bool DV = false>
struct SpmmTile {
    using Pr = Prec<DT>;
    using V = typename Pr::V;
    using X = typename Pr::X;
    using Y = typename Pr::Y;
    using P = typename Pr::P;
    using Acc = typename Pr::Acc;
    static constexpr int LPG = K / VW;      // lanes per group
    static constexpr int G = 32 / LPG;      // groups per warp
    static constexpr int SEG = ITEMS / G;   // merge items per group
    // nonzeros gathered ahead: 8 values per lane; at k = 1 (one lane per
    // group, latency-bound) 4, which measured 12% faster on the 128-matrix
    // R-MAT batch (2.25 -> 1.98 ms; 16 ahead: 2.55 ms).  The chunk size does
    // not change the order of the additions.
    static constexpr int CH = K == 1 ? 4 : 8 / VW;
    // Staged products (one lane per group, tiles of 224 or 352 items, no
    // fused dval): the warp gathers the X rows of all the tile's nonzeros
    // lane-contiguously, every gather in flight at once, and stores the
    // products in shared memory; each lane then walks its segment from
    // there.  The chunked walk instead keeps only CH nonzeros ahead per lane.
    static constexpr bool STAGEP = K == 2 && VW == 2 && (ITEMS == 224 || ITEMS == 352) && !DV;
    static constexpr int NJ = ITEMS / 32;  // staged products per lane
    static constexpr int CAP = ITEMS + 32;
    static constexpr int RPC = ITEMS + 16;  // row_ptr window (any rows per tile)
    static constexpr size_t rp_bytes = a16((size_t)RPC * 4);
    static constexpr size_t col_bytes = a16((size_t)CAP * 4);
    static constexpr size_t val_bytes = a16((size_t)CAP * sizeof(V));
    // DV: the tile's slice of the transpose permutation, staged like col
    static constexpr size_t perm_bytes = DV ? a16((size_t)CAP * 4) : 0;
    static constexpr size_t perm_offset = rp_bytes + col_bytes + val_bytes;
    static constexpr size_t prod_bytes = STAGEP ? a16((size_t)ITEMS * VW * sizeof(P)) : 0;
    static constexpr size_t prod_offset = perm_offset + perm_bytes;
    static constexpr size_t bar_offset = prod_offset + prod_bytes;
    static constexpr size_t bytes = bar_offset + 16;
    static constexpr int GV = 16 / (int)sizeof(V);
    static_assert(LPG >= 1 && LPG <= 32 && 32 % LPG == 0, "K/VW must divide 32");
    static_assert(SEG * G == ITEMS, "ITEMS must be a multiple of the group count");

    static __device__ __forceinline__ void issue(const SpmmDesc& d, int lt, unsigned char* ws,
                                                 uint64_t* bar, int lane,
                                                 const int* perm = nullptr) {
        const int2 c0 = d.coords[lt];
        const int2 c1 = d.coords[lt + 1];
        int* s_rp = reinterpret_cast<int*>(ws);
        int* s_col = reinterpret_cast<int*>(ws + rp_bytes);
        V* s_val = reinterpret_cast<V*>(ws + rp_bytes + col_bytes);
        const V* vals = static_cast<const V*>(d.vals);
        const int nrp = d.nrow + 1;
        // bulk copies need 16-byte aligned global addresses; an array whose
        // base is not 16-byte aligned (a caller's offset view) is staged by
        // plain loads instead (no transaction bytes)
        auto bb = [](const void* src, int s, int e, int n, int g, int esz) -> unsigned {
            if (e <= s || ((uintptr_t)src & 15u) != 0) return 0u;
            const int base = s & ~(g - 1), lim = n & ~(g - 1);
            const int b_end = min((e + g - 1) & ~(g - 1), lim);
            return b_end > base ? (unsigned)(b_end - base) * (unsigned)esz : 0u;
        };
        const unsigned tot = bb(d.row_ptr, c0.y, c1.y + 1, nrp, 4, 4) +
                             bb(d.col, c0.x, c1.x, d.nnz, 4, 4) +
                             bb(vals, c0.x, c1.x, d.nnz, GV, (int)sizeof(V)) +
                             (DV ? bb(perm, c0.x, c1.x, d.nnz, 4, 4) : 0u);
        __syncwarp();
        if (lane == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive_expect_tx(bar, tot);
        }
        const uint64_t pol = l2_evict_first_policy();
        auto stage = [&](auto* dst, const auto* src, int s, int e, int n) {
            using T = typename std::remove_pointer<decltype(dst)>::type;
            constexpr int GG = 16 / (int)sizeof(T);
            if (e <= s) return;
            const int base = s & ~(GG - 1), lim = n & ~(GG - 1);
            if (((uintptr_t)src & 15u) != 0) {  // warp-uniform: plain loads
                for (int i = s + lane; i < e; i += 32) dst[i - base] = src[i];
                return;
            }
            const int b_end = min((e + GG - 1) & ~(GG - 1), lim);
            if (b_end > base && lane == 0)
                bulk_g2s(dst, src + base, (unsigned)(b_end - base) * (unsigned)sizeof(T), bar, pol);
            const int p0 = max(b_end, s);
            if (lane < e - p0) dst[p0 + lane - base] = src[p0 + lane];
        };
        stage(s_rp, d.row_ptr, c0.y, c1.y + 1, nrp);
        stage(s_col, d.col, c0.x, c1.x, d.nnz);
        stage(s_val, vals, c0.x, c1.x, d.nnz);
        if (DV) stage(reinterpret_cast<int*>(ws + perm_offset), perm, c0.x, c1.x, d.nnz);
    }

    // Row ends of the tile as nonzero positions relative to x0.
    static __device__ __forceinline__ int row_end(const int* s_rp, int rpo, int r, int x0) {
        return s_rp[rpo + r + 1] - x0;
    }

    static __device__ __forceinline__ void process(const SpmmLaunch& a, const SpmmDesc& d,
                                                   int u, int lt, unsigned epoch,
                                                   unsigned char* ws, int lane) {
        unsigned long long* slots = a.slots;
        unsigned long long* xch = a.xch;
        const int nslots = a.nslots;
        LaunchState* st = a.state;
        const int* s_rp = reinterpret_cast<const int*>(ws);
        const int* s_col = reinterpret_cast<const int*>(ws + rp_bytes);
        const V* s_val = reinterpret_cast<const V*>(ws + rp_bytes + col_bytes);
        const int2 c0 = d.coords[lt];
        const int2 c1 = d.coords[lt + 1];
        const int prev_x = lt > 0 ? d.coords[lt - 1].x : 0;
        const int x0 = c0.x, y0 = c0.y, x1 = c1.x, y1 = c1.y;
        const int nz = x1 - x0, nr = y1 - y0, L = nz + nr;
        const int rpo = y0 - (y0 & ~3);
        const int col_o = x0 - (x0 & ~3);
        const int val_o = x0 - (x0 & ~(GV - 1));
        const int g = lane / LPG;        // group
        const int jl = lane % LPG;       // lane within group
        const int j0 = jl * VW;          // first RHS column of this lane
        const X* __restrict__ xm = static_cast<const X*>(d.x);
        Y* __restrict__ ym = static_cast<Y*>(d.y);
        const double alpha = a.alpha, beta = a.beta;

        // ---- this group's segment [ds, de) of the tile's merge path
        const int ds = min(g * SEG, L), de = min(ds + SEG, L);
        auto search = [&](int dl, int& lx, int& ly) {
            int lo = max(dl - nz, 0), hi = min(dl, nr);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (s_rp[rpo + mid + 1] - x0 <= dl - mid - 1)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            ly = lo;
            lx = dl - lo;
        };
        int lx, ly, lx_end, ly_end;
        search(ds, lx, ly);
        search(de, lx_end, ly_end);

        AccRow<Acc, VW, P, X> acc;
        acc.zero();
        constexpr bool AccPairs = AccRow<Acc, VW, P, X>::kPairs;
        int first_row = -1;
        double first_val[VW];
#pragma unroll
        for (int v = 0; v < VW; ++v) first_val[v] = 0.0;
        auto emit = [&](int r) {
            if (first_row < 0) {
                first_row = r;
#pragma unroll
                for (int v = 0; v < VW; ++v) first_val[v] = acc.value(v);
            } else {
#pragma unroll
                for (int v = 0; v < VW; ++v)
                    st_row(ym, (size_t)(y0 + r) * d.ldy + j0 + v, acc.value(v), alpha, beta);
            }
            acc.zero();
        };

        // ---- walk: chunks of CH nonzeros, the next chunk's x rows in flight
        // (two named buffers, so both stay in registers)
        X xa[CH][VW], xb[CH][VW];
        V va[CH], vb[CH];
        auto load_chunk = [&](int c, X (&xr)[CH][VW], V (&vv)[CH]) {
#pragma unroll
            for (int t = 0; t < CH; ++t) {
                if (c + t < lx_end) {
                    const int e = c + t;
                    const int colv = s_col[col_o + e];
                    vv[t] = s_val[val_o + e];
                    ld_vec<VW>(xm + (size_t)colv * d.ldx + j0, xr[t]);
                }
            }
        };
        // end of row ly (INT_MAX past the segment's last row), kept in a
        // register so the walk reads row_ptr once per row, not per nonzero
        int next_end = ly < ly_end ? row_end(s_rp, rpo, ly, x0) : INT_MAX;
        // fused dval: this lane's VW values of dv_x's current row
        const X* __restrict__ dvx = static_cast<const X*>(a.dv_x);
        X* __restrict__ dvo = static_cast<X*>(a.dv_out);
        X xrow[VW];
        int xrow_of = -1;
        const int* s_perm = reinterpret_cast<const int*>(ws + perm_offset);
        const unsigned gmask = LPG == 32 ? 0xFFFFFFFFu : (((1u << LPG) - 1u) << (g * LPG));
        auto dv_step = [&](int t, int e, const X (&xr)[CH][VW]) {
            if (y0 + ly != xrow_of) {  // uniform within the group
                xrow_of = y0 + ly;
                ld_vec<VW>(dvx + (size_t)xrow_of * a.dv_ldx + j0, xrow);
            }
            // in the x type: VW fused multiply-adds per lane, then a tree
            // over the group's lanes (error within (VW + log2 LPG) roundings
            // of sum |g x|)
            X dd = (X)0;
#pragma unroll
            for (int v = 0; v < VW; ++v) dd = fma(xr[t][v], xrow[v], dd);
#pragma unroll
            for (int o = LPG / 2; o > 0; o >>= 1) dd += __shfl_xor_sync(gmask, dd, o);
            if (jl == 0) dvo[s_perm[col_o + e]] = dd;
        };
        auto end_rows = [&](int e) {
            while (next_end <= e) {
                emit(ly);
                ++ly;
                next_end = ly < ly_end ? row_end(s_rp, rpo, ly, x0) : INT_MAX;
            }
        };
        auto consume = [&](int c, const X (&xr)[CH][VW], const V (&vv)[CH]) {
            if (AccPairs && CH == 2) {
                // two nonzeros of one row: one compensated addition of their
                // fused pair sum (fma(a1, x1, a0 x0)) instead of two
                if (c < lx_end) {
                    end_rows(c);
                    if (c + 1 < lx_end && next_end > c + 1) {
                        acc.add_pair(to_p(vv[0]), xr[0], to_p(vv[1]), xr[1 % CH]);
                        if (DV) {
                            dv_step(0, c, xr);
                            dv_step(1 % CH, c + 1, xr);
                        }
                        return;
                    }
                    acc.add(to_p(vv[0]), xr[0]);
                    if (DV) dv_step(0, c, xr);
                    if (c + 1 < lx_end) {
                        end_rows(c + 1);
                        acc.add(to_p(vv[1 % CH]), xr[1 % CH]);
                        if (DV) dv_step(1 % CH, c + 1, xr);
                    }
                }
                return;
            }
#pragma unroll
            for (int t = 0; t < CH; ++t) {
                const int e = c + t;
                if (e < lx_end) {
                    end_rows(e);
                    acc.add(to_p(vv[t]), xr[t]);
                    if (DV) dv_step(t, e, xr);
                }
            }
        };
        if constexpr (STAGEP) {
            // products of nonzero i (relative to the tile) at s_prod[i * VW]
            P* s_prod = reinterpret_cast<P*>(ws + prod_offset);
            {
                int cidx[NJ];
#pragma unroll
                for (int j = 0; j < NJ; ++j) {
                    const int i = lane + 32 * j;
                    cidx[j] = i < nz ? s_col[col_o + i] : 0;
                }
                X xr[NJ][VW];
#pragma unroll
                for (int j = 0; j < NJ; ++j)
                    if (lane + 32 * j < nz) ld_vec<VW>(xm + (size_t)cidx[j] * d.ldx, xr[j]);
#pragma unroll
                for (int j = 0; j < NJ; ++j) {
                    const int i = lane + 32 * j;
                    if (i < nz) {
                        const P av = to_p(s_val[val_o + i]);
#pragma unroll
                        for (int v = 0; v < VW; ++v) s_prod[(size_t)i * VW + v] = av * (P)xr[j][v];
                    }
                }
            }
            __syncwarp();
            for (int e = lx; e < lx_end; ++e) {
                end_rows(e);
                P pv[VW];
#pragma unroll
                for (int v = 0; v < VW; ++v) pv[v] = s_prod[(size_t)e * VW + v];
                acc.add_p(pv);
            }
        } else {
            if (lx < lx_end) load_chunk(lx, xa, va);
            for (int c = lx; c < lx_end; c += 2 * CH) {
                if (c + CH < lx_end) load_chunk(c + CH, xb, vb);
                consume(c, xa, va);
                if (c + CH >= lx_end) break;
                if (c + 2 * CH < lx_end) load_chunk(c + 2 * CH, xa, va);
                consume(c + CH, xb, vb);
            }
        }
        while (ly < ly_end) {
            emit(ly);
            ++ly;
        }

        // ---- group segmented scan, per RHS column (stride LPG lanes)
        int f = first_row >= 0;
        double sv[VW];
#pragma unroll
        for (int v = 0; v < VW; ++v) sv[v] = acc.value(v);
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
            double t[VW];
#pragma unroll
            for (int v = 0; v < VW; ++v) t[v] = __shfl_up_sync(0xFFFFFFFFu, sv[v], o * LPG);
            const int tf = __shfl_up_sync(0xFFFFFFFFu, f, o * LPG);
            if (g >= o) {
                if (!f) {
#pragma unroll
                    for (int v = 0; v < VW; ++v) sv[v] = t[v] + sv[v];
                }
                f |= tf;
            }
        }
        double ev[VW];
#pragma unroll
        for (int v = 0; v < VW; ++v) {
            ev[v] = G > 1 ? __shfl_up_sync(0xFFFFFFFFu, sv[v], LPG) : 0.0;
            if (g == 0) ev[v] = 0.0;
        }
        const int rs = s_rp[rpo];
        const bool need_lb = nr > 0 && rs < x0;
        const bool holds_first = first_row == 0 && need_lb;
        double rv[VW];
#pragma unroll
        for (int v = 0; v < VW; ++v) rv[v] = ev[v] + first_val[v];
        if (first_row >= 0 && !holds_first) {
#pragma unroll
            for (int v = 0; v < VW; ++v)
                st_row(ym, (size_t)(y0 + first_row) * d.ldy + j0 + v, rv[v], alpha, beta);
        }

        // ---- the tile's trailing partial (last group): published, and
        // swapped with the next tile when the row began in this tile
        const size_t par = (size_t)(epoch & 1u) * nslots;
        if (g == G - 1) {
#pragma unroll
            for (int v = 0; v < VW; ++v)
                st_relaxed_u64(slots + par + (size_t)u * K + j0 + v, dbits(sv[v]));
            if (y1 < d.nrow && lt + 1 < d.num_tiles) {
                const int rs1 = s_rp[rpo + nr];
                if (rs1 >= x0 && rs1 < x1) {
#pragma unroll
                    for (int v = 0; v < VW; ++v) {
                        const unsigned long long o =
                            atomicExch(xch + par + (size_t)(u + 1) * K + j0 + v, dbits(sv[v]));
                        if (o != kEmpty)
                            st_row(ym, (size_t)y1 * d.ldy + j0 + v,
                                   sv[v] + __longlong_as_double((long long)o), alpha, beta);
                    }
                }
            }
        }

        // ---- row y0 when it began in an earlier tile
        if (need_lb) {
            if (prev_x <= rs) {
                if (holds_first) {
#pragma unroll
                    for (int v = 0; v < VW; ++v) {
                        const unsigned long long o =
                            atomicExch(xch + par + (size_t)u * K + j0 + v, dbits(rv[v]));
                        if (o != kEmpty)
                            st_row(ym, (size_t)y0 * d.ldy + j0 + v,
                                   __longlong_as_double((long long)o) + rv[v], alpha, beta);
                    }
                }
            } else {
                // fixed-order look-back over the tiles back to the one that
                // holds the row start.  Lane l serves column l % K; a step
                // covers TPS * R tiles (tile offset l / K + TPS * r from
                // `base`), all loaded before any is summed, so a row spanning
                // hundreds of tiles takes few dependent round trips.  The
                // summation order depends only on the tile and the row start.
                constexpr int TPS = 32 / K > 0 ? 32 / K : 1;
                constexpr int R = 8;
                const bool lane_valid = lane < TPS * K;
                double tot = 0.0;  // column (lane % K) of the sum
                int base = lt - 1;
                for (;;) {
                    int tq[R];
                    int first = INT_MAX;  // smallest offset of a tile starting at or before rs
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int o = lane / K + TPS * r;
                        tq[r] = base - o;
                        if (lane_valid && (tq[r] < 0 || d.coords[tq[r]].x <= rs)) first = min(first, o);
                    }
                    first = __reduce_min_sync(0xFFFFFFFFu, first);
                    unsigned long long bits[R];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int o = lane / K + TPS * r;
                        bits[r] = 0ull;  // +0.0
                        if (lane_valid && tq[r] >= 0 && o <= first)
                            bits[r] = ld_relaxed_u64(slots + par + (size_t)(d.tile_begin + tq[r]) * K + (lane % K));
                    }
                    double c = 0.0;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const int o = lane / K + TPS * r;
                        if (lane_valid && tq[r] >= 0 && o <= first) {
                            if (bits[r] == kEmpty) {
                                const unsigned long long* p =
                                    slots + par + (size_t)(d.tile_begin + tq[r]) * K + (lane % K);
                                const unsigned long long t0 = global_timer_ns();
                                while ((bits[r] = ld_relaxed_u64(p)) == kEmpty) {
                                    __nanosleep(32);
                                    if (*(volatile int*)&st->error != 0) break;
                                    if (global_timer_ns() - t0 > kCarryWaitNs) {
                                        atomicExch(&st->error, (int)MERBIT_ERR_TIMEOUT);
                                        break;
                                    }
                                }
                            }
                            c += bits[r] == kEmpty ? 0.0 : __longlong_as_double((long long)bits[r]);
                        }
                    }
                    // sum over the step's tiles, per column (lanes l, l+K, ...)
#pragma unroll
                    for (int o = K; o < 32; o <<= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
                    tot += c;
                    if (first != INT_MAX) break;
                    base -= TPS * R;
                }
                double tv[VW];
#pragma unroll
                for (int v = 0; v < VW; ++v) tv[v] = __shfl_sync(0xFFFFFFFFu, tot, j0 + v);
                if (holds_first) {
#pragma unroll
                    for (int v = 0; v < VW; ++v)
                        st_row(ym, (size_t)y0 * d.ldy + j0 + v, tv[v] + rv[v], alpha, beta);
                }
            }
        }
    }
};

// The stage of a warp when a launch takes tiles of ITEMS or ITEMS2 items
// (ITEMS2 = 0: ITEMS only): large enough for either, one mbarrier after both.
template <int DT, int K, int VW, int ITEMS, int ITEMS2, bool DV>
struct SpmmStage {
    using T1 = SpmmTile<DT, K, VW, ITEMS, DV>;
    using T2 = SpmmTile<DT, K, VW, ITEMS2 ? ITEMS2 : ITEMS, DV>;
    static constexpr size_t bar_offset =
        T1::bar_offset > T2::bar_offset ? T1::bar_offset : T2::bar_offset;
    static constexpr size_t bytes = bar_offset + 16;
};

// ITEMS2 != 0: a batch whose matrices take tiles of either size; descriptor
// field `ipt` holds the tile items of its matrix (0 or ITEMS: ITEMS).
template <int DT, int K, int VW, int ITEMS, int ITEMS2, int WARPS, bool DV>
__global__ void __launch_bounds__(WARPS * 32) spmm_kernel(const SpmmLaunch a) {
    using St = SpmmStage<DT, K, VW, ITEMS, ITEMS2, DV>;
    using T = typename St::T1;
    using T2 = typename St::T2;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned s_epoch;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_epoch = *(volatile unsigned*)&a.state->epoch;
    unsigned char* ws = smem + (size_t)warp * St::bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(ws + St::bar_offset);
    if (lane == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const unsigned epoch = s_epoch;
    reset_other_parity(a.slots, a.nslots, epoch);
    reset_other_parity(a.xch, a.nslots, epoch);
    const int nw = (int)gridDim.x * WARPS;
    unsigned phase = 0;
    int m = 0;  // matrix of the current tile (tiles are visited in increasing order)
    for (int u = (int)blockIdx.x * WARPS + warp; u < a.total_tiles; u += nw) {
        const SpmmDesc* dp;
        if (a.ndesc == 0) {
            dp = &a.single;
        } else {
            while (m + 1 < a.ndesc && a.descs[m + 1].tile_begin <= u) ++m;
            dp = a.descs + m;
        }
        const SpmmDesc& d = *dp;
        const int lt = u - d.tile_begin;
        const bool second = ITEMS2 != 0 && d.ipt == ITEMS2;  // warp-uniform
        if (second)
            T2::issue(d, lt, ws, bar, lane, a.dv_perm);
        else
            T::issue(d, lt, ws, bar, lane, a.dv_perm);
        const bool ok = __all_sync(0xFFFFFFFFu, mbar_wait_bounded(bar, phase, a.state));
        phase ^= 1u;
        __syncwarp();
        if (ok) {
            if (second)
                T2::process(a, d, u, lt, epoch, ws, lane);
            else
                T::process(a, d, u, lt, epoch, ws, lane);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) finish_launch(a.state, epoch);
}

namespace {

template <int DT, int K, int VW, int ITEMS, int WARPS, bool DV, int ITEMS2 = 0>
int launch_spmm_cfg(const SpmmLaunch& a, cudaStream_t s) {
    constexpr size_t smem = SpmmStage<DT, K, VW, ITEMS, ITEMS2, DV>::bytes * WARPS;
    static int grid_cap[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64) return fail(MERBIT_ERR_UNSUPPORTED, "spmm: device ordinal >= 64");
    auto kern = spmm_kernel<DT, K, VW, ITEMS, ITEMS2, WARPS, DV>;
    // per-device cache; threads that race here compute the same value
    int cap = __atomic_load_n(&grid_cap[dev], __ATOMIC_ACQUIRE);
    if (cap == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(spmm)");
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WARPS * 32, smem);
        if (e != cudaSuccess) return cuda_fail(e, "occupancy(spmm)");
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
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, a);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? (int)MERBIT_OK : cuda_fail(e, "spmm_kernel launch");
}

// Configurations: (K, VW, ITEMS).  WARPS = 4.
template <int DT>
int launch_spmm_dt(int k, int vw, int items, int items2, const SpmmLaunch& a, cudaStream_t s) {
    constexpr bool kDv = DT != MERBIT_BF16;  // fused dval: F64 and F32 plans
    if (a.dv_out && !kDv) return fail(MERBIT_ERR_UNSUPPORTED, "spmm: fused dval needs F64 or F32 values");
    if (items2) {
        // batches whose matrices take either of two tile sizes (vector width 4)
        if (a.dv_out) return fail(MERBIT_ERR_UNSUPPORTED, "spmm: tile pairs take no fused dval");
#define MERBIT_SPMM_PAIR(KK, I1, I2) \
        if (k == KK && vw == 4 && items == I1 && items2 == I2) \
            return launch_spmm_cfg<DT, KK, 4, I1, 4, false, I2>(a, s);
        MERBIT_SPMM_PAIR(4, 256, 512)
        MERBIT_SPMM_PAIR(4, 288, 480)
        MERBIT_SPMM_PAIR(8, 256, 512)
        MERBIT_SPMM_PAIR(8, 272, 496)
        MERBIT_SPMM_PAIR(16, 256, 512)
        MERBIT_SPMM_PAIR(16, 264, 504)
        MERBIT_SPMM_PAIR(32, 256, 512)
        MERBIT_SPMM_PAIR(32, 260, 508)
#undef MERBIT_SPMM_PAIR
        return fail(MERBIT_ERR_INVALID, "spmm: no such tile pair");
    }
#define MERBIT_SPMM_CASE(KK, VV, II)                                                  \
    if (k == KK && vw == VV && items == II)                                           \
        return a.dv_out ? launch_spmm_cfg<DT, KK, VV, II, 4, kDv>(a, s)                \
                        : launch_spmm_cfg<DT, KK, VV, II, 4, false>(a, s);
    MERBIT_SPMM_CASE(1, 1, 256)
    MERBIT_SPMM_CASE(2, 1, 256)
    MERBIT_SPMM_CASE(2, 2, 256)
    MERBIT_SPMM_CASE(4, 1, 256)
    MERBIT_SPMM_CASE(4, 2, 256)
    MERBIT_SPMM_CASE(4, 4, 256)
    MERBIT_SPMM_CASE(8, 1, 256)
    MERBIT_SPMM_CASE(8, 2, 256)
    MERBIT_SPMM_CASE(8, 4, 256)
    MERBIT_SPMM_CASE(16, 1, 256)
    MERBIT_SPMM_CASE(16, 2, 256)
    MERBIT_SPMM_CASE(16, 4, 256)
    MERBIT_SPMM_CASE(32, 1, 256)
    MERBIT_SPMM_CASE(32, 2, 256)
    MERBIT_SPMM_CASE(32, 4, 256)
    MERBIT_SPMM_CASE(1, 1, 512)
    MERBIT_SPMM_CASE(4, 4, 512)
    MERBIT_SPMM_CASE(8, 4, 512)
    MERBIT_SPMM_CASE(16, 4, 512)
    MERBIT_SPMM_CASE(32, 4, 512)
    // odd segments per lane group (tile = groups x odd length): the groups'
    // shared-memory reads start in different banks
    MERBIT_SPMM_CASE(1, 1, 288)
    MERBIT_SPMM_CASE(1, 1, 480)
    MERBIT_SPMM_CASE(4, 4, 288)
    MERBIT_SPMM_CASE(4, 4, 480)
    MERBIT_SPMM_CASE(8, 4, 272)
    MERBIT_SPMM_CASE(8, 4, 496)
    MERBIT_SPMM_CASE(16, 4, 264)
    MERBIT_SPMM_CASE(16, 4, 504)
    MERBIT_SPMM_CASE(32, 4, 260)
    MERBIT_SPMM_CASE(32, 4, 508)
    // k = 2, one lane per group with staged products (SpmmTile::STAGEP):
    // 2.12 ms against 2.84 for the 128-matrix R-MAT batch; at k = 4 the
    // product slice and registers cost more warps than it saves (3.12 ms
    // against 2.39), so k = 4 has no such tile
    MERBIT_SPMM_CASE(2, 2, 224)
    MERBIT_SPMM_CASE(2, 2, 352)
#undef MERBIT_SPMM_CASE
    return fail(MERBIT_ERR_INVALID, "spmm: no such configuration");
}

}  // namespace

bool spmm_config_exists(int k, int vw, int items) {
    if (items == 256) return (k == 1 && vw == 1) || (k >= 2 && k <= 32 && (k & (k - 1)) == 0 && vw <= 4 && vw <= k && (vw & (vw - 1)) == 0 && !(k == 2 && vw == 4));
    if (items == 512) return (k == 1 && vw == 1) || (k >= 4 && k <= 32 && (k & (k - 1)) == 0 && vw == 4);
    if (items == 224 || items == 352) return k == 2 && vw == 2;
    if (k == 1) return vw == 1 && (items == 288 || items == 480);
    if (vw != 4) return false;
    switch (k) {
    case 4: return items == 288 || items == 480;
    case 8: return items == 272 || items == 496;
    case 16: return items == 264 || items == 504;
    case 32: return items == 260 || items == 508;
    }
    return false;
}

int spmm_tile_candidates(int k, int* out) {
    int n = 0;
    out[n++] = 256;
    out[n++] = 512;
    static const int odd[6][2] = {{288, 480}, {0, 0}, {288, 480}, {272, 496}, {264, 504}, {260, 508}};
    const int row = k == 1 ? 0 : k == 4 ? 2 : k == 8 ? 3 : k == 16 ? 4 : k == 32 ? 5 : 1;
    for (int j = 0; j < 2; ++j)
        if (odd[row][j]) out[n++] = odd[row][j];
    if (k == 2) {  // staged products
        out[n++] = 224;
        out[n++] = 352;
    }
    return n;
}

int spmm_odd_tile(int k) {
    switch (k) {
    case 4: return 480;
    case 8: return 496;
    case 16: return 504;
    case 32: return 508;
    }
    return 0;
}

bool spmm_pair_exists(int k, int vw, int items, int items2) {
    if (vw != 4 || !(k == 4 || k == 8 || k == 16 || k == 32)) return false;
    if (items == 256 && items2 == 512) return true;
    return items2 == spmm_odd_tile(k) && items == (k == 4 ? 288 : k == 8 ? 272 : k == 16 ? 264 : 260);
}

int spmm_launch(int dtype, int k, int vw, int items, const SpmmLaunch& a, cudaStream_t s,
                int items2) {
    if (a.total_tiles <= 0) return MERBIT_OK;
    switch (dtype) {
    case MERBIT_F64: return launch_spmm_dt<MERBIT_F64>(k, vw, items, items2, a, s);
    case MERBIT_F32: return launch_spmm_dt<MERBIT_F32>(k, vw, items, items2, a, s);
    case MERBIT_BF16: return launch_spmm_dt<MERBIT_BF16>(k, vw, items, items2, a, s);
    }
    return fail(MERBIT_ERR_INVALID, "spmm: bad dtype");
}

}  // namespace merbit
