// Internal definitions shared by the merbit_b200 CUDA sources.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
#include <map>
#include <string>
#include <vector>

#include "../../include/merbit.h"

namespace merbit {

// ---------------------------------------------------------------------------
// Launch bookkeeping shared by every kernel that carries partial row sums
// across tiles.  A launch hands out tiles in start order through `ticket`
// (so a tile's predecessors have always started: the carry wait cannot
// deadlock on an unscheduled CTA), publishes per-tile carries tagged with
// `epoch`, and the last CTA to finish resets `ticket`/`done` and advances
// `epoch`.  Nothing has to be cleared between launches, so launches can be
// captured into CUDA graphs and replayed.
// ---------------------------------------------------------------------------
struct LaunchState {
    unsigned long long ticket;
    unsigned int epoch;
    unsigned int done;
    int error;  // sticky merbit_status raised on the device (MERBIT_ERR_TIMEOUT)
    int pad[3];
};

// Upper bound on one carry wait.  Predecessor tiles publish their carry
// right after their own (wait-free) reduction, so a healthy wait lasts
// microseconds; the bound only turns a broken invariant into an error code.
constexpr unsigned long long kCarryWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- shared-memory barriers and bulk (TMA) copies, sm_90+ ----------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
// Makes an initialized mbarrier visible to the async (bulk copy) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// try_wait with a suspend-time hint: a waiting warp sleeps until the phase
// completes (or the hint runs out) instead of re-issuing the test, which
// would keep the shared-memory instruction queue busy for the warps that have
// work.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, unsigned phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase), "r"(100000u)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// L2 policy: streamed matrix data is evicted first so that x stays in L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// Bulk global->shared copy completing on `bar`; dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar,
                                         uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
        "[%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// Waits for phase `phase` of `bar` for at most kCarryWaitNs; on time-out
// raises MERBIT_ERR_TIMEOUT, waits once more (bounded) for the copies still
// in flight, and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase,
                                                  LaunchState* st,
                                                  unsigned long long wait_ns = kCarryWaitNs) {
    if (mbar_try_wait(bar, phase)) return true;
    unsigned long long t0 = global_timer_ns();
    for (;;) {
        if (mbar_try_wait_sleep(bar, phase)) return true;
        if (global_timer_ns() - t0 > wait_ns) break;
    }
    atomicExch(&st->error, (int)MERBIT_ERR_TIMEOUT);
    t0 = global_timer_ns();
    while (!mbar_try_wait(bar, phase) && global_timer_ns() - t0 < wait_ns) {
    }
    return false;
}

// Draws this CTA's tile (thread 0 only) and the launch epoch.
__device__ __forceinline__ void draw_tile(LaunchState* st, int* tile, unsigned* epoch) {
    *epoch = *(volatile unsigned*)&st->epoch;
    *tile = (int)atomicAdd(&st->ticket, 1ull);
}

// Called by thread 0 of every CTA after its last access to the carry slots.
__device__ __forceinline__ void finish_launch(LaunchState* st, unsigned epoch) {
    __threadfence();
    const unsigned prev = atomicAdd(&st->done, 1u);
    if (prev == gridDim.x - 1) {
        st->ticket = 0ull;
        st->done = 0u;
        __threadfence();
        *(volatile unsigned*)&st->epoch = epoch + 1u;
    }
}

// ---------------------------------------------------------------------------
// Carry slots.  Two arrays of nslots 8-byte words, selected by the parity of
// the launch epoch.  A tile publishes its trailing partial sum as one word in
// the current array; a reader spins until the word is no longer kEmpty, so
// one load returns both "ready" and the value.  Every launch refills the
// other array with kEmpty, which makes it ready for the next launch whatever
// tiles this one used (CUDA-graph replays included).  A value whose bits
// happen to equal kEmpty (a NaN) is published as the canonical NaN.
// ---------------------------------------------------------------------------
constexpr unsigned long long kEmpty = ~0ull;

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void publish_carry(unsigned long long* slots, int nslots,
                                              unsigned epoch, int t, double v) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    if (b == kEmpty) b = 0x7FF8000000000000ull;
    st_relaxed_u64(slots + (size_t)(epoch & 1u) * nslots + t, b);
}

// Reads tile t's carry, waiting (bounded) until it is published.
__device__ __forceinline__ double read_carry(const unsigned long long* slots, int nslots,
                                             unsigned epoch, int t, LaunchState* st,
                                             unsigned long long wait_ns = kCarryWaitNs) {
    const unsigned long long* p = slots + (size_t)(epoch & 1u) * nslots + t;
    unsigned long long b = ld_relaxed_u64(p);
    if (b != kEmpty) return __longlong_as_double((long long)b);
    const unsigned long long t0 = global_timer_ns();
    for (;;) {
        __nanosleep(32);
        b = ld_relaxed_u64(p);
        if (b != kEmpty) return __longlong_as_double((long long)b);
        if (*(volatile int*)&st->error != 0) return 0.0;
        if (global_timer_ns() - t0 > wait_ns) {
            atomicExch(&st->error, (int)MERBIT_ERR_TIMEOUT);
            return 0.0;
        }
    }
}

// Grid-strided refill of the other parity's slots.
__device__ __forceinline__ void reset_other_parity(unsigned long long* slots, int nslots,
                                                   unsigned epoch) {
    unsigned long long* o = slots + (size_t)((epoch + 1u) & 1u) * nslots;
    const int stride = (int)(gridDim.x * blockDim.x);
    for (int i = (int)(blockIdx.x * blockDim.x + threadIdx.x); i < nslots; i += stride)
        o[i] = kEmpty;
}

// Decoupled look-back by one warp: the sum of the carries of tiles u-1,
// u-2, ... down to the tile that contains nonzero index rs (the start of
// the row that tile u completes first), in a fixed order -- 32 tiles per
// step, butterfly reduction -- so the result does not depend on timing.
// Tile t's carry is in slot slot_base + t (a batch places each matrix's
// tiles at its own offset of one slot array).
__device__ __forceinline__ double look_back(const int2* coords, const unsigned long long* slots,
                                            int nslots, unsigned epoch, LaunchState* st, int u,
                                            int rs, int lane, int slot_base = 0) {
    double total = 0.0;
    int base = u - 1;
    for (;;) {
        const int tq = base - lane;
        const bool valid = tq >= 0;
        const int cx = valid ? coords[tq].x : 0;
        const unsigned m = __ballot_sync(0xFFFFFFFFu, !valid || cx <= rs);
        const int last = m ? __ffs(m) - 1 : 31;
        double c = 0.0;
        if (valid && lane <= last) c = read_carry(slots, nslots, epoch, slot_base + tq, st);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
        total += c;
        if (m) break;
        base -= 32;
    }
    return total;
}

// ---------------------------------------------------------------------------
// Precision policies.
//   F64 : values, x, y, products and accumulation in double (plain form).
//   F32 : values f32, x f32, products f32, two-sum (s, c) accumulation
//         (the warp tiles and row groups add blocks of 4 products, summed
//         in f32, per two-sum step; warp_tile.cuh, spmv_rows.cu).
//   BF16: values bf16, otherwise as F32.
// Carries between threads and tiles are always double.
// ---------------------------------------------------------------------------
struct AccF64 {
    double s;
    __device__ __forceinline__ void zero() { s = 0.0; }
    __device__ __forceinline__ void add(double p) { s += p; }
    __device__ __forceinline__ double value() const { return s; }
};

// Knuth's TwoSum: s + c carries the running sum with the rounding error of
// every addition recovered exactly into c.
struct AccTwoSum {
    float s, c;
    __device__ __forceinline__ void zero() {
        s = 0.f;
        c = 0.f;
    }
    __device__ __forceinline__ void add(float p) {
        const float t = __fadd_rn(s, p);
        const float bp = __fsub_rn(t, s);
        const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(p, bp));
        s = t;
        c = __fadd_rn(c, e);
    }
    __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

template <int DT>
struct Prec;
template <>
struct Prec<MERBIT_F64> {
    using V = double;
    using X = double;
    using Y = double;
    using P = double;
    using Acc = AccF64;
};
template <>
struct Prec<MERBIT_F32> {
    using V = float;
    using X = float;
    using Y = float;
    using P = float;
    using Acc = AccTwoSum;
};
template <>
struct Prec<MERBIT_BF16> {
    using V = __nv_bfloat16;
    using X = float;
    using Y = float;
    using P = float;
    using Acc = AccTwoSum;
};

__device__ __forceinline__ double to_p(double v) { return v; }
__device__ __forceinline__ float to_p(float v) { return v; }
__device__ __forceinline__ float to_p(__nv_bfloat16 v) { return __bfloat162float(v); }

// Four consecutive values starting at a 4-element-aligned index, streamed
// (evict-first) so that x keeps its place in L2.
__device__ __forceinline__ void ld4_stream(const double* p, double (&v)[4]) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
}
__device__ __forceinline__ void ld4_stream(const float* p, float (&v)[4]) {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(p));
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = a.w;
}
__device__ __forceinline__ void ld4_stream(const __nv_bfloat16* p, float (&v)[4]) {
    const uint2 a = __ldcs(reinterpret_cast<const uint2*>(p));
    v[0] = __uint_as_float(a.x << 16);
    v[1] = __uint_as_float(a.x & 0xFFFF0000u);
    v[2] = __uint_as_float(a.y << 16);
    v[3] = __uint_as_float(a.y & 0xFFFF0000u);
}

__device__ __forceinline__ void st4_shared(double* p, const double (&v)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st4_shared(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// ---------------------------------------------------------------------------
// Host-side helpers
// ---------------------------------------------------------------------------
void set_error_detail(const std::string& s);
int fail(int status, const std::string& detail);
int cuda_fail(cudaError_t e, const char* where);

#define MERBIT_CUDA(call)                                          \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return ::merbit::cuda_fail(_e, #call); \
    } while (0)

// Device memory (pool.cu): stream-ordered blocks from one pool per device
// that keeps released blocks mapped.  dev_alloc allocates on the current
// device, ordered on s; dev_free releases in order on s.  An owner released
// without a stream (plan or batch destroy) synchronizes the device first,
// as cudaFree would, and frees on the legacy stream.
int dev_alloc(void** p, size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);
template <class T>
int dev_alloc(T** p, size_t bytes, cudaStream_t s) {
    return dev_alloc(reinterpret_cast<void**>(p), bytes, s);
}

inline size_t dtype_size(int dt) { return dt == MERBIT_F64 ? 8 : dt == MERBIT_F32 ? 4 : 2; }
inline size_t xy_size(int dt) { return dt == MERBIT_F64 ? 8 : 4; }

// Partition of one matrix for one tile size: coords[t] = merge-path (x,y)
// at diagonal t*tile_items, t in [0, num_tiles].
struct Partition {
    int tile_items = 0;
    int num_tiles = 0;
    int max_rows = 0;  // largest number of row ends in one tile
    int2* coords = nullptr;
};

// Entries of the row_ptr window a warp-tile stage holds (32*ipt merge items
// per tile); a plan whose tiles end more than warp_rp_cap(ipt) - 8 rows
// cannot use that configuration.
constexpr int warp_rp_cap(int ipt) { return (32 * ipt) / 3 + 16; }

// Allocates out->coords and queues the merge-path search of every tile
// boundary on s, without synchronizing; the largest rows-per-tile is
// atomically maxed into *d_max_rows (zeroed by the caller), and
// out->max_rows stays -1 until the caller reads it back.
int build_partition_async(const int32_t* row_ptr, int nrow, int nnz, int tile_items,
                          Partition* out, int* d_max_rows, cudaStream_t s);

// Device words a plan build reads back once: validation result (error bits,
// first decreasing row, first bad column) and the new partition's largest
// rows-per-tile.  Lives right after the plan's LaunchState.
struct PlanScratch {
    int err;
    int first_bad[2];
    int max_rows;
    int max_row_len;  // longest row of the matrix
    int pad;          // keeps the size a multiple of 8 (the state layout)
};
// Launches the structural CSR checks into sc->err / sc->first_bad (the
// caller initializes them to 0 / INT_MAX) and the longest row into
// sc->max_row_len (initialized to 0); with check == false only the longest
// row is found.  validate_status turns the words read back into a status.
int validate_launch(const int32_t* row_ptr, const int32_t* col, int nrow, int ncol, int nnz,
                    PlanScratch* sc, bool check, cudaStream_t s);
int validate_status(const PlanScratch& h);

// Failure-detection self-test: one bounded wait (which = 0 the carry wait,
// 1 the mbarrier wait) on a flag nothing sets, recording its time-out in
// *st (selftest.cu).
int selftest_wait_on(LaunchState* st, int which, int wait_us, cudaStream_t s);

// Carry / swap words of one SpMM slot family (2 parities x 2 arrays x
// tiles x k) with its own launch state.
struct SpmmSlots {
    unsigned long long* words = nullptr;
    LaunchState* state = nullptr;
    long long nslots = 0;  // tiles * k
};
int alloc_spmm_slots(SpmmSlots* s, long long nslots, cudaStream_t st);

// SpMV kernel configurations (spmv.cu).
struct SpmvConfig {
    int kind;  // 0: CTA-tile kernel, 1: warp-tile kernel
    int block;
    int ipt;
    int stages;  // warp-tile kernel: shared-memory stages per warp (1)
    // Warp-tile kernel: preferred shared-memory carveout in percent (0: the
    // driver's choice, which for these kernels is all shared memory).  The
    // x gathers need L1 capacity for their misses in flight; giving L1 more
    // of the SM's 256 KB (fewer resident CTAs) pays on matrices whose
    // gathers miss L1.
    int carveout;
    int cg;  // 1: x gathers cached in L2 only (ld.global.cg)
    // Row-group kernel: 1 = a warp loads its row block's nonzeros as one
    // contiguous run (coalesced) and stages the products in shared memory
    // for the groups to reduce; 0 = each group reads its own row strided.
    // Warp-tile kernel: 1 = the row_ptr window holds a tile whose every item
    // ends a row (no cap on rows per tile), 0 = warp_rp_cap(ipt) entries.
    int stg;
};
constexpr int kCarveoutL1 = 72;     // ~164 KB shared memory, the rest L1
constexpr int kCarveoutL1Max = 58;  // ~132 KB shared memory
constexpr int kCarveoutL1Most = 44;  // ~100 KB shared memory
int spmv_num_configs(int dtype);
SpmvConfig spmv_config(int dtype, int idx);
int spmv_tile_items(const SpmvConfig& c);
bool spmv_config_allowed(const SpmvConfig& c, bool vec);
int spmv_config_row_cap(const SpmvConfig& c);

struct SpmvLaunch {
    const int32_t* row_ptr;
    const int32_t* col;
    const void* vals;
    const void* x;
    void* y;
    const int2* coords;
    unsigned long long* slots;  // 2 * nslots carry slots (see publish_carry)
    unsigned long long* xch;    // 2 * nslots boundary-swap slots (warp-tile kernel)
    LaunchState* state;
    int nrow, nnz;
    int num_tiles;
    int nslots;
    double alpha, beta;
    // Fused epilogue (PageRank step).  z: the vector beta multiplies (NULL:
    // y itself).  residual != NULL: the launch also writes
    // *residual = sum_r |y[r] - xres[r]|, reduced through partials[] (one
    // word per CTA of the warp-tile kernel, per tile of the CTA-tile kernel)
    // in a fixed order by the launch's last CTA.
    const void* z = nullptr;
    const void* xres = nullptr;
    double* partials = nullptr;
    double* residual = nullptr;
};
int spmv_launch(int dtype, int cfg, bool vec, const SpmvLaunch& a, cudaStream_t s);

// Final store of one row: y[r] = fma(beta, z[r], alpha * v) (z is y for a plain
// product; beta == 0 reads nothing).  RES adds |y[r] - xres[r]| of the value
// as stored to the thread's running residual.
template <typename Y, bool RES>
struct RowStore {
    Y* y;
    const Y* z;
    const Y* xres;
    double alpha, beta;
    double res;
    __device__ __forceinline__ explicit RowStore(const SpmvLaunch& a)
        : y(static_cast<Y*>(a.y)),
          z(static_cast<const Y*>(a.z ? a.z : a.y)),
          xres(static_cast<const Y*>(a.xres)),
          alpha(a.alpha),
          beta(a.beta),
          res(0.0) {}
    // explicit roundings: every kernel instantiation stores the same bits
    __device__ __forceinline__ void operator()(int r, double v) {
        double o = __dmul_rn(alpha, v);
        if (beta != 0.0) o = __fma_rn(beta, (double)z[r], o);
        const Y yo = (Y)o;
        y[r] = yo;
        if (RES) res += fabs((double)yo - (double)xres[r]);
    }
};

// finish_launch for a launch that reduces a residual: called by every thread
// of the CTA with its running residual `v`.  The CTA's sum (butterfly, then
// warps in order) goes to partials[idx]; the launch's last CTA sums
// partials[0, nparts) in a fixed order into *out, then resets the launch
// state as finish_launch does.  The result does not depend on timing.
template <int NW>
__device__ __forceinline__ void finish_launch_residual(LaunchState* st, unsigned epoch, double v,
                                                       double* partials, int idx, int nparts,
                                                       double* out) {
    __shared__ double s_red[NW];
    __shared__ int s_last;
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
        const unsigned prev = atomicAdd(&st->done, 1u);
        s_last = prev == gridDim.x - 1;
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
        st->ticket = 0ull;
        st->done = 0u;
        __threadfence();
        *(volatile unsigned*)&st->epoch = epoch + 1u;
    }
}

// One matrix of an SpMM launch (spmm.cu).  Tiles of ITEMS merge items;
// coords are the matrix's own partition (local tile indices), tile_begin
// its first tile in the launch's tile index space.
struct SpmmDesc {
    const int32_t* row_ptr;
    const int32_t* col;
    const void* vals;
    const void* x;
    void* y;
    long long ldx, ldy;
    const int2* coords;
    int nrow, nnz, num_tiles, tile_begin;
    int ipt;  // batched k = 1 warp-tile kernel: items per lane of this matrix's tiles
    int pad;
};

struct SpmmLaunch {
    SpmmDesc single;        // used when ndesc == 0
    const SpmmDesc* descs;  // device array of ndesc descriptors (a batch)
    int ndesc;
    unsigned long long* slots;  // 2 * nslots carry words (nslots = total_tiles * k)
    unsigned long long* xch;    // 2 * nslots boundary-swap words
    int nslots;
    LaunchState* state;
    int total_tiles;
    double alpha, beta;
    // Fused dL/dval (single matrix that is a transpose plan): for every
    // nonzero e of this matrix, dv_out[dv_perm[e]] = sum over the launch's
    // columns j of dv_x[row(e), j] * x[col(e), j].  NULL: not fused.
    const void* dv_x = nullptr;
    long long dv_ldx = 0;
    const int* dv_perm = nullptr;
    void* dv_out = nullptr;
};

// Launches the SpMM kernel for k right-hand sides, vw values per lane and
// `items` merge items per warp tile.
// items2 != 0: a batch whose matrices take tiles of `items` or `items2`
// (descriptor field ipt = the matrix's tile items); pairs exist for vector
// width 4 at k = 4, 8, 16, 32: (256, 512) and the two odd tiles of k.
int spmm_launch(int dtype, int k, int vw, int items, const SpmmLaunch& a, cudaStream_t s,
                int items2 = 0);
bool spmm_pair_exists(int k, int vw, int items, int items2);

// Batched warp-tile SpMV for k = 1 (batch_warp.cu): every descriptor's
// tiles hold 32 * ipt merge items, ipt one of kBatchIpts; variant indexes
// kBatchWarpVariants: gather hint, shared-memory carveout and the largest
// tile its stages hold (11, 15 or 23 items per lane).  A variant takes the
// items per lane up to its largest, from {7, 11, 15} or {15, 19, 23}.
constexpr int kBatchIpts[] = {7, 11, 15, 19, 23};
constexpr int kNumBatchIpts = 5;
constexpr int kBatchWarpVariants = 10;
constexpr int batch_variant_max_ipt(int variant) {
    return variant == 3 || variant == 4 ? 23 : variant >= 6 ? 11 : 15;
}
constexpr bool batch_variant_takes(int variant, int ipt) {
    return batch_variant_max_ipt(variant) == 23 ? (ipt == 15 || ipt == 19 || ipt == 23)
                                                : ((ipt == 7 || ipt == 11 || ipt == 15) &&
                                                   ipt <= batch_variant_max_ipt(variant));
}
// The items per lane a variant is timed with before the per-class search.
constexpr int batch_variant_start_ipt(int variant) {
    return batch_variant_max_ipt(variant) == 11 ? 11 : 15;
}
int batch_warp_launch(int dtype, int variant, const SpmmLaunch& a, cudaStream_t s);
// The tuning cache, shared by merbit_plan_tune and merbit_batch_tune: the
// items per lane of the batched k = 1 kernel for a plan's signature (-1:
// nothing cached) and the variant it was tuned in (*variant, -1 when only a
// warp-tile SpMV configuration suggested it), and the store of a batch
// tuner's choice.
int tune_cache_batch_ipt(const merbit_plan_s* p, int* variant);
void tune_cache_store_batch_ipt(const merbit_plan_s* p, int variant, int ipt);
bool spmm_config_exists(int k, int vw, int items);
// The tile sizes (merge items) the SpMM kernel has for k right-hand sides,
// into out[8]; returns how many.  spmm_odd_tile: the larger tile of an odd
// length per lane group at vector width 4 (0 if k has none).
int spmm_tile_candidates(int k, int* out);
int spmm_odd_tile(int k);

}  // namespace merbit

// Host-side plan object.
struct merbit_plan_s {
    int nrow = 0, ncol = 0, nnz = 0, dtype = 0;
    const int32_t* row_ptr = nullptr;
    const int32_t* col = nullptr;
    const void* vals = nullptr;
    bool vec = false;
    int device = 0;
    int cfg = 0;  // index into the SpMV config table
    int max_row_len = -1;  // longest row (-1: not measured)
    std::vector<merbit::Partition> parts;
    // carry slots shared by every launch of this plan (2 * slots words,
    // sized for the largest tile count in use)
    unsigned long long* carry = nullptr;
    int slots = 0;
    merbit::LaunchState* state = nullptr;
    merbit::PlanScratch* scratch = nullptr;  // same allocation as state
    // SpMM carry slots, keyed by (k << 20 | tile items)
    std::map<long long, merbit::SpmmSlots> spmm_slots;
    // adjoint support: row index of every nonzero (built on first use), and
    // for a transpose plan the permutation into the source's nonzeros plus
    // the device buffers the plan owns (col_ptr, row_idx, perm, values)
    int* row_of = nullptr;
    int* perm = nullptr;
    std::vector<void*> owned;
    // per-CTA residual partials of the fused PageRank step (grown on use)
    double* partials = nullptr;
    long long npartials = 0;
};

namespace merbit {
int plan_partition(merbit_plan_s* p, int tile_items, const Partition** out, cudaStream_t s);
}
