// Internal definitions shared by the merbit_b200 CUDA sources.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
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

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until *flag == epoch.  Returns false (and raises MERBIT_ERR_TIMEOUT
// in st->error) if that takes longer than kCarryWaitNs or another wait of
// this launch already gave up.
__device__ __forceinline__ bool wait_epoch(const unsigned* flag, unsigned epoch, LaunchState* st) {
    if (ld_acquire_u32(flag) == epoch) return true;
    const unsigned long long t0 = global_timer_ns();
    for (;;) {
        __nanosleep(64);
        if (ld_acquire_u32(flag) == epoch) return true;
        if (*(volatile int*)&st->error != 0) return false;
        if (global_timer_ns() - t0 > kCarryWaitNs) {
            atomicExch(&st->error, (int)MERBIT_ERR_TIMEOUT);
            return false;
        }
    }
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
// Precision policies.
//   F64 : values, x, y, products and accumulation in double (plain form).
//   F32 : values f32, x f32, products f32, two-sum (s, c) accumulation.
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

inline size_t dtype_size(int dt) { return dt == MERBIT_F64 ? 8 : dt == MERBIT_F32 ? 4 : 2; }
inline size_t xy_size(int dt) { return dt == MERBIT_F64 ? 8 : 4; }

// Partition of one matrix for one tile size: coords[t] = merge-path (x,y)
// at diagonal t*tile_items, t in [0, num_tiles].
struct Partition {
    int tile_items = 0;
    int num_tiles = 0;
    int2* coords = nullptr;
};

int build_partition(const int32_t* row_ptr, int nrow, int nnz, int tile_items, Partition* out,
                    cudaStream_t s);

// SpMV kernel configurations (spmv.cu).
struct SpmvConfig {
    int block;
    int ipt;
};
int spmv_num_configs(int dtype);
SpmvConfig spmv_config(int dtype, int idx);
int spmv_default_config(int dtype, int nrow, int nnz);

struct SpmvLaunch {
    const int32_t* row_ptr;
    const int32_t* col;
    const void* vals;
    const void* x;
    void* y;
    const int2* coords;
    double* agg;
    unsigned* flag;
    LaunchState* state;
    int num_tiles;
    double alpha, beta;
};
int spmv_launch(int dtype, int cfg, bool vec, const SpmvLaunch& a, cudaStream_t s);

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
    std::vector<merbit::Partition> parts;
    // carry slots shared by every launch of this plan (sized for the
    // largest tile count in use)
    double* agg = nullptr;
    unsigned* flag = nullptr;
    int slots = 0;
    merbit::LaunchState* state = nullptr;
};
