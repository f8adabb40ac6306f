// Failure-detection self-test: runs one of the library's bounded device
// waits on a flag that nothing ever sets, so the wait runs out, raises
// MERBIT_ERR_TIMEOUT in the plan's launch state and returns.  The GPU context
// stays usable; merbit_plan_check then reports (and clears) the status.
#include "merbit_internal.cuh"

namespace merbit {
namespace {

// A carry slot that is never published.
__device__ unsigned long long g_never_published = kEmpty;

__global__ void carry_wait_kernel(LaunchState* st, unsigned long long wait_ns) {
    if (threadIdx.x != 0) return;
    // nslots = 0: both parities resolve to the same never-published word
    (void)read_carry(&g_never_published, 0, 0u, 0, st, wait_ns);
}

__global__ void mbar_wait_kernel(LaunchState* st, unsigned long long wait_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);  // one arrival expected; none is made, no copy issued
    fence_mbar_init();
    (void)mbar_wait_bounded(&bar, 0, st, wait_ns);
}

}  // namespace

int selftest_wait_on(LaunchState* st, int which, int wait_us, cudaStream_t s) {
    const unsigned long long ns = 1000ull * (unsigned long long)wait_us;
    if (which == 0)
        carry_wait_kernel<<<1, 32, 0, s>>>(st, ns);
    else
        mbar_wait_kernel<<<1, 32, 0, s>>>(st, ns);
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

}  // namespace merbit

using namespace merbit;

extern "C" int merbit_plan_selftest_wait(merbit_plan plan, int32_t which, int32_t wait_us,
                                         void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "selftest_wait: plan is null");
    if (which != 0 && which != 1) return fail(MERBIT_ERR_INVALID, "selftest_wait: which is 0 or 1");
    if (wait_us < 1 || wait_us > 1000000)
        return fail(MERBIT_ERR_INVALID, "selftest_wait: wait_us outside [1, 1e6]");
    MERBIT_CUDA(cudaSetDevice(plan->device));
    return selftest_wait_on(plan->state, which, wait_us, (cudaStream_t)stream);
}
