// Device memory of the library: one stream-ordered memory pool per device.
//
// A plan owns a few small buffers (launch state, tile coordinates, carry
// slots) and, for adjoints and conversions, nnz-sized work arrays.  With
// cudaMalloc / cudaFree each buffer costs a mapping on allocation and a
// device-wide synchronization plus unmapping on release (about 0.6 ms per
// pair on B200), which dominated building a plan.  Blocks from a
// cudaMemPool stay mapped after release, up to kPoolKeepBytes, so building
// and destroying plans repeatedly costs microseconds, and temporaries are
// released in stream order without synchronizing.
#include <mutex>

#include "merbit_internal.cuh"

namespace merbit {

namespace {

// Released blocks the pool keeps mapped for reuse; above this, memory goes
// back to the device at the next synchronization.
constexpr uint64_t kPoolKeepBytes = 64ull << 20;

std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;

}  // namespace

cudaMemPool_t device_pool(int device) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(device);
    if (it != g_pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t keep = kPoolKeepBytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[device] = pool;
    return pool;
}

int dev_alloc(void** p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    // A stream-ordered allocation made while s is being captured would
    // belong to the captured graph, not to the plan that keeps the pointer:
    // refuse it, as cudaMalloc refuses allocation under capture.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    MERBIT_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(MERBIT_ERR_INVALID,
                    "device allocation while the stream is being captured: make the first "
                    "call of this kind (plan, SpMM slots, residual partials) before capture");
    int dev = 0;
    MERBIT_CUDA(cudaGetDevice(&dev));
    cudaMemPool_t pool = device_pool(dev);
    if (!pool) return fail(MERBIT_ERR_CUDA, "device memory pool: cudaMemPoolCreate failed");
    MERBIT_CUDA(cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, s));
    return MERBIT_OK;
}

void dev_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

}  // namespace merbit

extern "C" int merbit_release_cached_memory(void) {
    using namespace merbit;
    int dev = 0;
    MERBIT_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (g_pools.find(dev) == g_pools.end()) return MERBIT_OK;  // nothing allocated yet
    }
    MERBIT_CUDA(cudaDeviceSynchronize());  // frees in flight reach the pool
    MERBIT_CUDA(cudaMemPoolTrimTo(device_pool(dev), 0));
    return MERBIT_OK;
}
