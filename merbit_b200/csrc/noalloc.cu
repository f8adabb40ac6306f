// SpMV entry point that allocates no device memory.
//
// Some callers cannot allocate device memory on the call path: hosts that
// hand all device memory to their own pool allocator (a framework's caching
// allocator) and cannot have a library take memory behind its back, and
// latency-critical loops that cannot afford cudaMalloc's implicit
// synchronization.  merbit_spmv_noalloc serves them:
// the scratch a merge-path SpMV needs -- tile coordinates, carry slots,
// launch bookkeeping -- lives in one file-scope __device__ array of fixed
// size, which every GPU that loads this library holds until the process
// exits.  The caller still passes the matrix, x and y.
//
// The array's size bounds the matrix: kNoAllocMaxTiles tiles of
// kNoAllocTileItems merge items, i.e. nrow + nnz <= 58,720,256.
//
// Device status: a bounded wait that runs out sets LaunchState::error, and
// the kernels then stop waiting for carries.  Every call's prepare kernel
// therefore moves that word into a sticky report word and clears it, so one
// failed call cannot spoil the calls after it;
// merbit_spmv_noalloc_check reads and clears the report.
#include <cstddef>
#include <mutex>

#include "merbit_internal.cuh"

namespace merbit {
namespace {

constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocIpt = 7;
constexpr int kNoAllocTileItems = kNoAllocBlock * kNoAllocIpt;  // 1792
constexpr int kNoAllocMaxTiles = 32768;
constexpr long long kNoAllocMaxItems = (long long)kNoAllocMaxTiles * kNoAllocTileItems;

// Scratch layout: launch state (padded to 256 B; the status report word at
// byte kReportOffset), tile coordinates, carry slots (two launch parities),
// boundary-swap slots (two parities).
constexpr size_t kStateBytes = 256;
constexpr size_t kReportOffset = 128;
static_assert(sizeof(LaunchState) <= kReportOffset, "launch state overlaps the report word");
constexpr size_t kCoordBytes = sizeof(int2) * (size_t)(kNoAllocMaxTiles + 1);
constexpr size_t kCoordPad = (kCoordBytes + 255) & ~(size_t)255;
constexpr size_t kSlotBytes = sizeof(unsigned long long) * 2 * (size_t)kNoAllocMaxTiles;
constexpr size_t kScratchBytes = kStateBytes + kCoordPad + 2 * kSlotBytes;  // ~1.3 MB

}  // namespace

// In host code this name is a host-side stand-in, not a device address; the
// host reaches the array only through the address cudaGetSymbolAddress gives.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

__device__ __forceinline__ int* report_word(unsigned char* scratch) {
    return reinterpret_cast<int*>(scratch + kReportOffset);
}

__global__ void noalloc_init_kernel(unsigned char* scratch) {
    LaunchState* st = reinterpret_cast<LaunchState*>(scratch);
    unsigned long long* slots =
        reinterpret_cast<unsigned long long*>(scratch + kStateBytes + kCoordPad);
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * kNoAllocMaxTiles; i += stride)
        slots[i] = kEmpty;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->ticket = 0ull;
        st->epoch = 1u;
        st->done = 0u;
        st->error = 0;
        *report_word(scratch) = 0;
    }
}

// Tile coordinates at diagonals t * kNoAllocTileItems (the merge_search
// predicate and tie rule of the reference, include/utils.cuh:5-29), and the
// launch counters cleared for the SpMV that follows on the stream.  A status
// raised by an earlier call moves to the report word, so this call's waits
// start from a clean state.
__global__ void noalloc_prepare_kernel(const int32_t* __restrict__ row_ptr, int nrow, int nnz,
                                       int num_tiles, unsigned char* scratch) {
    int2* coords = reinterpret_cast<int2*>(scratch + kStateBytes);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        LaunchState* st = reinterpret_cast<LaunchState*>(scratch);
        st->ticket = 0ull;
        st->done = 0u;
        const int e = st->error;
        if (e != 0) {
            *report_word(scratch) = e;
            st->error = 0;
        }
    }
    if (t > num_tiles) return;
    const long long total = (long long)nrow + nnz;
    long long d = (long long)t * kNoAllocTileItems;
    if (d > total) d = total;
    long long lo = d - nnz > 0 ? d - nnz : 0;
    long long hi = d < nrow ? d : nrow;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((long long)__ldg(row_ptr + mid + 1) <= d - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    coords[t] = make_int2((int)(d - lo), (int)(lo < nrow ? lo : nrow));
}

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[64] = {};

// Device address of the scratch array on the current device.  The first
// call on a device looks it up, initializes the array on `s` and waits for
// that, so a later call on any stream finds it ready; it is refused while
// `s` is being captured (the set-up must run, not be recorded).
int noalloc_scratch(unsigned char** out, cudaStream_t s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "spmv_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(MERBIT_ERR_UNSUPPORTED, "spmv_noalloc: device ordinal >= 64");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        e = cudaStreamIsCapturing(s, &cs);
        if (e != cudaSuccess) return cuda_fail(e, "spmv_noalloc: cudaStreamIsCapturing");
        if (cs != cudaStreamCaptureStatusNone)
            return fail(MERBIT_ERR_INVALID,
                        "spmv_noalloc: the first call on a device sets up its scratch and "
                        "must not run under stream capture");
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "spmv_noalloc: cudaGetSymbolAddress");
        noalloc_init_kernel<<<64, 256, 0, s>>>(static_cast<unsigned char*>(p));
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "spmv_noalloc: init kernel");
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return MERBIT_OK;
}

}  // namespace
}  // namespace merbit

using namespace merbit;

extern "C" int merbit_spmv_noalloc(int32_t nrow, int32_t ncol, int32_t nnz,
                                   const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                   const void* d_vals, merbit_dtype dtype, double alpha,
                                   const void* d_x, double beta, void* d_y, void* stream) {
    if (nrow < 0 || ncol < 0 || nnz < 0) return fail(MERBIT_ERR_INVALID, "spmv_noalloc: negative size");
    if (dtype != MERBIT_F64 && dtype != MERBIT_F32 && dtype != MERBIT_BF16)
        return fail(MERBIT_ERR_INVALID, "spmv_noalloc: unknown dtype");
    if ((long long)nrow + nnz > kNoAllocMaxItems)
        return fail(MERBIT_ERR_INVALID,
                    "spmv_noalloc: nrow + nnz = " + std::to_string((long long)nrow + nnz) +
                        " exceeds this entry point's fixed scratch limit of " +
                        std::to_string(kNoAllocMaxItems) +
                        " (use merbit_plan_create / merbit_spmv for larger matrices)");
    if (nrow == 0) return MERBIT_OK;
    if (!d_row_ptr || !d_y || (nnz > 0 && (!d_col_idx || !d_vals)) || (ncol > 0 && !d_x))
        return fail(MERBIT_ERR_INVALID, "spmv_noalloc: null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* scratch = nullptr;
    int st = noalloc_scratch(&scratch, s);
    if (st != MERBIT_OK) return st;

    const long long total = (long long)nrow + nnz;
    const int num_tiles = (int)((total + kNoAllocTileItems - 1) / kNoAllocTileItems);
    noalloc_prepare_kernel<<<(num_tiles + 1 + 255) / 256, 256, 0, s>>>(d_row_ptr, nrow, nnz,
                                                                       num_tiles, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "spmv_noalloc: prepare kernel");

    int cfg = -1;
    for (int i = 0; i < spmv_num_configs(dtype); ++i) {
        const SpmvConfig c = spmv_config(dtype, i);
        if (c.kind == 0 && c.block == kNoAllocBlock && c.ipt == kNoAllocIpt) cfg = i;
    }
    if (cfg < 0) return fail(MERBIT_ERR_UNSUPPORTED, "spmv_noalloc: kernel configuration missing");

    SpmvLaunch a;
    a.row_ptr = d_row_ptr;
    a.col = d_col_idx;
    a.vals = d_vals;
    a.x = d_x;
    a.y = d_y;
    a.coords = reinterpret_cast<const int2*>(scratch + kStateBytes);
    a.slots = reinterpret_cast<unsigned long long*>(scratch + kStateBytes + kCoordPad);
    a.xch = a.slots + 2 * (size_t)kNoAllocMaxTiles;
    a.state = reinterpret_cast<LaunchState*>(scratch);
    a.nrow = nrow;
    a.nnz = nnz;
    a.num_tiles = num_tiles;
    a.nslots = kNoAllocMaxTiles;
    a.alpha = alpha;
    a.beta = beta;
    const bool vec = ((uintptr_t)d_col_idx & 15u) == 0 && ((uintptr_t)d_vals & 15u) == 0;
    return spmv_launch(dtype, cfg, vec, a, s);
}

extern "C" int merbit_spmv_noalloc_check(void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* scratch = nullptr;
    int st = noalloc_scratch(&scratch, s);
    if (st != MERBIT_OK) return st;
    // the live word of the launch state and the report word the prepare
    // kernel moves it to; both are read and cleared on `stream`
    int words[2] = {0, 0};
    const size_t err_off = offsetof(LaunchState, error);
    MERBIT_CUDA(cudaMemcpyAsync(&words[0], scratch + err_off, sizeof(int), cudaMemcpyDeviceToHost, s));
    MERBIT_CUDA(cudaMemcpyAsync(&words[1], scratch + kReportOffset, sizeof(int),
                                cudaMemcpyDeviceToHost, s));
    MERBIT_CUDA(cudaStreamSynchronize(s));
    if (words[0] == 0 && words[1] == 0) return MERBIT_OK;
    MERBIT_CUDA(cudaMemsetAsync(scratch + err_off, 0, sizeof(int), s));
    MERBIT_CUDA(cudaMemsetAsync(scratch + kReportOffset, 0, sizeof(int), s));
    MERBIT_CUDA(cudaStreamSynchronize(s));
    return fail(words[0] != 0 ? words[0] : words[1],
                "spmv_noalloc: a device-side wait ran out in a call since the last check");
}

extern "C" int merbit_spmv_noalloc_selftest_wait(int32_t which, int32_t wait_us, void* stream) {
    if (which != 0 && which != 1) return fail(MERBIT_ERR_INVALID, "selftest_wait: which is 0 or 1");
    if (wait_us < 1 || wait_us > 1000000)
        return fail(MERBIT_ERR_INVALID, "selftest_wait: wait_us outside [1, 1e6]");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* scratch = nullptr;
    int st = noalloc_scratch(&scratch, s);
    if (st != MERBIT_OK) return st;
    return selftest_wait_on(reinterpret_cast<LaunchState*>(scratch), which, wait_us, s);
}
