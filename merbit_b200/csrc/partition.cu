// Merge-path partitioning on sm_100a.
//
//  * merge_coords_kernel: one thread per requested diagonal, binary search
//    over row_ptr with the reference's predicate and tie rule
//    (include/utils.cuh:5-29): go right when row_ptr[mid+1] <= d - mid - 1,
//    so at equal positions the row end is consumed before the nonzero, and
//    coord_y is clamped to nrow.  Used for the SpMV plan (one diagonal per
//    tile boundary) and exported for parity checks.
//  * tile_build_kernel: the reference's Merbit plan format (TILE,
//    include/tile.cuh:4-122) reproduced bit for bit: one warp per tile of 32
//    lanes x sigma items, per-lane row-end bitmask and (dy, dx) offsets
//    packed 18/9 (32-bit) or 22/11 (64-bit), tile MSB flag for tiles without
//    a row end, sentinel (nnz, nrow).
//  * validate_kernel: structural checks of a caller's CSR arrays.
#include "merbit_internal.cuh"

namespace merbit {

__device__ __forceinline__ void merge_search_dev(const int32_t* __restrict__ row_ptr, int nrow,
                                                 int nnz, long long d, int* cx, int* cy) {
    long long lo = d - nnz > 0 ? d - nnz : 0;
    long long hi = d < nrow ? d : nrow;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((long long)__ldg(row_ptr + mid + 1) <= d - mid - 1)
            lo = mid + 1;
        else
            hi = mid;
    }
    *cx = (int)(d - lo);
    *cy = (int)(lo < nrow ? lo : nrow);
}

__global__ void merge_coords_kernel(const int32_t* __restrict__ row_ptr, int nrow, int nnz,
                                    long long stride, long long count, int* __restrict__ out_x,
                                    int* __restrict__ out_y, int2* __restrict__ out_xy) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long total = (long long)nrow + nnz;
    long long d = i * stride;
    if (d > total) d = total;
    int cx, cy;
    merge_search_dev(row_ptr, nrow, nnz, d, &cx, &cy);
    if (out_xy) {
        out_xy[i] = make_int2(cx, cy);
    } else {
        out_x[i] = cx;
        out_y[i] = cy;
    }
}

template <bool WIDE>
__global__ void tile_build_kernel(const int32_t* __restrict__ row_ptr, int nrow, int nnz,
                                  int sigma, int tile_num, int lane_num,
                                  unsigned* __restrict__ tile_x, unsigned* __restrict__ tile_y,
                                  void* __restrict__ lane_desc) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const long long tile = gid >> 5;
    if (gid == 0) {
        tile_x[tile_num] = (unsigned)nnz;
        tile_y[tile_num] = (unsigned)nrow;
    }
    if (tile >= tile_num) return;  // whole warp leaves together
    const bool active = gid < lane_num;
    const long long total = (long long)nrow + nnz;
    const long long d = gid * sigma;
    int cx = 0, cy = 0;
    if (active) merge_search_dev(row_ptr, nrow, nnz, d, &cx, &cy);
    const int wx = __shfl_sync(0xFFFFFFFFu, cx, 0);
    const int wy = __shfl_sync(0xFFFFFFFFu, cy, 0);
    unsigned long long bits = 0ull;
    const unsigned long long dx = (unsigned long long)(unsigned)(cx - wx);
    const unsigned long long dy = (unsigned long long)(unsigned)(cy - wy);
    if (active) {
        const long long rem = total - d;
        const int n = rem < sigma ? (int)rem : sigma;
        int end = cy < nrow ? __ldg(row_ptr + cy + 1) : INT_MAX;
        for (int idx = 0; idx < n; ++idx) {
            if (cx < end) {
                ++cx;
            } else {
                bits |= 1ull << idx;
                ++cy;
                end = cy < nrow ? __ldg(row_ptr + cy + 1) : INT_MAX;
            }
        }
        if (WIDE) {
            static_cast<unsigned long long*>(lane_desc)[gid] = (bits << 22) | (dy << 11) | dx;
        } else {
            static_cast<unsigned*>(lane_desc)[gid] = (unsigned)((bits << 18) | (dy << 9) | dx);
        }
    }
    const bool fast = __all_sync(0xFFFFFFFFu, !active || cy == wy);
    if (lane == 0) {
        tile_x[tile] = (unsigned)wx;
        tile_y[tile] = (unsigned)wy | (fast ? 0x80000000u : 0u);
    }
}

// err bits: 1 = row_ptr[0] != 0, 2 = row_ptr[nrow] != nnz, 4 = decreasing,
// 8 = column out of range.  first_bad receives the lowest offending index
// of the decreasing / column checks.
__global__ void validate_kernel(const int32_t* __restrict__ row_ptr,
                                const int32_t* __restrict__ col, int nrow, int ncol, int nnz,
                                int* __restrict__ err, int* __restrict__ first_bad,
                                int* __restrict__ max_len, bool check) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (check && i0 == 0) {
        if (__ldg(row_ptr) != 0) atomicOr(err, 1);
        if (__ldg(row_ptr + nrow) != nnz) atomicOr(err, 2);
    }
    int longest = 0;
    for (long long i = i0; i < nrow; i += stride) {
        const int len = __ldg(row_ptr + i + 1) - __ldg(row_ptr + i);
        if (len < 0) {
            if (check) {
                atomicOr(err, 4);
                atomicMin(first_bad, (int)i);
            }
        } else {
            longest = max(longest, len);
        }
    }
    for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xFFFFFFFFu, longest, o));
    if ((threadIdx.x & 31) == 0 && longest > 0) atomicMax(max_len, longest);
    if (!check) return;
    for (long long e = i0; e < nnz; e += stride) {
        const int c = __ldg(col + e);
        if (c < 0 || c >= ncol) {
            atomicOr(err, 8);
            atomicMin(first_bad + 1, (int)e);
        }
    }
}

__global__ void max_rows_kernel(const int2* __restrict__ coords, int num_tiles,
                                int* __restrict__ out) {
    int m = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < num_tiles;
         t += gridDim.x * blockDim.x)
        m = max(m, coords[t + 1].y - coords[t].y);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

int build_partition_async(const int32_t* row_ptr, int nrow, int nnz, int tile_items,
                          Partition* out, int* d_max_rows, cudaStream_t s) {
    const long long total = (long long)nrow + nnz;
    const long long T = (total + tile_items - 1) / tile_items;
    if (T > INT_MAX - 2) return fail(MERBIT_ERR_OVERFLOW, "partition: too many tiles");
    out->tile_items = tile_items;
    out->num_tiles = (int)T;
    out->max_rows = -1;
    int st = dev_alloc(&out->coords, sizeof(int2) * (size_t)(T + 1), s);
    if (st != MERBIT_OK) return st;
    const long long count = T + 1;
    const int bs = 256;
    const unsigned grid = (unsigned)((count + bs - 1) / bs);
    merge_coords_kernel<<<grid, bs, 0, s>>>(row_ptr, nrow, nnz, tile_items, count, nullptr,
                                            nullptr, out->coords);
    MERBIT_CUDA(cudaGetLastError());
    // largest rows-per-tile, which decides the configurations the plan can use
    if (T > 0) {
        max_rows_kernel<<<(unsigned)min((T + 255) / 256, 1024LL), 256, 0, s>>>(out->coords, (int)T,
                                                                               d_max_rows);
        MERBIT_CUDA(cudaGetLastError());
    }
    return MERBIT_OK;
}

int validate_launch(const int32_t* row_ptr, const int32_t* col, int nrow, int ncol, int nnz,
                    PlanScratch* sc, bool check, cudaStream_t s) {
    int dev = 0, sms = 148;
    MERBIT_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // blockDim a multiple of 32 and every thread reaches the warp reduction
    validate_kernel<<<sms * 8, 256, 0, s>>>(row_ptr, col, nrow, ncol, nnz, &sc->err,
                                            sc->first_bad, &sc->max_row_len, check);
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

int validate_status(const PlanScratch& h) {
    if (h.err & 1) return fail(MERBIT_ERR_MATRIX, "row_ptr[0] != 0");
    if (h.err & 2) return fail(MERBIT_ERR_MATRIX, "row_ptr[nrow] != nnz");
    if (h.err & 4)
        return fail(MERBIT_ERR_MATRIX,
                    "row_ptr decreases after row " + std::to_string(h.first_bad[0]));
    if (h.err & 8)
        return fail(MERBIT_ERR_MATRIX,
                    "column index out of range at nonzero " + std::to_string(h.first_bad[1]));
    return MERBIT_OK;
}

}  // namespace merbit

using namespace merbit;

extern "C" {

int merbit_merge_coords(const int32_t* d_row_ptr, int32_t nrow, int32_t nnz, int64_t stride,
                        int64_t count, int32_t* d_coord_x, int32_t* d_coord_y, void* stream) {
    if (nrow < 0 || nnz < 0 || stride < 0 || count < 0)
        return fail(MERBIT_ERR_INVALID, "merge_coords: negative size");
    if (count == 0) return MERBIT_OK;
    if (!d_row_ptr || !d_coord_x || !d_coord_y)
        return fail(MERBIT_ERR_INVALID, "merge_coords: null pointer");
    if ((long long)nrow + nnz > INT_MAX)
        return fail(MERBIT_ERR_OVERFLOW, "merge_coords: nrow+nnz exceeds int32");
    const int bs = 256;
    const long long grid = (count + bs - 1) / bs;
    if (grid > INT_MAX) return fail(MERBIT_ERR_INVALID, "merge_coords: count too large");
    merge_coords_kernel<<<(unsigned)grid, bs, 0, (cudaStream_t)stream>>>(
        d_row_ptr, nrow, nnz, stride, count, d_coord_x, d_coord_y, nullptr);
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

int merbit_tile_dims(int32_t nrow, int32_t nnz, int32_t sigma, int32_t* tile_num,
                     int32_t* lane_num) {
    if (nrow < 0 || nnz < 0 || sigma < 1 || sigma > 42 || !tile_num || !lane_num)
        return fail(MERBIT_ERR_INVALID, "tile_dims: bad argument");
    const long long ln = ((long long)nrow + nnz + sigma - 1) / sigma;
    if ((long long)nrow + nnz > INT_MAX) return fail(MERBIT_ERR_OVERFLOW, "tile_dims: overflow");
    *lane_num = (int32_t)ln;
    *tile_num = (int32_t)((ln + 31) / 32);
    return MERBIT_OK;
}

int merbit_tile_build(const int32_t* d_row_ptr, int32_t nrow, int32_t nnz, int32_t sigma,
                      uint32_t* d_tile_x, uint32_t* d_tile_y, void* d_lane_desc, void* stream) {
    int32_t tile_num = 0, lane_num = 0;
    int st = merbit_tile_dims(nrow, nnz, sigma, &tile_num, &lane_num);
    if (st != MERBIT_OK) return st;
    if (!d_row_ptr || !d_tile_x || !d_tile_y || (lane_num > 0 && !d_lane_desc))
        return fail(MERBIT_ERR_INVALID, "tile_build: null pointer");
    const int bs = 256;
    const long long threads = (long long)tile_num * 32;
    const unsigned grid = (unsigned)(threads > 0 ? (threads + bs - 1) / bs : 1);
    cudaStream_t s = (cudaStream_t)stream;
    if (sigma >= 15)
        tile_build_kernel<true><<<grid, bs, 0, s>>>(d_row_ptr, nrow, nnz, sigma, tile_num,
                                                    lane_num, d_tile_x, d_tile_y, d_lane_desc);
    else
        tile_build_kernel<false><<<grid, bs, 0, s>>>(d_row_ptr, nrow, nnz, sigma, tile_num,
                                                     lane_num, d_tile_x, d_tile_y, d_lane_desc);
    MERBIT_CUDA(cudaGetLastError());
    return MERBIT_OK;
}

}  // extern "C"
