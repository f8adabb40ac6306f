/*
 * C++ host API of the Merbit harness, re-expressed over the merbit_b200 C
 * ABI, so that a harness written against the reference (src/main.cu) builds
 * unchanged against this header and libmerbit_b200.so.
 *
 *   Timer        include/class.cuh:5-31
 *   ENV          include/class.cuh:36-59   (stream only: no cuSPARSE/cuBLAS
 *                                            handles -- nothing here uses them)
 *   GRAPH<V>     include/class.cuh:62-81, src/class.cu:50-177,417-425
 *                (Matrix Market loader with the reference's symmetric doubling,
 *                 "basezero" detection and 1/outdegree values; sort)
 *   PARAMETER<V> include/class.cuh:119-146
 *   TILE<B,S>    include/tile.cuh:6-25,106-122  (the reference plan format,
 *                built by merbit_tile_build)
 *   Fun_Merbit<V,B,S>  include/tile.cuh:563-615  (same steps, same log line;
 *                the SpMV is merbit_spmv on a plan)
 *
 * Header-only host C++ (no kernels): compile with any C++17 compiler, link
 * libmerbit_b200.so and the CUDA runtime.  Errors throw std::runtime_error
 * with merbit_last_error_detail() (the reference printed and went on).
 * The harness defines `std::fstream FSTR;` as src/main.cu:2 does.
 */
#ifndef MERBIT_COMPAT_HPP
#define MERBIT_COMPAT_HPP

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "merbit.h"

extern std::fstream FSTR;

namespace merbit_compat {
inline void check(int status, const char* where) {
    if (status != MERBIT_OK)
        throw std::runtime_error(std::string(where) + ": " + merbit_status_string(status) + ": " +
                                 merbit_last_error_detail());
}
inline void check_cuda(cudaError_t e, const char* where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}
template <typename V>
struct dtype_of;
template <>
struct dtype_of<double> {
    static constexpr merbit_dtype value = MERBIT_F64;
};
template <>
struct dtype_of<float> {
    static constexpr merbit_dtype value = MERBIT_F32;
};
}  // namespace merbit_compat

struct Timer {
    cudaEvent_t start_event, stop_event;
    Timer() {
        cudaEventCreate(&start_event);
        cudaEventCreate(&stop_event);
    }
    void start(cudaStream_t stream) {
        cudaDeviceSynchronize();
        cudaEventRecord(start_event, stream);
    }
    float stop(cudaStream_t stream) {
        cudaEventRecord(stop_event, stream);
        cudaEventSynchronize(stop_event);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, start_event, stop_event);
        return ms;
    }
    ~Timer() {
        cudaEventDestroy(start_event);
        cudaEventDestroy(stop_event);
    }
};

struct ENV {
    const int device_id = 0;
    const std::string config;
    const std::string log;
    cudaStream_t stream;
    ENV(const int id, const std::string& config, const std::string log)
        : device_id(id), config(config), log(log) {
        merbit_compat::check_cuda(cudaSetDevice(device_id), "ENV: cudaSetDevice");
        merbit_compat::check_cuda(cudaStreamCreate(&stream), "ENV: cudaStreamCreate");
    }
    ~ENV() { cudaStreamDestroy(stream); }
};

template <typename ValueType>
struct GRAPH {
    int graph_id = -1;
    int nrow = 0;
    int nnz = 0;
    bool owner = true;
    int* row_ind = nullptr;
    int* col_ind = nullptr;
    ValueType* values = nullptr;

    GRAPH() {}
    GRAPH(const bool own) : owner(own) {}

    // src/class.cu:60-141: find `gid` in the config file ("id path ..."
    // per line), read the Matrix Market file (a "symmetric" header doubles
    // every entry, a "basezero" header means zero-based indices), upload,
    // and replace the values by 1/outdegree of row_ind.
    GRAPH(const std::string& config, const int gid) {
        std::ifstream cf(config);
        if (!cf) throw std::runtime_error("GRAPH: cannot open config " + config);
        std::string line, filename;
        int id = -1;
        bool found = false;
        while (std::getline(cf, line)) {
            std::stringstream ss(line);
            if (ss >> id >> filename && id == gid) {
                found = true;
                break;
            }
        }
        if (!found) throw std::runtime_error("GRAPH: graph id not in config");
        std::ifstream mf(filename);
        if (!mf) throw std::runtime_error("GRAPH: cannot open " + filename);
        bool symmetric = false, zero_base = false;
        int i = 0;
        do {
            std::getline(mf, line);
            if (i == 0) {
                symmetric = line.find("symmetric") != std::string::npos;
                zero_base = line.find("basezero") != std::string::npos;
            }
            ++i;
        } while (!line.empty() && line[0] == '%');
        long long R = 0, Cc = 0, N = 0;
        std::stringstream(line) >> R >> Cc >> N;
        graph_id = gid;
        nrow = (int)R;
        nnz = (int)(symmetric ? 2 * N : N);
        std::vector<int> hr(nnz), hc(nnz);
        long long k = 0;
        while (k < N && std::getline(mf, line)) {
            if (line.empty() || line[0] == '%') continue;
            long long r = 0, c = 0;
            std::stringstream(line) >> r >> c;
            hr[k] = (int)(zero_base ? r : r - 1);
            hc[k] = (int)(zero_base ? c : c - 1);
            if (symmetric) {
                hr[N + k] = hc[k];
                hc[N + k] = hr[k];
            }
            ++k;
        }
        if (k != N) throw std::runtime_error("GRAPH: " + filename + " has fewer entries than its header says");
        merbit_compat::check_cuda(cudaMalloc(&row_ind, sizeof(int) * (size_t)std::max(nnz, 1)), "GRAPH");
        merbit_compat::check_cuda(cudaMalloc(&col_ind, sizeof(int) * (size_t)std::max(nnz, 1)), "GRAPH");
        merbit_compat::check_cuda(cudaMalloc(&values, sizeof(ValueType) * (size_t)std::max(nnz, 1)), "GRAPH");
        cudaMemcpy(row_ind, hr.data(), sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice);
        cudaMemcpy(col_ind, hc.data(), sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice);
        merbit_compat::check(merbit_outdegree_values(nnz, nrow, row_ind, values,
                                                     merbit_compat::dtype_of<ValueType>::value, nullptr),
                             "GRAPH: values");
    }

    // src/class.cu:143-177: dir = true orders by (row_ind, col_ind), false
    // by (col_ind, row_ind).
    void sort(const bool dir) {
        if (dir)
            merbit_compat::check(merbit_coo_sort(nnz, row_ind, col_ind, values,
                                                 merbit_compat::dtype_of<ValueType>::value, nullptr),
                                 "GRAPH::sort");
        else
            merbit_compat::check(merbit_coo_sort(nnz, col_ind, row_ind, values,
                                                 merbit_compat::dtype_of<ValueType>::value, nullptr),
                                 "GRAPH::sort");
    }

    // src/class.cu:384-415: prints the dense matrix (small graphs only).
    void show() {
        std::vector<int> r(nnz), c(nnz);
        std::vector<ValueType> v(nnz);
        cudaMemcpy(r.data(), row_ind, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost);
        cudaMemcpy(c.data(), col_ind, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost);
        cudaMemcpy(v.data(), values, sizeof(ValueType) * (size_t)nnz, cudaMemcpyDeviceToHost);
        std::vector<ValueType> d((size_t)nrow * nrow, 0);
        for (int e = 0; e < nnz; ++e) d[(size_t)r[e] * nrow + c[e]] += v[e];
        for (int a = 0; a < nrow; ++a) {
            for (int b = 0; b < nrow; ++b) std::cout << " " << d[(size_t)a * nrow + b];
            std::cout << "\n";
        }
    }

    ~GRAPH() {
        if (owner) {
            cudaFree(row_ind);
            cudaFree(col_ind);
            cudaFree(values);
        }
    }
};

template <typename ValueType>
struct PARAMETER {
    GRAPH<ValueType>* graph;
    double damp;
    int perrnd;
    int maxiter;
    int iter;
    int BOUND;
    char TYPE;
    ValueType* person;
    ValueType* pagerank_real;
    PARAMETER(GRAPH<ValueType>* graph, double damp, int perrnd, int maxiter)
        : graph(graph), damp(damp), perrnd(perrnd), maxiter(maxiter), iter(0), BOUND(0), TYPE(0) {
        merbit_compat::check_cuda(cudaMalloc(&person, sizeof(ValueType) * (size_t)std::max(graph->nrow, 1)), "PARAMETER");
        merbit_compat::check_cuda(cudaMalloc(&pagerank_real, sizeof(ValueType) * (size_t)std::max(graph->nrow, 1)), "PARAMETER");
        std::vector<ValueType> ones((size_t)graph->nrow, (ValueType)1.0);  // include/class.cuh:139
        cudaMemcpy(person, ones.data(), sizeof(ValueType) * ones.size(), cudaMemcpyHostToDevice);
    }
    ~PARAMETER() {
        cudaFree(person);
        cudaFree(pagerank_real);
    }
};

template <unsigned int BLOCK, unsigned int SIGMA>
struct TILE {
    unsigned int* tile_x = nullptr;
    unsigned int* tile_y = nullptr;
    void* lane_desc = nullptr;  // unsigned int[] when SIGMA < 15, unsigned long long[] otherwise
    int tile_num = 0;
    int lane_num = 0;
    TILE() {}
    TILE(const int* offset, const int nrow, const int nnz) {
        merbit_compat::check(merbit_tile_dims(nrow, nnz, (int)SIGMA, &tile_num, &lane_num), "TILE");
        const size_t dsz = SIGMA < 15 ? sizeof(unsigned int) : sizeof(unsigned long long);
        merbit_compat::check_cuda(cudaMalloc(&tile_x, sizeof(unsigned) * (size_t)(tile_num + 1)), "TILE");
        merbit_compat::check_cuda(cudaMalloc(&tile_y, sizeof(unsigned) * (size_t)(tile_num + 1)), "TILE");
        merbit_compat::check_cuda(cudaMalloc(&lane_desc, dsz * (size_t)std::max(lane_num, 1)), "TILE");
        merbit_compat::check(merbit_tile_build(offset, nrow, nnz, (int)SIGMA, tile_x, tile_y, lane_desc,
                                               nullptr),
                             "TILE");
    }
    ~TILE() {
        cudaFree(tile_x);
        cudaFree(tile_y);
        cudaFree(lane_desc);
    }
};

// include/tile.cuh:563-615: sort the COO by (col, row), build the offsets,
// build the plan (timed as tim1), run maxiter*perrnd SpMVs y = P^T x with
// the y/z ping-pong (timed as tim2, reported per SpMV), copy the last y to
// pagerank_real and append " gid&MERBIT&SIGMA&tim1&tim2/n" to FSTR.  As in
// the reference, the CSR rows are col_ind and the CSR columns row_ind.
template <typename ValueType, unsigned int BLOCK, unsigned int SIGMA>
void Fun_Merbit(const ENV& env, const PARAMETER<ValueType>& para) {
    Timer timer;
    float tim1 = 0.f, tim2 = 0.f;
    GRAPH<ValueType>* g = para.graph;
    g->sort(false);
    int* offset = nullptr;
    merbit_compat::check_cuda(cudaMalloc(&offset, sizeof(int) * ((size_t)g->nrow + 1)), "Fun_Merbit");
    merbit_compat::check(merbit_coo_to_csr(g->nnz, g->col_ind, g->nrow, offset, env.stream), "Fun_Merbit");
    ValueType *d_y = nullptr, *d_z = nullptr;
    merbit_compat::check_cuda(cudaMalloc(&d_y, sizeof(ValueType) * (size_t)std::max(g->nrow, 1)), "Fun_Merbit");
    merbit_compat::check_cuda(cudaMalloc(&d_z, sizeof(ValueType) * (size_t)std::max(g->nrow, 1)), "Fun_Merbit");

    timer.start(env.stream);
    merbit_plan plan = nullptr;
    merbit_compat::check(merbit_plan_create(&plan, g->nrow, g->nrow, g->nnz, offset, g->row_ind,
                                            g->values, merbit_compat::dtype_of<ValueType>::value, 0,
                                            env.stream),
                         "Fun_Merbit: plan");
    tim1 = timer.stop(env.stream);
    std::cout << "tim1 = " << tim1 << std::endl;

    cudaMemsetAsync(d_y, 0, sizeof(ValueType) * (size_t)g->nrow, env.stream);
    timer.start(env.stream);
    const int rounds = para.maxiter * para.perrnd;
    for (int rnd = 0; rnd < rounds; ++rnd) {
        merbit_compat::check(merbit_spmv(plan, 1.0, para.person, 0.0, d_y, env.stream), "Fun_Merbit: spmv");
        std::swap(d_y, d_z);
    }
    cudaMemcpyAsync(para.pagerank_real, d_z, sizeof(ValueType) * (size_t)g->nrow,
                    cudaMemcpyDeviceToDevice, env.stream);
    tim2 = timer.stop(env.stream);
    merbit_compat::check(merbit_plan_check(plan, env.stream), "Fun_Merbit: device status");
    FSTR << " " << g->graph_id << "&MERBIT&" << SIGMA << "&" << tim1 << "&"
         << tim2 / (rounds > 0 ? rounds : 1) << "\n";
    merbit_plan_destroy(plan);
    cudaFree(offset);
    cudaFree(d_y);
    cudaFree(d_z);
}

#endif /* MERBIT_COMPAT_HPP */
