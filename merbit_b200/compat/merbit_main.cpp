// A harness in the shape of the reference's src/main.cu, built against
// include/merbit_compat.hpp: the same ENV / GRAPH / PARAMETER / Fun_Merbit
// calls, with the device id, config and log path taken from the command line
// instead of hard-coded (src/main.cu:6-8).
//
//   merbit_main <gid> <config> <log> [device] [y_out.bin]
//
// y_out.bin, when given, receives pagerank_real (nrow values of ValueType).
#include <cstdio>

#include "merbit_compat.hpp"

#ifndef VALUETYPE
#define VALUETYPE double
#endif

std::fstream FSTR;

int main(int argc, char* argv[]) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <gid> <config> <log> [device] [y_out.bin]\n", argv[0]);
        return 2;
    }
    const int gid = std::stoi(argv[1]);
    const std::string config = argv[2];
    const std::string log = argv[3];
    const int device_id = argc > 4 ? std::stoi(argv[4]) : 0;
    FSTR.open(log, std::ios_base::out | std::ios_base::app);
    try {
        ENV env(device_id, config, log);
        using ValueType = VALUETYPE;
        GRAPH<ValueType> graph(config, gid);
        PARAMETER<ValueType> para(&graph, 0.85, 20, 20);
        const int BLOCK = 256;
        const int SIGMA = 14;
        Fun_Merbit<ValueType, BLOCK, SIGMA>(env, para);
        if (argc > 5) {
            std::vector<ValueType> y((size_t)graph.nrow);
            cudaMemcpy(y.data(), para.pagerank_real, sizeof(ValueType) * y.size(),
                       cudaMemcpyDeviceToHost);
            std::FILE* f = std::fopen(argv[5], "wb");
            if (!f) throw std::runtime_error("cannot write y");
            std::fwrite(y.data(), sizeof(ValueType), y.size(), f);
            std::fclose(f);
        }
        std::cout << "graph = " << graph.graph_id << ", block = " << BLOCK << ", sigma = " << SIGMA
                  << std::endl;
    } catch (const std::exception& e) {
        std::cerr << "Exception caught: " << e.what() << std::endl;
        FSTR.close();
        return 1;
    }
    FSTR.close();
    return 0;
}
