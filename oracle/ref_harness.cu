// Runs the reference's own GPU decomposition, dcore(Graph&) (main.cu:197-262),
// on a graph stored in its binary layout and writes the result with its own
// writer, writeDecompFile (src/utils.h:97-108).  Test and benchmark
// infrastructure only: compiled by oracle/ref_build.py together with the
// reference's sources into oracle/_ref/ref_dcore.
//
//   ref_dcore <base> <out>   reads <base>-binary-g=1, writes <out>.decomp and
//                            prints one JSON line with the host-timed call
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#include "graph.h"

#undef main

std::vector<std::vector<degree>>& dcore(Graph& g);
void writeDecompFile(Graph& g, const std::string& filename);

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <graph base path> <output base path>\n", argv[0]);
        return 2;
    }
    Graph g{std::string(argv[1])};
    if (g.V >= 1000000u) {
        // the reference's per-block peel buffers hold 1,000,000 entries
        // without a bound check (src/cuda_utils.cuh:10-13)
        std::fprintf(stderr, "refusing V = %u >= 1,000,000\n", g.V);
        return 3;
    }
    cudaFree(nullptr);  // context creation outside the timed call
    auto t0 = std::chrono::steady_clock::now();
    dcore(g);
    cudaError_t e = cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e));
        return 4;
    }
    writeDecompFile(g, std::string(argv[2]));
    std::printf("{\"V\": %u, \"E\": %u, \"kmax\": %d, \"lmax\": %d, \"ms\": %.3f}\n", g.V, g.E, g.kmax, g.lmax,
                std::chrono::duration<double, std::milli>(t1 - t0).count());
    return 0;
}
