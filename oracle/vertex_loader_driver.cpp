// Test infrastructure: GraphLoader's vertex-file readers
// (loader/graph_loader.h:131-227) on one file: LoadVertexStatusFromTxt with
// an integer token parser, a floating-point token parser and a raw-string
// parser, then LoadVertexVecFromTxt<cpu, float>.  Results go to OUT (the
// loaders log to stdout).  Compiled once against GraphOne's own headers
// (_ref/tests_ref/vertex_loader) and once against this repository's.
// Usage: vertex_loader_driver FILE REORDER(0|1) N OUT
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "GraphOne/utils/string.hpp"
#include "GraphOne/loader/graph_loader.h"

using namespace graph_one;

int main(int argc, char** argv) {
    if (argc != 5) return 2;
    const bool reorder = argv[2][0] == '1';
    const vid_t n = (vid_t)std::strtoul(argv[3], nullptr, 10);
    FILE* o = std::fopen(argv[4], "w");
    if (!o) return 4;
    {
        GraphLoader<vstart_t::FROM_0_TO_0> loader(reorder);
        loader.LoadVertexStatusFromTxt<int32_t>(argv[1], [&](vid_t vid, std::vector<int32_t>& v) {
            std::fprintf(o, "T %u", (unsigned)vid);
            for (auto x : v) std::fprintf(o, " %d", x);
            std::fprintf(o, "\n");
            return v.size() != 2;  // rows of two values take the warning path
        });
    }
    {
        GraphLoader<vstart_t::FROM_0_TO_0> loader(reorder);
        loader.LoadVertexStatusFromTxt<double>(argv[1], [&](vid_t vid, std::vector<double>& v) {
            std::fprintf(o, "D %u", (unsigned)vid);
            for (auto x : v) std::fprintf(o, " %.17g", x);
            std::fprintf(o, "\n");
            return true;
        });
    }
    {
        GraphLoader<vstart_t::FROM_0_TO_0> loader(reorder);
        loader.LoadVertexStatusFromTxt<char*>(argv[1], [&](vid_t vid, char* rest) {
            std::fprintf(o, "S %u [%s]\n", (unsigned)vid, rest ? rest : "");
            return true;
        });
    }
    {
        GraphLoader<vstart_t::FROM_0_TO_0> loader(false);
        auto vec = loader.LoadVertexVecFromTxt<arch_t::cpu, float>(argv[1], n);
        std::fprintf(o, "V");
        for (vid_t i = 0; i < n; ++i) std::fprintf(o, " %.9g", (double)vec[i]);
        std::fprintf(o, "\n");
    }
    std::fclose(o);
    return 0;
}
