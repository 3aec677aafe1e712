// Prints the CSR that the drop-in GraphOne loader (include/GraphOne/loader/
// loader.h) builds from an .adj file: for the out-edge then the in-edge
// orientation, a line "n m" and the row offsets, columns and values, then
// the same for GraphLoader::LoadCsrFromTxt (out-edge CSR).
// Usage: loader_driver FILE.adj DIRECTED REORDER KEEP_SELF KEEP_DUP (each 0|1)
#include <cstdio>

#include "GraphOne/loader/loader.h"

using namespace graph_one;

int main(int argc, char** argv) {
    if (argc != 6) return 2;
    LoadEdgeOpts opts;
    opts.is_directed = argv[2][0] == '1';
    opts.keep_self_loop = argv[4][0] == '1';
    opts.keep_duplicate_edges = argv[5][0] == '1';
    GraphLoader<vstart_t::FROM_0_TO_0> loader(argv[3][0] == '1');
    auto cache = loader.LoadEdgesFromTxt<uint32_t>(argv[1], opts);
    for (int t = 0; t < 2; ++t) {
        std::vector<eid_t> rp;
        std::vector<vid_t> ci;
        std::vector<uint32_t> v;
        if (t)
            cache.BuildCsr<true>(rp, ci, v);
        else
            cache.BuildCsr<false>(rp, ci, v);
        std::printf("%u %llu\n", (unsigned)cache.num_vertices(), (unsigned long long)cache.num_edges());
        for (auto x : rp) std::printf("%llu ", (unsigned long long)x);
        std::printf("\n");
        for (auto x : ci) std::printf("%u ", (unsigned)x);
        std::printf("\n");
        for (auto x : v) std::printf("%u ", (unsigned)x);
        std::printf("\n");
    }
    // LoadCsrFromTxt: the out-edge CSR straight from the file
    GraphLoader<vstart_t::FROM_0_TO_0> loader2(argv[3][0] == '1');
    auto csr = loader2.LoadCsrFromTxt<arch_t::cpu, uint32_t>(argv[1], opts);
    std::printf("%u %llu\n", (unsigned)csr.n_rows, (unsigned long long)csr.nnz);
    for (size_t i = 0; i < csr.row_offsets.size(); ++i) std::printf("%llu ", (unsigned long long)csr.row_offsets[i]);
    std::printf("\n");
    for (size_t i = 0; i < csr.col_indices.size(); ++i) std::printf("%u ", (unsigned)csr.col_indices[i]);
    std::printf("\n");
    for (size_t i = 0; i < csr.values.size(); ++i) std::printf("%u ", (unsigned)csr.values[i]);
    std::printf("\n");
    // LoadCsrFromTxt with the arch argument alone: edge data defaults to double
    GraphLoader<vstart_t::FROM_0_TO_0> loader3(argv[3][0] == '1');
    auto csr_d = loader3.LoadCsrFromTxt<arch_t::cpu>(argv[1], opts);
    constexpr bool is_double = std::is_same_v<typename decltype(csr_d)::value_type, double>;
    std::printf("default-edata %u %llu %d\n", (unsigned)csr_d.n_rows, (unsigned long long)csr_d.nnz,
                (int)is_double);
    return 0;
}
