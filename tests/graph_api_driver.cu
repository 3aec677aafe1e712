// Builds a graph with GraphOne's graph::build (both views) from an .adj file
// and writes what the Graph accessors return.
//   graph_api_driver FILE.adj OUT
// OUT: u32 n, u32 m, u32 out_degree[n], u32 in_degree[n], then graph_mat()
//      (row_offsets n+1, col m, val m) and graph_transpose_mat() (same).
#include <cstdio>
#include <type_traits>
#include <vector>

#include "GraphOne/graph_one.h"

using namespace graph_one;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    LoadEdgeOpts opts;
    opts.is_directed = true;
    GraphLoader<vstart_t::FROM_0_TO_0> loader;
    auto cache = loader.LoadEdgesFromTxt<uint32_t>(argv[1], opts);
    auto g = graph::build<arch_t::cuda, BlasViews | graph_view_t::normal>(cache);
    static_assert(std::is_same_v<std::decay_t<decltype(g.vprops())>, empty_t>);
    const uint32_t n = g.num_vertices(), m = g.num_edges();
    std::vector<uint32_t> od(n), id(n);
    for (uint32_t v = 0; v < n; ++v) {
        od[v] = g.get_out_degree(v);
        id[v] = g.get_in_degree(v);
    }
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 4;
    std::fwrite(&n, 4, 1, o);
    std::fwrite(&m, 4, 1, o);
    std::fwrite(od.data(), 4, n, o);
    std::fwrite(id.data(), 4, n, o);
    for (const auto* mat : {&g.graph_mat(), &g.graph_transpose_mat()}) {
        const auto rp = mat->row_offsets.template to<arch_t::cpu>();
        const auto ci = mat->col_indices.template to<arch_t::cpu>();
        const auto vv = mat->values.template to<arch_t::cpu>();
        std::fwrite(rp.data(), 4, n + 1, o);
        std::fwrite(ci.data(), 4, m, o);
        std::fwrite(vv.data(), 4, m, o);
    }
    std::fclose(o);
    return 0;
}
