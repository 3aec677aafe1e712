// Test infrastructure: parses a command line the way GraphOne's apps declare
// theirs (apps/sssp_blas.cu:88-96: add_common_args + a required --src;
// apps/pagerank_blas.cu:129-137: an optional --alpha) and prints the parsed
// values, one per line.  Compiled once against GraphOne's own
// utils/cli.hpp (CLI11 2.3.2, into _ref/cli_ref) and once against this
// repository's include/GraphOne/utils/cli.hpp, so the two parsers can be
// compared on the same argument vectors (exit code and output).
#include <cstdint>
#include <cstdio>
#include <string>

#include "GraphOne/utils/string.hpp"
#include "GraphOne/utils/cli.hpp"

using namespace graph_one;

int main(int argc, char** argv) {
    std::string input_graph, output_path;
    bool reorder = false;
    LoadEdgeOpts opts;
    uint32_t src = 0;
    float alpha = 0.85f;
    CLI::App app;
    add_common_args(app, input_graph, output_path, reorder, opts);
    app.add_option("--src", src, "source vertex in SSSP")->required();
    app.add_option("--alpha", alpha, "alpha (factor) in PageRank");
    CLI11_PARSE(app, argc, argv);
    std::printf("input=%s\noutput=%s\nreorder=%d\nfile_ext=%s\ncomment_prefix=%s\nline_sep=[%s]\n",
                input_graph.c_str(), output_path.c_str(), (int)reorder, opts.file_ext.c_str(),
                opts.comment_prefix.c_str(), opts.line_sep.c_str());
    std::printf("directed=%d\nkeep_self=%d\nkeep_dup=%d\nsrc=%u\nalpha=%.9g\n", (int)opts.is_directed,
                (int)opts.keep_self_loop, (int)opts.keep_duplicate_edges, (unsigned)src, (double)alpha);
    return 0;
}
