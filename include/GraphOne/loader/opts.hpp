#pragma once
// Edge-list loading options (reference: loader/opts.hpp:7-34).

#include <string>

#include "GraphOne/utils/string.hpp"

namespace graph_one {

struct LoadEdgeOpts {
    std::string file_ext = ".adj";      // required file name suffix
    std::string comment_prefix = "%";   // lines starting with it are skipped
    std::string line_sep = " \t";       // field separators
    bool is_directed = false;           // undirected input is symmetrised
    bool keep_self_loop = false;
    bool keep_duplicate_edges = false;

    std::string ToString() const {
        return "LoadEdgeOpts{ file_ext: " + file_ext + ", comment_prefix: " + comment_prefix +
               ", line_sep: " + line_sep + ", is_directed: " + utils::ToString(is_directed) +
               ", keep_self_loop: " + utils::ToString(keep_self_loop) +
               ", keep_duplicate_edges: " + utils::ToString(keep_duplicate_edges) + " }";
    }
};

struct LoadVertexOpts {
    std::string comment_prefix = "%";
    std::string vertex_sep = " \t";
    std::string vdata_sep = " \t";
};

}  // namespace graph_one
