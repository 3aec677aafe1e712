#pragma once
// Edge-list ingest of the GraphOne API (reference: loader/graph_loader.h:
// 32-122, loader/edge_cache.h:50-105, mat/csr.h:16-68).
//
// A ".adj" text file holds one edge per line, "src dst [weight]" (a missing
// weight reads as 1); lines starting with the comment prefix are skipped.
// Self loops are dropped unless kept, undirected inputs get both
// directions, ids may be renumbered in first-seen order, and duplicates are
// merged after sorting by (src, dst) -- here with a stable sort, so the
// first occurrence in the file keeps its weight.  num_vertices is the
// largest id + 1.  ToCsr is a counting sort (stable in edge order).

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "GraphOne/base/buffer.h"
#include "GraphOne/loader/opts.hpp"
#include "GraphOne/type.hpp"
#include "GraphOne/utils/log.hpp"
#include "GraphOne/utils/string.hpp"

namespace graph_one {

template <arch_t arch, typename value_t, typename index_t = uint32_t, typename offset_t = uint64_t,
          vstart_t v_start = vstart_t::FROM_0_TO_0>
struct CsrMat {
    constexpr static arch_t arch_value = arch;
    constexpr static vstart_t vstart_value = v_start;
    using value_type = value_t;
    using index_type = index_t;
    using offset_type = offset_t;

    CsrMat() = default;
    CsrMat(index_t rows, index_t cols, offset_t nz, Buffer<arch, offset_t, index_t>&& rp,
           Buffer<arch, index_t, offset_t>&& ci, Buffer<arch, value_t, offset_t>&& v)
        : n_rows(rows), n_cols(cols), nnz(nz), row_offsets(std::move(rp)),
          col_indices(std::move(ci)), values(std::move(v)) {}

    std::string ToString() const {
        return "CsrMat{ arch_value:" + utils::ToString(arch_value) + ", n_rows:" + utils::NumToString(n_rows) +
               ", n_cols:" + utils::NumToString(n_cols) + ", nnz:" + utils::NumToString(nnz) +
               ", row_offsets:" + row_offsets.ToString() + ", col_indices:" + col_indices.ToString() +
               ", values:" + values.ToString() + " }";
    }

    index_t n_rows{0};
    index_t n_cols{0};
    offset_t nnz{0};
    Buffer<arch, offset_t, index_t> row_offsets;
    Buffer<arch, index_t, offset_t> col_indices;
    Buffer<arch, value_t, offset_t> values;
};

template <typename edata_t, typename index_t>
struct EdgeUnit {
    index_t src;
    index_t dst;
    edata_t edata;
    bool operator<(const EdgeUnit& o) const { return src < o.src || (src == o.src && dst < o.dst); }
    bool operator==(const EdgeUnit& o) const { return src == o.src && dst == o.dst; }
};

template <vstart_t v_start, typename edata_t, typename index_t, typename offset_t>
class EdgeCache : public std::vector<EdgeUnit<edata_t, index_t>> {
    using base_t = std::vector<EdgeUnit<edata_t, index_t>>;

public:
    void push_back(const EdgeUnit<edata_t, index_t>& e) {
        base_t::push_back(e);
        max_vid_ = std::max(max_vid_, std::max(e.src, e.dst));
    }
    index_t max_vid() const { return max_vid_; }
    offset_t num_edges() const { return offset_t(base_t::size()); }
    index_t num_vertices() const { return max_vid_ + 1; }

    // Host CSR arrays (row offsets n+1, columns, values), rows by src or, with
    // transpose, by dst.
    template <bool transpose>
    void BuildCsr(std::vector<offset_t>& rp, std::vector<index_t>& ci,
                  std::vector<edata_t>& val) const {
        const index_t n = num_vertices();
        const offset_t m = num_edges();
        rp.assign(size_t(n) + 1, 0);
        ci.resize(m);
        val.resize(m);
        for (const auto& e : *this) ++rp[size_t(transpose ? e.dst : e.src) + 1];
        for (index_t r = 0; r < n; ++r) rp[r + 1] += rp[r];
        std::vector<offset_t> cur(rp.begin(), rp.end() - 1);
        for (const auto& e : *this) {
            const index_t row = transpose ? e.dst : e.src;
            const offset_t p = cur[row]++;
            ci[p] = transpose ? e.src : e.dst;
            val[p] = e.edata;
        }
    }

    template <arch_t arch, bool transpose = false>
    CsrMat<arch, edata_t, index_t, offset_t, v_start> ToCsr() const {
        std::vector<offset_t> rp;
        std::vector<index_t> ci;
        std::vector<edata_t> val;
        BuildCsr<transpose>(rp, ci, val);
        return CsrMat<arch, edata_t, index_t, offset_t, v_start>(
            num_vertices(), num_vertices(), num_edges(),
            Buffer<arch, offset_t, index_t>(Buffer<arch_t::cpu, offset_t, index_t>(rp)),
            Buffer<arch, index_t, offset_t>(Buffer<arch_t::cpu, index_t, offset_t>(ci)),
            Buffer<arch, edata_t, offset_t>(Buffer<arch_t::cpu, edata_t, offset_t>(val)));
    }

private:
    index_t max_vid_{0};
};

template <vstart_t v_start = vstart_t::FROM_0_TO_0, typename index_t = vid_t,
          typename offset_t = eid_t>
class GraphLoader {
public:
    explicit GraphLoader(bool reorder_vid = false)
        : reorder_vid_(reorder_vid), next_vid_(v_start == vstart_t::FROM_0_TO_0 ? 0 : 1) {}

    template <typename edata_t>
    EdgeCache<v_start, edata_t, index_t, offset_t> LoadEdgesFromTxt(
        const std::string& path, const LoadEdgeOpts& opts = LoadEdgeOpts()) {
        if (!utils::StrEndWith(path, opts.file_ext))
            LOG_ERROR("file extension does not match, it should \"", opts.file_ext, "\"");
        std::ifstream fin(path);
        if (fin.fail()) LOG_ERROR("cannot open graph adj file: ", path);
        EdgeCache<v_start, edata_t, index_t, offset_t> cache;
        std::string line;
        while (std::getline(fin, line)) {
            line = utils::StrStrip(line);
            if (line.empty() || utils::StrStartWith(line, opts.comment_prefix)) continue;
            char* save = nullptr;
            char* tok = strtok_r(line.data(), opts.line_sep.c_str(), &save);
            if (!tok) continue;
            EdgeUnit<edata_t, index_t> e;
            e.src = index_t(std::strtoul(tok, nullptr, 10));
            tok = strtok_r(nullptr, opts.line_sep.c_str(), &save);
            if (!tok) {
                LOG_WARNING("can not extract destination from (", line, ")");
                continue;
            }
            e.dst = index_t(std::strtoul(tok, nullptr, 10));
            tok = strtok_r(nullptr, opts.line_sep.c_str(), &save);
            if constexpr (std::is_integral_v<edata_t>)
                e.edata = tok ? edata_t(std::strtoul(tok, nullptr, 10)) : edata_t(1);
            else
                e.edata = tok ? edata_t(std::strtod(tok, nullptr)) : edata_t(1);
            if (!opts.keep_self_loop && e.src == e.dst) continue;
            if constexpr (v_start == vstart_t::FROM_1_TO_0) {
                if (e.src == 0 || e.dst == 0) {
                    LOG_WARNING("edge with vertex 0 in a 1-based file: (", e.src, ", ", e.dst, ")");
                    continue;
                }
                --e.src;
                --e.dst;
            }
            if (reorder_vid_) {
                e.src = renumber_(e.src);
                e.dst = renumber_(e.dst);
            }
            cache.push_back(e);
            if (!opts.is_directed && e.src != e.dst) cache.push_back({e.dst, e.src, e.edata});
        }
        if (!opts.keep_duplicate_edges) {
            std::stable_sort(cache.begin(), cache.end());
            cache.erase(std::unique(cache.begin(), cache.end()), cache.end());
        }
        return cache;
    }

    // LoadEdgesFromTxt then ToCsr (reference: loader/graph_loader.h:124-129).
    template <arch_t arch, typename edata_t = double>
    CsrMat<arch, edata_t, index_t, offset_t, v_start> LoadCsrFromTxt(const std::string& path,
                                                                     const LoadEdgeOpts& opts = LoadEdgeOpts()) {
        return LoadEdgesFromTxt<edata_t>(path, opts).template ToCsr<arch>();
    }

    // Per-vertex lines "vid data..." (reference: loader/graph_loader.h:131-198):
    // lines starting with the comment prefix are skipped, the id is the first
    // token (renumbered like the edges when reordering is on), and the parser
    // gets either the rest of the line (parse_t = char*) or its tokens parsed
    // as parse_t.  A parser returning false logs a warning.
    template <typename parse_t, typename parse_func>
    void LoadVertexStatusFromTxt(const std::string& path, parse_func&& parser,
                                 const LoadVertexOpts& opts = LoadVertexOpts()) {
        std::ifstream fin(path);
        if (fin.fail()) LOG_ERROR("cannot open graph vertex file: ", path);
        std::string line;
        std::vector<parse_t> splits;
        while (std::getline(fin, line)) {
            if (utils::StrStartWith(line, opts.comment_prefix)) continue;
            char* save = nullptr;
            char* tok = strtok_r(line.data(), opts.vertex_sep.c_str(), &save);
            if (!tok) continue;  // blank line
            index_t vid = index_t(std::strtoul(tok, nullptr, 10));
            if (reorder_vid_) vid = renumber_(vid);
            if constexpr (std::is_same_v<parse_t, char*>) {
                if (!parser(vid, save)) LOG_WARNING("can not decode vertex data of vertex ", vid);
            } else {
                static_assert(std::is_integral_v<parse_t> || std::is_floating_point_v<parse_t>);
                splits.clear();
                for (tok = strtok_r(nullptr, opts.vdata_sep.c_str(), &save); tok;
                     tok = strtok_r(nullptr, opts.vdata_sep.c_str(), &save)) {
                    if constexpr (std::is_integral_v<parse_t>)
                        splits.push_back(parse_t(std::strtoul(tok, nullptr, 10)));
                    else
                        splits.push_back(parse_t(std::strtod(tok, nullptr)));
                }
                if (!parser(vid, splits))
                    LOG_WARNING("can not decode vertex data of vertex ", vid, ": ", utils::VecToString(splits));
            }
        }
    }

    // One value per vertex from "vid value" lines (reference:
    // loader/graph_loader.h:199-223); vertices without a line keep 0.  An id
    // at or beyond num_vertices is skipped with a warning (the reference
    // writes past the end of its vector).
    template <arch_t arch, typename vdata_t>
    DenseVec<arch, vdata_t, index_t> LoadVertexVecFromTxt(const std::string& path, index_t num_vertices,
                                                          const LoadVertexOpts& opts = LoadVertexOpts()) {
        static_assert(std::is_integral_v<vdata_t> || std::is_floating_point_v<vdata_t>);
        DenseVec<arch_t::cpu, vdata_t, index_t> h(num_vertices);
        LoadVertexStatusFromTxt<char*>(
            path,
            [&](index_t vid, char* rest) {
                if (vid >= num_vertices) return false;
                if constexpr (std::is_integral_v<vdata_t>)
                    h[vid] = vdata_t(std::strtoul(rest, nullptr, 10));
                else
                    h[vid] = vdata_t(std::strtod(rest, nullptr));
                return true;
            },
            opts);
        if constexpr (arch == arch_t::cpu)
            return h;
        else
            return h.template to<arch>();
    }

    /// maps an id of the file to its renumbered id; false when it never appeared
    bool ReorderedVid(index_t& vid) const {
        if (!reorder_vid_) return true;
        auto it = vid_map_.find(vid);
        if (it == vid_map_.end()) return false;
        vid = it->second;
        return true;
    }

    const std::unordered_map<index_t, index_t>& get_vid_map() const { return vid_map_; }

private:
    index_t renumber_(index_t v) {
        auto it = vid_map_.find(v);
        if (it != vid_map_.end()) return it->second;
        vid_map_.emplace(v, next_vid_);
        return next_vid_++;
    }

    bool reorder_vid_;
    index_t next_vid_;
    std::unordered_map<index_t, index_t> vid_map_;
};

}  // namespace graph_one
