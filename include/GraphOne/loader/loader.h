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
#include <sstream>
#include <string>
#include <thread>
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

namespace loader_detail {

// Host threads for reading edge files: G1_LOADER_THREADS when set (>= 1),
// else the hardware's, at most 64.
inline size_t loader_threads() {
    if (const char* e = std::getenv("G1_LOADER_THREADS")) {
        const long v = std::strtol(e, nullptr, 10);
        if (v >= 1) return (size_t)std::min<long>(v, 64);
    }
    const unsigned hw = std::thread::hardware_concurrency();
    return std::max<size_t>(1, std::min<size_t>(hw ? hw : 1, 64));
}

// f(0) .. f(parts - 1), each on its own thread (part 0 on the caller's).
template <typename F>
void run_parts(size_t parts, F&& f) {
    std::vector<std::thread> th;
    th.reserve(parts > 0 ? parts - 1 : 0);
    for (size_t p = 1; p < parts; ++p) th.emplace_back([&f, p] { f(p); });
    if (parts > 0) f(0);
    for (auto& t : th) t.join();
}

// A stable sort in `parts` sorted runs (one thread each), then rounds of
// pairwise merges (std::merge keeps the first run's element first among
// equals): the same order as one std::stable_sort.
template <typename T>
void parallel_stable_sort(std::vector<T>& v, size_t parts) {
    constexpr size_t kMinRun = size_t(1) << 16;
    parts = std::max<size_t>(1, std::min(parts, v.size() / kMinRun));
    if (parts <= 1) {
        std::stable_sort(v.begin(), v.end());
        return;
    }
    std::vector<size_t> b(parts + 1);
    for (size_t i = 0; i <= parts; ++i) b[i] = v.size() * i / parts;
    run_parts(parts, [&](size_t p) { std::stable_sort(v.begin() + b[p], v.begin() + b[p + 1]); });
    std::vector<T> tmp(v.size());
    while (b.size() > 2) {
        const size_t runs = b.size() - 1, pairs = (runs + 1) / 2;
        std::vector<size_t> nb(pairs + 1);
        for (size_t q = 0; q < pairs; ++q) nb[q] = b[2 * q];
        nb[pairs] = b[runs];
        run_parts(pairs, [&](size_t q) {
            const size_t lo = b[2 * q], mid = b[std::min(2 * q + 1, runs)], hi = b[std::min(2 * q + 2, runs)];
            std::merge(v.begin() + lo, v.begin() + mid, v.begin() + mid, v.begin() + hi, tmp.begin() + lo);
        });
        v.swap(tmp);
        b.swap(nb);
    }
}

}  // namespace loader_detail

template <vstart_t v_start, typename edata_t, typename index_t, typename offset_t>
class EdgeCache : public std::vector<EdgeUnit<edata_t, index_t>> {
    using base_t = std::vector<EdgeUnit<edata_t, index_t>>;

public:
    void push_back(const EdgeUnit<edata_t, index_t>& e) {
        base_t::push_back(e);
        max_vid_ = std::max(max_vid_, std::max(e.src, e.dst));
    }
    // Takes in the largest id of the edges placed without push_back.
    void update_max_vid() {
        for (const auto& e : *this) max_vid_ = std::max(max_vid_, std::max(e.src, e.dst));
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

    // Reads an edge list (reference: loader/graph_loader.h:32-122, 255-296):
    // one edge "src dst [weight]" per line, tokens split at any of
    // opts.line_sep, a missing weight read as 1, comment and blank lines
    // skipped, self loops dropped unless kept, ids renumbered in first-seen
    // order when asked, the reverse edge added for undirected input, and
    // duplicates merged (the first in file order keeps its weight) unless kept.
    //
    // The file is read once and split at line ends into one part per host
    // thread (about 1 MiB or more each); the threads parse their lines, the
    // warnings are printed afterwards in file order, the first-seen
    // renumbering runs over the edges in file order, and the merge of
    // duplicates sorts in parallel stable runs.  The result is the same as
    // reading the lines one by one.
    template <typename edata_t>
    EdgeCache<v_start, edata_t, index_t, offset_t> LoadEdgesFromTxt(
        const std::string& path, const LoadEdgeOpts& opts = LoadEdgeOpts()) {
        using unit_t = EdgeUnit<edata_t, index_t>;
        if (!utils::StrEndWith(path, opts.file_ext))
            LOG_ERROR("file extension does not match, it should \"", opts.file_ext, "\"");
        std::ifstream fin(path, std::ios::binary);
        if (fin.fail()) LOG_ERROR("cannot open graph adj file: ", path);
        fin.seekg(0, std::ios::end);
        const std::streamoff len = fin.tellg();
        fin.seekg(0, std::ios::beg);
        std::string text(len > 0 ? size_t(len) : size_t(0), '\0');
        if (len > 0) fin.read(&text[0], len);
        text.resize(size_t(std::max<std::streamoff>(0, fin.gcount())));
        const size_t size = text.size();
        constexpr size_t kMinPartBytes = size_t(1) << 20;
        const size_t threads = loader_detail::loader_threads();
        size_t parts = std::max<size_t>(1, std::min(threads, size / kMinPartBytes));
        // part p covers [cut[p], cut[p + 1]), each cut just after a line end
        std::vector<size_t> cut(parts + 1, size);
        cut[0] = 0;
        for (size_t p = 1; p < parts; ++p) {
            size_t c = std::max(cut[p - 1], size * p / parts);
            const void* nl = c < size ? std::memchr(text.data() + c, '\n', size - c) : nullptr;
            cut[p] = nl ? size_t(static_cast<const char*>(nl) - text.data()) + 1 : size;
        }
        std::vector<std::vector<unit_t>> edges(parts);
        std::vector<std::vector<std::string>> warnings(parts);
        loader_detail::run_parts(parts, [&](size_t p) {
            size_t pos = cut[p];
            const size_t end = cut[p + 1];
            std::string line;
            while (pos < end) {
                const void* nl = std::memchr(text.data() + pos, '\n', end - pos);
                const size_t stop = nl ? size_t(static_cast<const char*>(nl) - text.data()) : end;
                line.assign(text.data() + pos, stop - pos);
                pos = nl ? stop + 1 : end;
                parse_edge_line<edata_t>(line, opts, edges[p], warnings[p]);
            }
        });
        for (auto& w : warnings)
            for (auto& msg : w) LOG_WARNING(msg);
        EdgeCache<v_start, edata_t, index_t, offset_t> cache;
        size_t total = 0;
        for (auto& e : edges) total += e.size();
        cache.reserve(total);
        for (auto& e : edges) {
            cache.insert(cache.end(), e.begin(), e.end());
            std::vector<unit_t>().swap(e);
        }
        if (reorder_vid_) {
            // first-seen order over the edges in file order (a reverse edge
            // follows its edge and names no new vertex)
            for (auto& e : cache) {
                e.src = renumber_(e.src);
                e.dst = renumber_(e.dst);
            }
        }
        cache.update_max_vid();
        if (!opts.keep_duplicate_edges) {
            loader_detail::parallel_stable_sort(cache, threads);
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
    // One line of an edge list (everything but the renumbering): appends the
    // edge, and its reverse for undirected input, or a warning.
    template <typename edata_t>
    static void parse_edge_line(std::string& line, const LoadEdgeOpts& opts,
                                std::vector<EdgeUnit<edata_t, index_t>>& out,
                                std::vector<std::string>& warnings) {
        // utils::StrStrip's trim (" \t\n\r"), in place in the reused buffer
        const auto first = line.find_first_not_of(" \t\n\r");
        if (first == std::string::npos) return;
        line.erase(line.find_last_not_of(" \t\n\r") + 1);
        line.erase(0, first);
        if (utils::StrStartWith(line, opts.comment_prefix)) return;
        char* save = nullptr;
        char* tok = strtok_r(line.data(), opts.line_sep.c_str(), &save);
        if (!tok) return;
        EdgeUnit<edata_t, index_t> e;
        e.src = index_t(std::strtoul(tok, nullptr, 10));
        tok = strtok_r(nullptr, opts.line_sep.c_str(), &save);
        if (!tok) {
            warnings.push_back("can not extract destination from (" + line + ")");
            return;
        }
        e.dst = index_t(std::strtoul(tok, nullptr, 10));
        tok = strtok_r(nullptr, opts.line_sep.c_str(), &save);
        if constexpr (std::is_integral_v<edata_t>)
            e.edata = tok ? edata_t(std::strtoul(tok, nullptr, 10)) : edata_t(1);
        else
            e.edata = tok ? edata_t(std::strtod(tok, nullptr)) : edata_t(1);
        if (!opts.keep_self_loop && e.src == e.dst) return;
        if constexpr (v_start == vstart_t::FROM_1_TO_0) {
            if (e.src == 0 || e.dst == 0) {
                std::ostringstream os;
                os << "edge with vertex 0 in a 1-based file: (" << e.src << ", " << e.dst << ")";
                warnings.push_back(os.str());
                return;
            }
            --e.src;
            --e.dst;
        }
        out.push_back(e);
        if (!opts.is_directed && e.src != e.dst) out.push_back({e.dst, e.src, e.edata});
    }

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
