#pragma once
// Device-resident graphs of the GraphOne API (reference: graph/graph.h:18-140,
// graph/graph_arch_ref.h:23-116, graph/graph_view.hpp:10-60,
// graph/builder.h:9-46).
//
// A Graph owns a g1_graph of libgraphone_b200 (CSR arrays padded and
// validated on the device, merge-path plans cached with it).  `views`
// selects the orientations: normal (out-edges), transpose (in-edges), or
// both; the first view listed is the "main" CSR that ToArch() exposes as
// row_offsets/col_indices/values, exactly as in GraphOne (a transpose-only
// graph's main CSR is the transpose).

#include <cstdint>
#include <memory>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "graphone_b200.h"
#include "GraphOne/loader/loader.h"
#include "GraphOne/macros.h"
#include "GraphOne/type.hpp"
#include "GraphOne/utils/log.hpp"
#include "GraphOne/utils/pinned.h"

namespace graph_one {

enum class graph_view_t : uint8_t { normal = 1 << 0, transpose = 1 << 1, coo = 1 << 2, csr = 1 << 3 };

constexpr graph_view_t operator|(graph_view_t a, graph_view_t b) {
    return static_cast<graph_view_t>(static_cast<uint8_t>(a) | static_cast<uint8_t>(b));
}
constexpr bool has_view(graph_view_t v, graph_view_t m) {
    return (static_cast<uint8_t>(v) & static_cast<uint8_t>(m)) == static_cast<uint8_t>(m);
}
template <typename... M>
constexpr bool has_all_views(graph_view_t v, M... m) {
    return (has_view(v, m) && ...);
}
template <typename... M>
constexpr bool has_some_views(graph_view_t v, M... m) {
    return (has_view(v, m) || ...);
}
constexpr graph_view_t set_view(graph_view_t v, graph_view_t m) { return v | m; }
constexpr graph_view_t unset_view(graph_view_t v, graph_view_t m) {
    return static_cast<graph_view_t>(static_cast<uint8_t>(v) & ~static_cast<uint8_t>(m));
}
// Position (1-based) of the highest set bit of N; 0 for N == 0.
template <uint8_t N>
struct highest_bit {
    static constexpr uint8_t value = N == 0 ? 0 : 1 + highest_bit<N / 2>::value;
};
template <>
struct highest_bit<0> {
    static constexpr uint8_t value = 0;
};

template <graph_view_t views, arch_t arch, vstart_t v_start, typename vprop_t, typename vertex_t,
          typename edge_t, typename weight_t>
struct GraphArchRef {
    using vprop_type = vprop_t;
    using vertex_type = vertex_t;
    using edge_type = edge_t;
    using weight_type = weight_t;
    constexpr static arch_t arch_value = arch;
    constexpr static vstart_t vstart_value = v_start;
    constexpr static bool both_mat = has_all_views(views, graph_view_t::normal, graph_view_t::transpose);

    template <graph_view_t V = views, std::enable_if_t<has_view(V, graph_view_t::normal), int> = 0>
    __host__ __device__ vertex_t get_out_degree(vertex_t v) const {
        return row_offsets[v + 1] - row_offsets[v];
    }
    template <graph_view_t V = views, std::enable_if_t<has_view(V, graph_view_t::transpose), int> = 0>
    __host__ __device__ vertex_t get_in_degree(vertex_t v) const {
        if constexpr (both_mat)
            return trans_row_offsets[v + 1] - trans_row_offsets[v];
        else
            return row_offsets[v + 1] - row_offsets[v];
    }
    template <graph_view_t V = views, std::enable_if_t<has_view(V, graph_view_t::normal), int> = 0>
    __host__ __device__ edge_t get_starting_out_edge(vertex_t v) const {
        return row_offsets[v];
    }
    template <graph_view_t V = views, std::enable_if_t<has_view(V, graph_view_t::normal), int> = 0>
    __host__ __device__ vertex_t get_dst_vertex_by_out_edge(edge_t e) const {
        return col_indices[e];
    }
    template <graph_view_t V = views, std::enable_if_t<has_view(V, graph_view_t::normal), int> = 0>
    __host__ __device__ weight_t get_out_edge_weight(edge_t e) const {
        return values[e];
    }

    vertex_t num_vertices{0};
    edge_t num_edges{0};
    const edge_t* row_offsets{nullptr};
    const vertex_t* col_indices{nullptr};
    const weight_t* values{nullptr};
    const edge_t* trans_row_offsets{nullptr};
    const vertex_t* trans_col_indices{nullptr};
    const weight_t* trans_values{nullptr};
    vprop_t vprops{};
};

namespace detail {
struct GraphHandleDeleter {
    void operator()(g1_graph* g) const { g1_graph_destroy(g); }
};
}  // namespace detail

template <arch_t arch, graph_view_t views, vstart_t v_start, typename vprop_t, typename vertex_t,
          typename edge_t, typename weight_t>
class Graph {
public:
    static_assert(arch == arch_t::cuda, "graphs live on the GPU");
    static_assert(has_some_views(views, graph_view_t::normal, graph_view_t::transpose),
                  "a graph needs the normal or the transpose view");
    static_assert(sizeof(vertex_t) == 4 && sizeof(edge_t) == 4, "32-bit vertex and edge ids");
    static_assert(sizeof(weight_t) == 4, "4-byte edge values (u32/i32/f32)");

    using vprop_type = vprop_t;
    using vertex_type = vertex_t;
    using edge_type = edge_t;
    using weight_type = weight_t;
    using arch_ref_t = GraphArchRef<views, arch, v_start, vprop_t, vertex_t, edge_t, weight_t>;
    constexpr static arch_t arch_value = arch;
    constexpr static vstart_t vstart_value = v_start;
    constexpr static graph_view_t views_value = views;
    constexpr static bool has_normal = has_view(views, graph_view_t::normal);
    constexpr static bool has_transpose = has_view(views, graph_view_t::transpose);
    constexpr static bool both_mat = has_normal && has_transpose;

    Graph(g1_graph* handle, vertex_t n, edge_t m)
        : h_(handle, detail::GraphHandleDeleter()), n_(n), m_(m) {}

    using graph_mat_t = CsrMat<arch, weight_t, vertex_t, edge_t, v_start>;
    using graph_tmat_t = std::conditional_t<both_mat, graph_mat_t, empty_t>;

    vertex_t num_vertices() const { return n_; }
    edge_t num_edges() const { return m_; }
    g1_graph* handle() const { return h_.get(); }
    const vprop_t& vprops() const { return vprops_; }

    // Degrees from the device CSR: one 8-byte copy to the host per call, like
    // an element read of a device Buffer (reference: graph/graph.h:62-84).
    template <graph_view_t V = views>
    std::enable_if_t<has_view(V, graph_view_t::normal), vertex_t> get_out_degree(vertex_t vid) const {
        return degree_(0, vid);
    }
    template <graph_view_t V = views>
    std::enable_if_t<has_view(V, graph_view_t::transpose), vertex_t> get_in_degree(vertex_t vid) const {
        return degree_(1, vid);
    }

    // The CSR of the first view (and, with both views, the transpose) as
    // CsrMat.  The library owns the graph's arrays, so these are device
    // copies made on the first call and kept with the graph: same contents
    // as ToArch()'s arrays, other addresses (reference: graph/graph.h:86-92).
    const graph_mat_t& graph_mat() const {
        if (!mats_->mat) mats_->mat.reset(new graph_mat_t(copy_mat_(has_normal ? 0 : 1)));
        return *mats_->mat;
    }
    const graph_tmat_t& graph_transpose_mat() const {
        if constexpr (both_mat) {
            if (!mats_->tmat) mats_->tmat.reset(new graph_mat_t(copy_mat_(1)));
            return *mats_->tmat;
        } else {
            return mats_->none;
        }
    }

    arch_ref_t ToArch() const {
        arch_ref_t r;
        r.num_vertices = n_;
        r.num_edges = m_;
        const int main_side = has_normal ? 0 : 1;
        fetch_(main_side, &r.row_offsets, &r.col_indices, &r.values);
        if constexpr (both_mat) fetch_(1, &r.trans_row_offsets, &r.trans_col_indices, &r.trans_values);
        return r;
    }

    std::string ToString() const {
        return "Graph{ num_vertices:" + utils::NumToString(n_) + ", num_edges:" +
               utils::NumToString(m_) + " }";
    }

private:
    struct Mats {
        std::unique_ptr<graph_mat_t> mat, tmat;
        empty_t none{};
    };

    vertex_t degree_(int side, vertex_t vid) const {
        const edge_t *rp = nullptr;
        const vertex_t* ci = nullptr;
        const weight_t* v = nullptr;
        fetch_(side, &rp, &ci, &v);
        edge_t two[2] = {0, 0};
        ::graph_one::detail::mem_copy<arch_t::cpu, arch_t::cuda>(two, rp + vid, sizeof(two));
        return (vertex_t)(two[1] - two[0]);
    }

    graph_mat_t copy_mat_(int side) const {
        const edge_t *rp = nullptr;
        const vertex_t* ci = nullptr;
        const weight_t* v = nullptr;
        fetch_(side, &rp, &ci, &v);
        Buffer<arch, edge_t, vertex_t> b_rp((vertex_t)(n_ + 1));
        Buffer<arch, vertex_t, edge_t> b_ci(m_);
        Buffer<arch, weight_t, edge_t> b_v(m_);
        ::graph_one::detail::mem_copy<arch, arch>(b_rp.data(), rp, sizeof(edge_t) * ((size_t)n_ + 1));
        ::graph_one::detail::mem_copy<arch, arch>(b_ci.data(), ci, sizeof(vertex_t) * (size_t)m_);
        ::graph_one::detail::mem_copy<arch, arch>(b_v.data(), v, sizeof(weight_t) * (size_t)m_);
        return graph_mat_t(n_, n_, m_, std::move(b_rp), std::move(b_ci), std::move(b_v));
    }

    void fetch_(int side, const edge_t** rp, const vertex_t** ci, const weight_t** v) const {
        const uint32_t *a = nullptr, *b = nullptr;
        const void* c = nullptr;
        if (g1_graph_arrays(h_.get(), side, &a, &b, &c) != G1_OK)
            LOG_ERROR("graph arrays: ", g1_last_error());
        *rp = reinterpret_cast<const edge_t*>(a);
        *ci = reinterpret_cast<const vertex_t*>(b);
        *v = static_cast<const weight_t*>(c);
    }

    std::shared_ptr<g1_graph> h_;
    vertex_t n_;
    edge_t m_;
    vprop_t vprops_{};
    std::shared_ptr<Mats> mats_ = std::make_shared<Mats>();
};

namespace graph {

// graph::build (reference: graph/builder.h:9-46): the host CSR of the first
// needed orientation is made by EdgeCache's counting sort and handed to
// libgraphone_b200, which builds the other orientation on the GPU when the
// views ask for both.
template <arch_t arch, graph_view_t views, vstart_t v_start, typename vertex_t, typename edge_t,
          typename weight_t>
Graph<arch, views, v_start, empty_t, vertex_t, edge_t, weight_t> build(
    EdgeCache<v_start, weight_t, vertex_t, edge_t>& cache) {
    using G = Graph<arch, views, v_start, empty_t, vertex_t, edge_t, weight_t>;
    // The application's own CUDA runtime (its kernels live in its binary)
    // starts here, with the graph, rather than inside the first Run; the
    // library's runtime starts with g1_graph_create below.
    // The engines' pinned read-back block is made here too, for the same reason.
    if constexpr (arch == arch_t::cuda) {
        cudaFree(nullptr);
        (void)::graph_one::detail::PinnedSlots::get();
    }
    std::vector<edge_t> rp;
    std::vector<vertex_t> ci;
    std::vector<weight_t> val;
    uint32_t flags = 0;
    if constexpr (G::has_normal) {
        cache.template BuildCsr<false>(rp, ci, val);
        if constexpr (G::has_transpose) flags |= G1_GRAPH_BUILD_OTHER;
    } else {
        cache.template BuildCsr<true>(rp, ci, val);
        flags |= G1_GRAPH_INPUT_TRANSPOSE;
    }
    const g1_dtype vt = std::is_floating_point_v<weight_t> ? G1_F32 : G1_U32;
    g1_graph* h = nullptr;
    const g1_status s = g1_graph_create(rp.data(), ci.data(), val.data(), vt, cache.num_vertices(),
                                        (uint32_t)cache.num_edges(), flags, nullptr, &h);
    if (s != G1_OK) LOG_ERROR("graph::build: ", g1_status_string(s), ": ", g1_last_error());
    return G(h, cache.num_vertices(), (edge_t)cache.num_edges());
}

}  // namespace graph
}  // namespace graph_one
