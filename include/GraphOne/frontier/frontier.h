#pragma once
// Frontiers of the GraphOne API (reference: frontier/base.h:7-35,
// frontier/sparse_dbl.h:18-181, frontier/dense_dbl.h:17-67,
// frontier/all_active.h:15-49).  Vertex lists live on the device; sizes are
// kept on the host (the engines read the new size back once per iteration).

#include <algorithm>
#include <cstdint>
#include <initializer_list>
#include <string>
#include <vector>

#include "GraphOne/base/buffer.h"
#include "GraphOne/macros.h"
#include "GraphOne/type.hpp"
#include "GraphOne/utils/string.hpp"

namespace graph_one {

enum FrontierKind : uint8_t {
    SPARSE_BASED = 1 << 1,
    DENSE_BASED = 1 << 2,
    ALL_ACTIVE = (1 << 1) | (1 << 2)
};

constexpr FrontierKind operator|(FrontierKind a, FrontierKind b) {
    return static_cast<FrontierKind>(static_cast<uint8_t>(a) | static_cast<uint8_t>(b));
}

constexpr bool check_frontier(FrontierKind target, FrontierKind base) {
    return (static_cast<uint8_t>(target) & static_cast<uint8_t>(base)) == static_cast<uint8_t>(base);
}

template <FrontierKind kind_, bool has_output_>
struct BaseFrontier {
    constexpr static FrontierKind kind = kind_;
    constexpr static bool has_output = has_output_;
    virtual ~BaseFrontier() = default;
    virtual void BeforeEngine() {}
    virtual void AfterEngine() {}
    virtual bool IsConvergent() = 0;
};

// Two device vertex lists (input, output) swapped after every iteration.
template <arch_t arch, typename vertex_t, typename index_t = vertex_t>
class SpDblFrontier : public BaseFrontier<SPARSE_BASED, true> {
public:
    using vertex_type = vertex_t;
    using index_type = index_t;

    struct arch_ref_t {
        constexpr static bool has_output = true;
        using vertex_type = vertex_t;
        using index_type = index_t;
        __device__ __forceinline__ vertex_t get(index_t i) const { return frontiers[input_selector][i]; }
        __device__ __forceinline__ void set(index_t i, vertex_t v) { frontiers[input_selector ^ 1][i] = v; }
        __device__ __forceinline__ const vertex_t* input() const { return frontiers[input_selector]; }
        __device__ __forceinline__ vertex_t* ouput() { return frontiers[input_selector ^ 1]; }
        int input_selector;
        index_t input_size;
        index_t output_size;
        vertex_t* frontiers[2];
    };

    SpDblFrontier(index_t size, std::initializer_list<vertex_t> vids) {
        const index_t sz = index_t(vids.size());
        const index_t cap = std::max(size, sz);
        frontiers_[0] = Buffer<arch, vertex_t, index_t>(std::max<index_t>(cap, 1));
        frontiers_[1] = Buffer<arch, vertex_t, index_t>(std::max<index_t>(cap, 1));
        frontiers_[0].copy_from(std::vector<vertex_t>(vids));
        in_size_ = sz;
    }

    void reserve_input(index_t size) { grow_(input_selector_, size); }
    void reserve_output(index_t size) { grow_(input_selector_ ^ 1, size); }
    void reset_input(index_t size) {
        grow_(input_selector_, size);
        in_size_ = size;
    }
    void reset_output(index_t size) {
        grow_(input_selector_ ^ 1, size);
        out_size_ = size;
    }
    index_t input_size() const { return in_size_; }
    index_t output_size() const { return out_size_; }
    void swap_inout() {
        input_selector_ ^= 1;
        std::swap(in_size_, out_size_);
    }
    const Buffer<arch, vertex_t, index_t>& input() const { return frontiers_[input_selector_]; }
    Buffer<arch, vertex_t, index_t>& input() { return frontiers_[input_selector_]; }
    Buffer<arch, vertex_t, index_t>& output() { return frontiers_[input_selector_ ^ 1]; }

    arch_ref_t ToArch() {
        arch_ref_t r;
        r.input_selector = input_selector_;
        r.input_size = in_size_;
        r.output_size = out_size_;
        r.frontiers[0] = frontiers_[0].data();
        r.frontiers[1] = frontiers_[1].data();
        return r;
    }

    std::string ToString() const {
        return "SpDblFrontier{ input_selector_:" + utils::NumToString(input_selector_) +
               ", in_size_:" + utils::NumToString(in_size_) +
               ", out_size_:" + utils::NumToString(out_size_) + " }";
    }

    void AfterEngine() override { swap_inout(); }
    bool IsConvergent() override { return in_size_ == 0; }

private:
    // Grows a list to at least `size` entries, keeping its contents.
    void grow_(int which, index_t size) {
        if (size <= frontiers_[which].size()) return;
        Buffer<arch, vertex_t, index_t> bigger(size * 2);
        bigger.copy_from(frontiers_[which]);
        frontiers_[which] = std::move(bigger);
    }

    int input_selector_{0};
    index_t in_size_{0};
    index_t out_size_{0};
    Buffer<arch, vertex_t, index_t> frontiers_[2];
};

// Host-side counts only: the BLAS engine keeps the active set in its
// dense vectors; init_buf holds the seed vertices until the first iteration.
template <arch_t arch, typename vertex_t, typename index_t = vertex_t>
class DenDblFrontier : public BaseFrontier<DENSE_BASED, true> {
public:
    using vertex_type = vertex_t;
    using index_type = index_t;

    DenDblFrontier(index_t size, std::initializer_list<vertex_t> vids)
        : in_size_(index_t(vids.size())), init_buf_(index_t(vids.size())) {
        (void)size;
        init_buf_.copy_from(std::vector<vertex_t>(vids));
    }

    index_t input_size() const { return in_size_; }
    index_t& output_size() { return out_size_; }
    void swap_inout() { std::swap(in_size_, out_size_); }
    Buffer<arch, vertex_t, index_t>& init_buf() { return init_buf_; }

    std::string ToString() const {
        return "DenDblFrontier{ in_size_:" + utils::NumToString(in_size_) +
               ", out_size_:" + utils::NumToString(out_size_) + " }";
    }

    void AfterEngine() override { swap_inout(); }
    bool IsConvergent() override { return in_size_ == 0; }

protected:
    index_t in_size_{0};
    index_t out_size_{0};
    Buffer<arch, vertex_t, index_t> init_buf_;
};

// Every vertex is active in every iteration; never converges by itself.
template <arch_t arch, typename vertex_t, typename index_t = vertex_t>
class AllActiveFrontier : public BaseFrontier<ALL_ACTIVE, false> {
public:
    using vertex_type = vertex_t;
    using index_type = index_t;
    AllActiveFrontier(index_t size, std::initializer_list<vertex_t>) : size_(size) {}
    index_t input_size() const { return size_; }
    index_t output_size() const { return size_; }
    index_t size() const { return size_; }
    bool IsConvergent() override { return false; }
    std::string ToString() const {
        return "AllActiveFrontier{ size_: " + utils::NumToString(size_) + " }";
    }

protected:
    index_t size_;
};

// The name the GraphOne README uses for the double-buffered sparse frontier.
template <arch_t arch, typename vertex_t, typename index_t = vertex_t>
using DblBufFrontier = SpDblFrontier<arch, vertex_t, index_t>;

}  // namespace graph_one
