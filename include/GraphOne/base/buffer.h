#pragma once
// Host or device arrays of the GraphOne API (reference: base/buffer.h:12-202,
// vec/dense.h:10-42).  Device memory comes from libgraphone_b200
// (g1_mem_alloc zero-fills, like the reference's constructor memset);
// element access from the host copies one element across.

#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <string>
#include <type_traits>
#include <vector>

#include "graphone_b200.h"
#include "GraphOne/type.hpp"
#include "GraphOne/utils/string.hpp"

namespace graph_one {

namespace detail {
[[noreturn]] inline void buffer_fail(g1_status s, const char* what) {
    std::fprintf(stderr, "[ERROR] %s: %s (%s)\n", what, g1_status_string(s), g1_last_error());
    std::exit(1);
}

template <arch_t arch>
inline void* mem_alloc(size_t bytes) {
    if constexpr (arch == arch_t::cpu) {
        void* p = std::calloc(bytes ? bytes : 1, 1);
        if (!p) buffer_fail(G1_ERR_OOM, "host allocation");
        return p;
    } else {
        void* p = nullptr;
        const g1_status s = g1_mem_alloc(&p, bytes);
        if (s != G1_OK) buffer_fail(s, "device allocation");
        return p;
    }
}

template <arch_t arch>
inline void mem_free(void* p) {
    if (!p) return;
    if constexpr (arch == arch_t::cpu)
        std::free(p);
    else
        g1_mem_free(p);
}

// dst (arch_to) <- src (arch_from)
template <arch_t to, arch_t from>
inline void mem_copy(void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    if constexpr (to == arch_t::cpu && from == arch_t::cpu) {
        std::memcpy(dst, src, bytes);
    } else {
        const int kind = (from == arch_t::cpu) ? 0 : (to == arch_t::cpu ? 1 : 2);
        const g1_status s = g1_mem_copy(dst, src, bytes, kind, nullptr);
        if (s != G1_OK) buffer_fail(s, "copy");
        if (kind != 1) g1_stream_sync(nullptr);
    }
}
}  // namespace detail

template <arch_t arch, typename value_t, typename index_t = std::size_t>
class Buffer {
public:
    Buffer() = default;

    explicit Buffer(index_t size) : size_(size), data_(alloc_(size)) {}

    explicit Buffer(const std::vector<value_t>& vec) : size_(vec.size()), data_(alloc_(vec.size())) {
        detail::mem_copy<arch, arch_t::cpu>(data_, vec.data(), sizeof(value_t) * size_);
    }

    Buffer(const Buffer& rhs) : size_(rhs.size_), data_(alloc_(rhs.size_)) {
        detail::mem_copy<arch, arch>(data_, rhs.data_, sizeof(value_t) * size_);
    }

    template <arch_t from>
    Buffer(const Buffer<from, value_t, index_t>& rhs) : size_(rhs.size()), data_(alloc_(rhs.size())) {
        detail::mem_copy<arch, from>(data_, rhs.data(), sizeof(value_t) * size_);
    }

    Buffer(Buffer&& rhs) noexcept : size_(rhs.size_), data_(rhs.data_) {
        rhs.size_ = 0;
        rhs.data_ = nullptr;
    }

    Buffer& operator=(const Buffer& rhs) {
        if (this != &rhs) {
            reset_(rhs.size_);
            detail::mem_copy<arch, arch>(data_, rhs.data_, sizeof(value_t) * size_);
        }
        return *this;
    }

    template <arch_t from>
    Buffer& operator=(const Buffer<from, value_t, index_t>& rhs) {
        reset_(rhs.size());
        detail::mem_copy<arch, from>(data_, rhs.data(), sizeof(value_t) * size_);
        return *this;
    }

    Buffer& operator=(Buffer&& rhs) noexcept {
        if (this != &rhs) {
            detail::mem_free<arch>(data_);
            size_ = rhs.size_;
            data_ = rhs.data_;
            rhs.size_ = 0;
            rhs.data_ = nullptr;
        }
        return *this;
    }

    ~Buffer() { detail::mem_free<arch>(data_); }

    /// copies the host values into [buf_begin, ...) (clamped to the size)
    void copy_from(const std::vector<value_t>& vec, index_t buf_begin = 0) {
        const index_t len = std::min<index_t>(index_t(vec.size()), size_ - buf_begin);
        detail::mem_copy<arch, arch_t::cpu>(data_ + buf_begin, vec.data(), sizeof(value_t) * len);
    }

    template <arch_t from>
    void copy_from(const Buffer<from, value_t, index_t>& src, index_t buf_begin = 0) {
        const index_t len = std::min<index_t>(src.size(), size_ - buf_begin);
        detail::mem_copy<arch, from>(data_ + buf_begin, src.data(), sizeof(value_t) * len);
    }

    std::conditional_t<arch == arch_t::cpu, const value_t&, value_t> operator[](index_t i) const {
        if constexpr (arch == arch_t::cpu)
            return data_[i];
        else
            return get(i);
    }

    std::conditional_t<arch == arch_t::cpu, value_t&, void> operator[](index_t i) {
        if constexpr (arch == arch_t::cpu) return data_[i];
    }

    void set(index_t i, const value_t& v) {
        detail::mem_copy<arch, arch_t::cpu>(data_ + i, &v, sizeof(value_t));
    }

    value_t get(index_t i) const {
        value_t v;
        detail::mem_copy<arch_t::cpu, arch>(&v, data_ + i, sizeof(value_t));
        return v;
    }

    value_t* begin() { return data_; }
    const value_t* begin() const { return data_; }
    value_t* end() { return data_ + size_; }
    const value_t* end() const { return data_ + size_; }
    value_t* data() { return data_; }
    const value_t* data() const { return data_; }
    index_t size() const { return size_; }
    bool empty() const { return size_ == 0; }

    /// zero-fills the current contents
    void resize() { fill_zero_(size_); }

    /// reallocates to `size` elements (when it changes) and zero-fills
    void resize(index_t size) {
        if (size != size_) reset_(size);
        fill_zero_(size_);
    }

    template <arch_t dst_arch>
    Buffer<dst_arch, value_t, index_t> to() const {
        return Buffer<dst_arch, value_t, index_t>(*this);
    }

    std::string ToString() const {
        std::vector<value_t> h(size_);
        detail::mem_copy<arch_t::cpu, arch>(h.data(), data_, sizeof(value_t) * size_);
        std::string s = "Buffer{ size_:" + utils::NumToString(size_) + ", data_:[";
        for (index_t i = 0; i < size_; ++i) s += (i ? "," : "") + utils::ToString(h[i]);
        return s + "] }";
    }

protected:
    static value_t* alloc_(index_t n) {
        return static_cast<value_t*>(detail::mem_alloc<arch>(sizeof(value_t) * size_t(n)));
    }
    void reset_(index_t n) {
        detail::mem_free<arch>(data_);
        data_ = alloc_(n);
        size_ = n;
    }
    void fill_zero_(index_t n) {
        if constexpr (arch == arch_t::cpu) {
            std::memset(static_cast<void*>(data_), 0, sizeof(value_t) * n);
        } else if (n) {
            std::vector<unsigned char> z(sizeof(value_t) * n, 0);
            detail::mem_copy<arch, arch_t::cpu>(data_, z.data(), z.size());
        }
    }

    index_t size_{0};
    value_t* data_{nullptr};
};

template <arch_t arch, typename value_t, typename index_t = uint32_t>
class DenseVec : public Buffer<arch, value_t, index_t> {
public:
    using Buffer<arch, value_t, index_t>::Buffer;
    constexpr static arch_t arch_value = arch;

    DenseVec() = default;
    DenseVec(const Buffer<arch, value_t, index_t>& b) : Buffer<arch, value_t, index_t>(b) {}
    DenseVec(Buffer<arch, value_t, index_t>&& b) : Buffer<arch, value_t, index_t>(std::move(b)) {}

    template <arch_t dst_arch>
    DenseVec<dst_arch, value_t, index_t> to() const {
        return DenseVec<dst_arch, value_t, index_t>(Buffer<dst_arch, value_t, index_t>(*this));
    }
};

}  // namespace graph_one
