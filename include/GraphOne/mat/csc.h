#pragma once
// Column-compressed matrices of the GraphOne API (reference: mat/csc.h:9-58):
// col_offsets (n_cols + 1), row_indices and values (nnz each).

#include <cstdint>
#include <string>
#include <utility>

#include "GraphOne/base/buffer.h"
#include "GraphOne/type.hpp"
#include "GraphOne/utils/string.hpp"

namespace graph_one {

template <arch_t arch, typename value_t, typename index_t = uint32_t, typename offset_t = uint64_t,
          vstart_t v_start = vstart_t::FROM_0_TO_0>
struct CscMat {
    constexpr static arch_t arch_value = arch;
    constexpr static vstart_t vstart_value = v_start;
    using value_type = value_t;
    using index_type = index_t;
    using offset_type = offset_t;

    CscMat() = default;
    CscMat(index_t rows, index_t cols, offset_t nz, Buffer<arch, offset_t, index_t>&& co,
           Buffer<arch, index_t, offset_t>&& ri, Buffer<arch, value_t, offset_t>&& v)
        : n_rows(rows), n_cols(cols), nnz(nz), col_offsets(std::move(co)), row_indices(std::move(ri)),
          values(std::move(v)) {}
    CscMat(index_t rows, index_t cols, offset_t nz, const Buffer<arch, offset_t, index_t>& co,
           const Buffer<arch, index_t, offset_t>& ri, const Buffer<arch, value_t, offset_t>& v)
        : n_rows(rows), n_cols(cols), nnz(nz), col_offsets(co), row_indices(ri), values(v) {}

    std::string ToString() const {
        return "CscMat{ arch_value:" + utils::ToString(arch_value) + ", n_rows:" + utils::NumToString(n_rows) +
               ", n_cols:" + utils::NumToString(n_cols) + ", nnz:" + utils::NumToString(nnz) +
               ", col_offsets:" + col_offsets.ToString() + ", row_indices:" + row_indices.ToString() +
               ", values:" + values.ToString() + " }";
    }

    index_t n_rows{0};
    index_t n_cols{0};
    offset_t nnz{0};
    Buffer<arch, offset_t, index_t> col_offsets;
    Buffer<arch, index_t, offset_t> row_indices;
    Buffer<arch, value_t, offset_t> values;
};

}  // namespace graph_one
