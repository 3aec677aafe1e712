#pragma once
// Sparse-format conversions of the GraphOne API (reference: mat/convert.h:
// 16-88), with thrust on the arrays' own side (host for arch_t::cpu, device
// for arch_t::cuda), as the reference does.
//
//   OffsetsToIndices(offsets, nnz)   the row of each nonzero (offsets of
//                                    n + 1 entries, nnz results);
//   IndicesToOffsets(indices, size)  offsets[i] = first k with indices[k] >= i
//                                    (sorted indices), `size` results;
//   ToCsc(csr)                       the CSC of a CSR: nonzeros stably sorted by
//                                    column, so rows ascend within a column.
//
// Difference from the reference, result-neutral for well-formed input: its
// OffsetsToIndices walks i over [0, nnz - 1) and reads offsets[i + 1], past
// the end of offsets whenever nnz > n + 1; here each nonzero's row is found
// by a binary search over offsets[1..n], and the result has exactly nnz
// entries.

#include <thrust/binary_search.h>
#include <thrust/execution_policy.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/zip_iterator.h>
#include <thrust/sort.h>
#include <thrust/tuple.h>

#include "GraphOne/base/buffer.h"
#include "GraphOne/loader/loader.h"
#include "GraphOne/mat/csc.h"
#include "GraphOne/type.hpp"

namespace graph_one::mat {

namespace detail {
template <arch_t arch>
constexpr auto policy() {
    if constexpr (arch == arch_t::cpu)
        return thrust::host;
    else
        return thrust::device;
}
}  // namespace detail

template <arch_t arch, typename index_t, typename offset_t>
Buffer<arch, index_t, offset_t> OffsetsToIndices(const Buffer<arch, offset_t, index_t>& offsets,
                                                 offset_t indices_size) {
    Buffer<arch, index_t, offset_t> indices(indices_size);
    if (indices_size == 0 || offsets.size() < 2) return indices;
    const offset_t* ends = offsets.data() + 1;  // row r ends at offsets[r + 1]
    thrust::upper_bound(detail::policy<arch>(), ends, ends + (offsets.size() - 1),
                        thrust::counting_iterator<offset_t>(0), thrust::counting_iterator<offset_t>(indices_size),
                        indices.data());
    return indices;
}

template <arch_t arch, typename index_t, typename offset_t>
Buffer<arch, offset_t, index_t> IndicesToOffsets(const Buffer<arch, index_t, offset_t>& indices,
                                                 index_t offsets_size) {
    Buffer<arch, offset_t, index_t> offsets(offsets_size);
    if (offsets_size == 0) return offsets;
    thrust::lower_bound(detail::policy<arch>(), indices.data(), indices.data() + indices.size(),
                        thrust::counting_iterator<index_t>(0), thrust::counting_iterator<index_t>(offsets_size),
                        offsets.data());
    return offsets;
}

template <arch_t arch, typename value_t, typename index_t, typename offset_t, vstart_t v_start>
CscMat<arch, value_t, index_t, offset_t, v_start> ToCsc(const CsrMat<arch, value_t, index_t, offset_t, v_start>& csr) {
    Buffer<arch, index_t, offset_t> row_indices = OffsetsToIndices<arch, index_t, offset_t>(csr.row_offsets, csr.nnz);
    Buffer<arch, index_t, offset_t> col_indices = csr.col_indices;
    Buffer<arch, value_t, offset_t> values = csr.values;
    if (csr.nnz > 0) {
        auto payload = thrust::make_zip_iterator(thrust::make_tuple(row_indices.data(), values.data()));
        thrust::stable_sort_by_key(detail::policy<arch>(), col_indices.data(), col_indices.data() + csr.nnz,
                                   payload);
    }
    Buffer<arch, offset_t, index_t> col_offsets =
        IndicesToOffsets<arch, index_t, offset_t>(col_indices, index_t(csr.n_cols + 1));
    return CscMat<arch, value_t, index_t, offset_t, v_start>(csr.n_rows, csr.n_cols, csr.nnz, std::move(col_offsets),
                                                             std::move(row_indices), std::move(values));
}

}  // namespace graph_one::mat
