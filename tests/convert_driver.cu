// Runs GraphOne's mat::ToCsc and mat::OffsetsToIndices
// (GraphOne/mat/convert.h) on a host CSR read from a file.
//   convert_driver IN OUT
// IN:  u32 n, u32 m, u32 row_ptr[n+1], u32 col[m], u32 val[m]
// OUT: u32 col_offsets[n+1], u32 row_indices[m], u32 values[m],
//      u32 row_of_nonzero[m] (OffsetsToIndices of row_ptr)
#include <cstdio>
#include <vector>

#include "GraphOne/mat/convert.h"

using namespace graph_one;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    uint32_t n = 0, m = 0;
    if (std::fread(&n, 4, 1, f) != 1 || std::fread(&m, 4, 1, f) != 1) return 3;
    std::vector<uint32_t> rp(n + 1), ci(m), v(m);
    if (std::fread(rp.data(), 4, n + 1, f) != n + 1 || std::fread(ci.data(), 4, m, f) != m ||
        std::fread(v.data(), 4, m, f) != m)
        return 3;
    std::fclose(f);
    using csr_t = CsrMat<arch_t::cpu, uint32_t, uint32_t, uint32_t>;
    csr_t csr(n, n, m, Buffer<arch_t::cpu, uint32_t, uint32_t>(rp), Buffer<arch_t::cpu, uint32_t, uint32_t>(ci),
              Buffer<arch_t::cpu, uint32_t, uint32_t>(v));
    auto csc = mat::ToCsc(csr);
    auto rows = mat::OffsetsToIndices<arch_t::cpu, uint32_t, uint32_t>(csr.row_offsets, m);
    if (csc.col_offsets.size() != n + 1 || csc.row_indices.size() != m || csc.values.size() != m ||
        rows.size() != m)
        return 5;
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 4;
    std::fwrite(csc.col_offsets.data(), 4, n + 1, o);
    std::fwrite(csc.row_indices.data(), 4, m, o);
    std::fwrite(csc.values.data(), 4, m, o);
    std::fwrite(rows.data(), 4, m, o);
    std::fclose(o);
    return 0;
}
