// Runs GraphOne's archi:: primitives (GraphOne/archi/archi.cuh) on arrays
// read from a file, on the host (cpu) or the GPU (cuda), and writes the
// results.
//   archi_driver cpu|cuda IN OUT
// IN:  u32 n, then n-entry u32 arrays: keys (distinct), vals, flags (0/1),
//      map (a permutation), sorted (ascending), queries
// OUT: u32 count, then n-entry u32 arrays: copy_if (first count valid),
//      inclusive max-scan, lower_bound, scatter, scatter_if (zeros where not
//      written), keys sorted, vals by key, fill(7), transform(3v+1),
//      2v+5 (cuda: a kernel launched by archi::LaunchKernel), then u64
//      transform_reduce(sum of v*v), u64 for_each sum of v
#include <cstdio>
#include <string>
#include <vector>

#include "GraphOne/archi/archi.cuh"

using namespace graph_one;

// y[i] = 2 x[i] + 5 over a grid-stride loop, launched by archi::LaunchKernel
template <typename tparams>
__global__ void twice_plus5(const uint32_t* x, uint32_t* y, uint32_t n) {
    for (uint32_t i = tparams::global_tid(); i < n; i += tparams::grid_threads()) y[i] = 2u * x[i] + 5u;
}

template <arch_t A>
static int run(const std::vector<std::vector<uint32_t>>& in, FILE* o) {
    const size_t n = in[0].size();
    auto up = [&](const std::vector<uint32_t>& h) {
        uint32_t* p = archi::memalloc<A, uint32_t>(n);
        archi::memcpy<A, arch_t::cpu, uint32_t>(p, h.data(), n);
        return p;
    };
    auto down = [&](const uint32_t* p) {
        std::vector<uint32_t> h(n);
        archi::memcpy<arch_t::cpu, A, uint32_t>(h.data(), p, n);
        return h;
    };
    uint32_t *keys = up(in[0]), *vals = up(in[1]), *flags = up(in[2]), *map = up(in[3]), *sorted = up(in[4]),
             *queries = up(in[5]);
    uint32_t* out = archi::memalloc<A, uint32_t>(n);
    std::vector<std::vector<uint32_t>> res;
    // copy_if with a stencil
    uint32_t* end = archi::copy_if<A>(vals, vals + n, flags, out,
                                      [] __host__ __device__(uint32_t f) { return f != 0; });
    const uint32_t count = (uint32_t)(end - out);
    res.push_back(down(out));
    archi::inclusive_scan<A>(vals, vals + n, out, [] __host__ __device__(uint32_t a, uint32_t b) { return a > b ? a : b; });
    res.push_back(down(out));
    archi::lower_bound<A>(sorted, sorted + n, queries, queries + n, out);
    res.push_back(down(out));
    archi::scatter<A>(vals, vals + n, map, out);
    res.push_back(down(out));
    archi::memset<A, uint32_t>(out, 0, n);
    archi::scatter_if<A>(vals, vals + n, map, flags, out);
    res.push_back(down(out));
    archi::sort_by_key<A>(keys, keys + n, vals);
    res.push_back(down(keys));
    res.push_back(down(vals));
    archi::memcpy<A, arch_t::cpu, uint32_t>(vals, in[1].data(), n);  // restore vals
    archi::fill<A>(out, out + n, 7u);
    res.push_back(down(out));
    archi::transform<A>(vals, vals + n, out, [] __host__ __device__(uint32_t v) { return 3u * v + 1u; });
    res.push_back(down(out));
    const unsigned long long sq = archi::transform_reduce<A>(
        vals, vals + n, [] __host__ __device__(uint32_t v) { return (unsigned long long)v * v; }, 0ull,
        [] __host__ __device__(unsigned long long a, unsigned long long b) { return a + b; });
    unsigned long long* acc = archi::memalloc<A, unsigned long long>(1);
    archi::memset<A, unsigned long long>(acc, 0, 1);
    archi::for_each<A>(vals, vals + n, [acc] __host__ __device__(uint32_t v) {
#ifdef __CUDA_ARCH__
        atomicAdd(acc, (unsigned long long)v);
#else
        *acc += v;
#endif
    });
    unsigned long long each = 0;
    archi::memcpy<arch_t::cpu, A, unsigned long long>(&each, acc, 1);
    if constexpr (A == arch_t::cuda) {
        using tp = archi::LaunchTparams<arch_t::cuda>;
        auto kernel = twice_plus5<tp>;
        checkArchErrors(A, (archi::LaunchKernel<A, empty_t>({(int64_t)n}, kernel, vals, out, (uint32_t)n)));
        checkArchErrors(A, archi::LaunchSync<A>());
        res.push_back(down(out));
    } else {
        std::vector<uint32_t> h(n);
        for (size_t i = 0; i < n; ++i) h[i] = 2u * in[1][i] + 5u;
        res.push_back(h);
    }
    std::fwrite(&count, 4, 1, o);
    for (auto& r : res) std::fwrite(r.data(), 4, n, o);
    std::fwrite(&sq, 8, 1, o);
    std::fwrite(&each, 8, 1, o);
    for (uint32_t* p : {keys, vals, flags, map, sorted, queries, out}) archi::memfree<A, uint32_t>(p);
    archi::memfree<A, unsigned long long>(acc);
    return 0;
}

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) return 3;
    uint32_t n = 0;
    if (std::fread(&n, 4, 1, f) != 1) return 3;
    std::vector<std::vector<uint32_t>> in(6, std::vector<uint32_t>(n));
    for (auto& a : in)
        if (n && std::fread(a.data(), 4, n, f) != n) return 3;
    std::fclose(f);
    FILE* o = std::fopen(argv[3], "wb");
    if (!o) return 4;
    const std::string kind = argv[1];
    const int rc = kind == "cpu" ? run<arch_t::cpu>(in, o) : kind == "cuda" ? run<arch_t::cuda>(in, o) : 2;
    std::fclose(o);
    return rc;
}
