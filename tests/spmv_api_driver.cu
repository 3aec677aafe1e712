// Runs GraphOne's SpMV operator API (GraphOne/archi/blas/spmv/spmv.h) with
// three functors on a CSR read from a file and writes the results.
//   spmv_api_driver KIND IN OUT      KIND: cpu | vector | merge
// IN:  u32 n, u32 m, u32 row_ptr[n+1], u32 col[m], i32 wi[m], f32 wf[m],
//      i32 xi[n], f32 xf[n]
// OUT: i32 y_minplus[n] (the shortest-path functor of GraphOne's
//      test/spmv_test.cu: INT_MAX-guarded add, min), f32 y_plustimes[n],
//      i32 y_default[n] (blas::DefaultSpmvFunctor: sum of min(a, x))
// cpu runs on host arrays; vector and merge copy the inputs to the GPU.
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "GraphOne/archi/blas/spmv/spmv.h"

using namespace graph_one;

struct MinPlusInt {
    __ONE_ARCH_INL__ static int initialize() { return INT_MAX; }
    __ONE_ARCH_INL__ static int combine(const int& w, const int& x) { return x == INT_MAX ? x : w + x; }
    __ONE_ARCH_INL__ static int reduce(const int& a, const int& b) { return a < b ? a : b; }
};

struct PlusTimesFloat {
    __ONE_ARCH_INL__ static float initialize() { return 0.0f; }
    __ONE_ARCH_INL__ static float combine(const float& w, const float& x) { return w * x; }
    __ONE_ARCH_INL__ static float reduce(const float& a, const float& b) { return a + b; }
};

using DefaultInt = blas::DefaultSpmvFunctor<int, int, int>;

template <class T>
static bool read_n(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

template <class T>
static T* to_device(const std::vector<T>& h) {
    T* d = nullptr;
    cudaMalloc(&d, std::max<size_t>(1, h.size()) * sizeof(T));
    if (!h.empty()) cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

template <class Kind, class F, class W, class X, class Y>
static void run_gpu(uint32_t n, uint32_t m, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                    const std::vector<W>& w, const std::vector<X>& x, std::vector<Y>& y) {
    uint32_t* d_rp = to_device(rp);
    uint32_t* d_ci = to_device(ci);
    W* d_w = to_device(w);
    X* d_x = to_device(x);
    Y* d_y = nullptr;
    cudaMalloc(&d_y, std::max<size_t>(1, n) * sizeof(Y));
    {
        auto spmv = blas::MakeCsrSpMV<arch_t::cuda, Kind, F>(n, n, m, (const uint32_t*)d_rp, (const uint32_t*)d_ci,
                                                             (const W*)d_w, (const X*)d_x, d_y);
        spmv();
        spmv();  // a second call on the same plan gives the same result
    }
    y.resize(n);
    if (n) cudaMemcpy(y.data(), d_y, n * sizeof(Y), cudaMemcpyDeviceToHost);
    cudaFree(d_rp);
    cudaFree(d_ci);
    cudaFree(d_w);
    cudaFree(d_x);
    cudaFree(d_y);
}

template <class F, class W, class X, class Y>
static void run_cpu(uint32_t n, uint32_t m, const std::vector<uint32_t>& rp, const std::vector<uint32_t>& ci,
                    const std::vector<W>& w, const std::vector<X>& x, std::vector<Y>& y) {
    y.assign(n, Y{});
    auto spmv = blas::MakeCsrSpMV<arch_t::cpu, blas::SpmvCpuNaive, F>(n, n, m, rp.data(), ci.data(), w.data(),
                                                                      x.data(), y.data());
    spmv();
}

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    const std::string kind = argv[1];
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) return 3;
    uint32_t n = 0, m = 0;
    if (std::fread(&n, 4, 1, f) != 1 || std::fread(&m, 4, 1, f) != 1) return 3;
    std::vector<uint32_t> rp, ci;
    std::vector<int> wi, xi;
    std::vector<float> wf, xf;
    if (!read_n(f, rp, (size_t)n + 1) || !read_n(f, ci, m) || !read_n(f, wi, m) || !read_n(f, wf, m) ||
        !read_n(f, xi, n) || !read_n(f, xf, n))
        return 3;
    std::fclose(f);
    std::vector<int> y1, y3;
    std::vector<float> y2;
    if (kind == "cpu") {
        run_cpu<MinPlusInt>(n, m, rp, ci, wi, xi, y1);
        run_cpu<PlusTimesFloat>(n, m, rp, ci, wf, xf, y2);
        run_cpu<DefaultInt>(n, m, rp, ci, wi, xi, y3);
    } else if (kind == "vector") {
        run_gpu<blas::SpmvCudaCsrVector, MinPlusInt>(n, m, rp, ci, wi, xi, y1);
        run_gpu<blas::SpmvCudaCsrVector, PlusTimesFloat>(n, m, rp, ci, wf, xf, y2);
        run_gpu<blas::SpmvCudaCsrVector, DefaultInt>(n, m, rp, ci, wi, xi, y3);
    } else if (kind == "merge") {
        run_gpu<blas::SpmvCudaCsrMergeBased, MinPlusInt>(n, m, rp, ci, wi, xi, y1);
        run_gpu<blas::SpmvCudaCsrMergeBased, PlusTimesFloat>(n, m, rp, ci, wf, xf, y2);
        run_gpu<blas::SpmvCudaCsrMergeBased, DefaultInt>(n, m, rp, ci, wi, xi, y3);
    } else {
        return 2;
    }
    FILE* o = std::fopen(argv[3], "wb");
    if (!o) return 4;
    std::fwrite(y1.data(), 4, n, o);
    std::fwrite(y2.data(), 4, n, o);
    std::fwrite(y3.data(), 4, n, o);
    std::fclose(o);
    return 0;
}
