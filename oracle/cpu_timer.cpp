// cpu_timer.cpp -- times a CPU library's batch Monte Carlo entry point from C++
// (TEST INFRASTRUCTURE: the CPU baselines of the benchmark).
//
//   cpu_timer <library.so> <symbol> <inputs.bin> <reps>
//
// <inputs.bin> holds one batch: four int32 -- the count of float64 arrays, of
// int32 arrays, of uint64 arrays, and n -- then the arrays in that order, n
// elements each.  The counts select the reference's qk_api.h signature:
//   10 f64, 3 i32, 1 u64  Heston batch (spot, strike, t, r, q, v0, kappa,
//                         theta, sigma, rho, option_type, paths, steps, seed)
//    6 f64, 2 i32, 1 u64  terminal batch (spot, strike, t, vol, r, q,
//                         option_type, paths, seed): standard MC, antithetic
//    6 f64, 3 i32, 1 u64  stepwise batch (spot, strike, t, vol, r, q,
//                         option_type, paths, steps, seed): Euler-Maruyama,
//                         Milstein, local vol
// each followed by (int32 n, double* out_prices).  The call is made <reps>
// times, each bracketed by std::chrono::steady_clock.  Prints one JSON line:
// the seconds of every call and the sum of the last call's prices.  OpenMP
// threads come from OMP_NUM_THREADS as for any caller.
#include <dlfcn.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

using HestonFn = int32_t (*)(const double*, const double*, const double*, const double*,
                             const double*, const double*, const double*, const double*,
                             const double*, const double*, const int32_t*, const int32_t*,
                             const int32_t*, const uint64_t*, int32_t, double*);
using TerminalFn = int32_t (*)(const double*, const double*, const double*, const double*,
                               const double*, const double*, const int32_t*, const int32_t*,
                               const uint64_t*, int32_t, double*);
using StepwiseFn = int32_t (*)(const double*, const double*, const double*, const double*,
                               const double*, const double*, const int32_t*, const int32_t*,
                               const int32_t*, const uint64_t*, int32_t, double*);

template <typename T>
static bool read_array(std::FILE* f, std::vector<T>& v, int32_t n) {
    v.resize(static_cast<size_t>(n));
    return std::fread(v.data(), sizeof(T), v.size(), f) == v.size();
}

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: %s <library.so> <symbol> <inputs.bin> <reps>\n", argv[0]);
        return 2;
    }
    void* lib = dlopen(argv[1], RTLD_NOW | RTLD_LOCAL);
    if (!lib) {
        std::fprintf(stderr, "dlopen: %s\n", dlerror());
        return 1;
    }
    void* sym = dlsym(lib, argv[2]);
    if (!sym) {
        std::fprintf(stderr, "dlsym: %s\n", dlerror());
        return 1;
    }
    std::FILE* f = std::fopen(argv[3], "rb");
    if (!f) {
        std::fprintf(stderr, "cannot open %s\n", argv[3]);
        return 1;
    }
    int32_t head[4] = {0, 0, 0, 0};
    bool ok = std::fread(head, sizeof(int32_t), 4, f) == 4;
    const int32_t nd = head[0], ni = head[1], nu = head[2], n = head[3];
    ok = ok && n > 0 && nu == 1 &&
         ((nd == 10 && ni == 3) || (nd == 6 && ni == 2) || (nd == 6 && ni == 3));
    std::vector<double> d[10];
    std::vector<int32_t> iv[3];
    std::vector<uint64_t> seed;
    for (int i = 0; ok && i < nd; ++i) ok = read_array(f, d[i], n);
    for (int i = 0; ok && i < ni; ++i) ok = read_array(f, iv[i], n);
    ok = ok && read_array(f, seed, n);
    std::fclose(f);
    if (!ok) {
        std::fprintf(stderr, "bad input file %s\n", argv[3]);
        return 1;
    }
    const int reps = std::atoi(argv[4]);
    std::vector<double> out(static_cast<size_t>(n));
    auto call = [&]() -> int32_t {
        if (nd == 10)
            return reinterpret_cast<HestonFn>(sym)(
                d[0].data(), d[1].data(), d[2].data(), d[3].data(), d[4].data(), d[5].data(),
                d[6].data(), d[7].data(), d[8].data(), d[9].data(), iv[0].data(), iv[1].data(),
                iv[2].data(), seed.data(), n, out.data());
        if (ni == 2)
            return reinterpret_cast<TerminalFn>(sym)(d[0].data(), d[1].data(), d[2].data(),
                                                     d[3].data(), d[4].data(), d[5].data(),
                                                     iv[0].data(), iv[1].data(), seed.data(), n,
                                                     out.data());
        return reinterpret_cast<StepwiseFn>(sym)(d[0].data(), d[1].data(), d[2].data(),
                                                 d[3].data(), d[4].data(), d[5].data(),
                                                 iv[0].data(), iv[1].data(), iv[2].data(),
                                                 seed.data(), n, out.data());
    };
    std::printf("{\"seconds\": [");
    for (int r = 0; r < reps; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        const int32_t rc = call();
        const auto t1 = std::chrono::steady_clock::now();
        if (rc != 0) {
            std::fprintf(stderr, "batch call returned %d\n", rc);
            return 1;
        }
        std::printf("%s%.9f", r ? ", " : "", std::chrono::duration<double>(t1 - t0).count());
    }
    double sum = 0.0;
    for (double x : out) sum += x;
    std::printf("], \"price_sum\": %.17g}\n", sum);
    return 0;
}
