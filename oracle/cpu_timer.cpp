// cpu_timer.cpp -- times a CPU library's batch Heston Monte Carlo entry point
// from C++ (TEST INFRASTRUCTURE: the CPU baseline of the benchmark).
//
//   cpu_timer <library.so> <symbol> <inputs.bin> <reps>
//
// Loads <symbol> with the qk_mcm_heston_monte_carlo_price_batch signature of
// the reference's qk_api.h (spot, strike, t, r, q, v0, kappa, theta, sigma,
// rho, option_type, paths, steps, seed, n, out_prices), reads the batch from
// <inputs.bin> (int32 n, ten float64[n], three int32[n], one uint64[n]), and
// calls it <reps> times, each bracketed by std::chrono::steady_clock.  Prints
// one JSON line: the seconds of every call and the sum of the last call's
// prices.  OpenMP threads come from OMP_NUM_THREADS as for any caller.
#include <dlfcn.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

using BatchFn = int32_t (*)(const double*, const double*, const double*, const double*,
                            const double*, const double*, const double*, const double*,
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
    auto fn = reinterpret_cast<BatchFn>(dlsym(lib, argv[2]));
    if (!fn) {
        std::fprintf(stderr, "dlsym: %s\n", dlerror());
        return 1;
    }
    std::FILE* f = std::fopen(argv[3], "rb");
    if (!f) {
        std::fprintf(stderr, "cannot open %s\n", argv[3]);
        return 1;
    }
    int32_t n = 0;
    std::vector<double> d[10];
    std::vector<int32_t> ot, paths, steps;
    std::vector<uint64_t> seed;
    bool ok = std::fread(&n, sizeof n, 1, f) == 1 && n > 0;
    for (int i = 0; ok && i < 10; ++i) ok = read_array(f, d[i], n);
    ok = ok && read_array(f, ot, n) && read_array(f, paths, n) && read_array(f, steps, n) &&
         read_array(f, seed, n);
    std::fclose(f);
    if (!ok) {
        std::fprintf(stderr, "bad input file %s\n", argv[3]);
        return 1;
    }
    const int reps = std::atoi(argv[4]);
    std::vector<double> out(static_cast<size_t>(n));
    std::printf("{\"seconds\": [");
    for (int r = 0; r < reps; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        const int32_t rc = fn(d[0].data(), d[1].data(), d[2].data(), d[3].data(), d[4].data(),
                              d[5].data(), d[6].data(), d[7].data(), d[8].data(), d[9].data(),
                              ot.data(), paths.data(), steps.data(), seed.data(), n, out.data());
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
