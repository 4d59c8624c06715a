// cf_kernels.h -- host interface of the batch Heston Fourier pricers: the
// characteristic-function price with Gauss-Legendre P1/P2 integration and the
// Fang-Oosterlee COS expansion (one CTA per option, FP64).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qkb {

enum : int32_t { kCfMethodGl = 0, kCfMethodCos = 1 };

// One option record, 128 bytes.  mode 0: integrate; mode 1: the entry checks
// already decided the result, which is const_price (NaN or intrinsic value).
struct alignas(16) CfOption {
    double spot, strike, t, r, q;
    double v0, kappa, theta, sigma, rho;
    double limit;        // GL: integration limit; COS: lower end a of [a, b]
    double const_price;
    double hi;           // COS: upper end b
    double pad;
    int32_t option_type;
    int32_t panels;      // GL: ceil(integration_steps / 64) panels; COS: n_terms
    int32_t mode;
    int32_t method;      // kCfMethodGl or kCfMethodCos (one method per batch)
};
static_assert(sizeof(CfOption) == 128, "CfOption layout");

// Applies the reference's entry checks (heston.cpp:10-24) and packs a record.
CfOption pack_cf_option(double spot, double strike, double t, double r, double q, double v0,
                        double kappa, double theta, double sigma, double rho, int32_t option_type,
                        int32_t integration_steps, double integration_limit);

// Applies the reference's entry checks (cos_method.cpp:38-53) and packs a
// COS record with its truncation interval.
CfOption pack_cos_option(double spot, double strike, double t, double r, double q, double v0,
                         double kappa, double theta, double sigma, double rho, int32_t option_type,
                         int32_t n_terms, double truncation_width);

// Prices n packed records into d_out (device) on stream st; the Gauss-Legendre
// table is uploaded to the current device on first use.
cudaError_t launch_heston_cf(const CfOption* d_opts, int32_t n, double* d_out, cudaStream_t st);
cudaError_t launch_heston_cos(const CfOption* d_opts, int32_t n, double* d_out, cudaStream_t st);

// Host records in (all of one method), host prices out: stages through the
// calling thread's pinned and device buffers on its own stream and waits for
// the result.
cudaError_t heston_cf_price_host(const CfOption* h_opts, int32_t n, double* out);

}  // namespace qkb
