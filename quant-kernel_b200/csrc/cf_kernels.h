// cf_kernels.h -- host interface of the batch Heston characteristic-function
// pricer (one CTA per option, FP64).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qkb {

// One option record, 112 bytes.  mode 0: integrate; mode 1: the entry checks
// already decided the result, which is const_price (NaN or intrinsic value).
struct alignas(16) CfOption {
    double spot, strike, t, r, q;
    double v0, kappa, theta, sigma, rho;
    double limit;
    double const_price;
    int32_t option_type;
    int32_t panels;  // ceil(integration_steps / 64) Gauss-Legendre panels
    int32_t mode;
    int32_t pad;
};
static_assert(sizeof(CfOption) == 112, "CfOption layout");

// Applies the reference's entry checks (heston.cpp:10-24) and packs a record.
CfOption pack_cf_option(double spot, double strike, double t, double r, double q, double v0,
                        double kappa, double theta, double sigma, double rho, int32_t option_type,
                        int32_t integration_steps, double integration_limit);

// Prices n packed records into d_out (device) on stream st; the Gauss-Legendre
// table is uploaded to the current device on first use.
cudaError_t launch_heston_cf(const CfOption* d_opts, int32_t n, double* d_out, cudaStream_t st);

// Host records in, host prices out: stages through the calling thread's pinned
// and device buffers on its own stream and waits for the result.
cudaError_t heston_cf_price_host(const CfOption* h_opts, int32_t n, double* out);

}  // namespace qkb
