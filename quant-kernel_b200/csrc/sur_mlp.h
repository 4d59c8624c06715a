// sur_mlp.h -- the Heston price surrogate: MLP 9 -> 256 -> 256 -> 256 -> 1,
// SiLU, BF16 weights/activations, FP32 accumulation, FP32 master weights and
// Adam moments, trained and evaluated on the GPU with the tcgen05 GEMM.
//
// The network learns a residual: price / S = base(f) + MLP(normalised f),
// with base the Black-Scholes call / S at the Heston model's mean variance
// over [0, T] (see sur_base).  The base carries the bulk of the price
// surface, so the network's absolute error shrinks with the residual's scale.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace qkb {

constexpr int kSurIn = 9;        // S/K, T, r, q, v0, kappa, theta, sigma, rho
constexpr int kSurInPad = 64;    // layer-1 K, zero-padded for the 64-wide k-block
constexpr int kSurHid = 256;
// Base of the residual (stored in checkpoints).
enum : int32_t { kSurBaseNone = 0, kSurBaseBsmMeanVar = 1 };

constexpr int kSurParams = kSurHid * kSurIn + kSurHid + 2 * (kSurHid * kSurHid + kSurHid) +
                           kSurHid + 1;  // 134,401 trainable values

// Internal flat layout of the FP32 master copy (W1 keeps its zero padding).
struct SurLayout {
    static constexpr int W1 = 0;
    static constexpr int b1 = W1 + kSurHid * kSurInPad;
    static constexpr int W2 = b1 + kSurHid;
    static constexpr int b2 = W2 + kSurHid * kSurHid;
    static constexpr int W3 = b2 + kSurHid;
    static constexpr int b3 = W3 + kSurHid * kSurHid;
    static constexpr int w4 = b3 + kSurHid;
    static constexpr int b4 = w4 + kSurHid;
    static constexpr int total = b4 + 4;  // padded to 16 bytes
};

// Training state read by the kernels of a captured step (graph replays see
// the current values).
struct SurState {
    int step;          // completed optimiser steps
    int total_steps;   // cosine schedule length
    int steps_per_epoch;
    int batch;
    float lr0, beta1, beta2, eps;
    int err;           // GEMM error word
    int step_begin;    // first step of the current schedule
    int pad[2];
};

struct SurBox {
    double lo[kSurIn];
    double hi[kSurIn];
};

class SurModel {
public:
    SurModel() = default;
    ~SurModel();
    SurModel(const SurModel&) = delete;
    SurModel& operator=(const SurModel&) = delete;

    cudaError_t init(uint64_t seed, const SurBox& box);
    // Raw features (n x 9, the order of kSurIn) -> normalised bf16 rows.
    void normalise(const double* features, int64_t n, __nv_bfloat16* out_rows) const;
    // The residual's base (price / S, FP64 rounded to FP32) for each row; 0
    // for a model without one.
    void base_host(const double* features, int64_t n, float* out_base) const;
    // Device features (n x 9 FP64, DEVICE) -> normalised rows and base (DEVICE),
    // the same values as normalise and base_host, asynchronous on st.
    cudaError_t features_device(const double* features, int64_t n, __nv_bfloat16* rows,
                                float* base, cudaStream_t st);
    int32_t base_kind() const { return base_kind_; }
    bool in_box(const double* f) const;

    cudaError_t set_dataset(const double* features, const double* target, int64_t n);
    cudaError_t train(int epochs, int batch, float lr0, uint64_t shuffle_seed, float* out_loss_last,
                      float* out_epoch_loss);
    // price / spot of calls for raw features, host in and out.
    cudaError_t predict(const double* features, int64_t n, double* out);
    // Device-resident inference on normalised bf16 rows [n][64] plus the
    // rows' base (required when base_kind() != kSurBaseNone): the fused kernel
    // (all three layers per 128-row tile in one persistent launch), or with
    // layered = true the layer-by-layer GEMMs it is tested against.
    cudaError_t predict_device(const __nv_bfloat16* x_rows, const float* base, int64_t n, float* y,
                               cudaStream_t st, bool layered = false);
    // One forward + backward without an update: loss and the 134,401 gradients.
    cudaError_t gradients(const double* features, const double* target, int n, double* grads,
                          double* loss);
    cudaError_t parameters(double* out) const;            // canonical order, 134,401
    cudaError_t set_parameters(const double* in);
    cudaError_t save(const char* path);
    cudaError_t load(const char* path);
    const SurBox& box() const { return box_; }
    int device() const { return device_; }
    int steps_done() const;
    int device_error();

private:
    cudaError_t ensure_batch_buffers(int batch);
    cudaError_t ensure_predict_buffers(int64_t rows);
    cudaError_t run_step(cudaStream_t st, bool update);
    cudaError_t refresh_bf16(cudaStream_t st);

    int device_ = -1;
    cudaStream_t stream_ = nullptr;
    // the training step's side branches (loss and bias sums with the dW3
    // GEMM; the dW2 GEMM with db2) run on these beside the backward chain,
    // forked and joined by events (inside the captured step graph too)
    cudaStream_t aux_[2] = {nullptr, nullptr};
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    SurBox box_{};
    int32_t base_kind_ = kSurBaseBsmMeanVar;
    // parameters, Adam moments, gradient
    float* P_ = nullptr;
    float* M_ = nullptr;
    float* V_ = nullptr;
    float* G_ = nullptr;
    __nv_bfloat16 *W1b_ = nullptr, *W2b_ = nullptr, *W3b_ = nullptr, *W2Tb_ = nullptr, *W3Tb_ = nullptr;
    SurState* state_ = nullptr;  // device
    // dataset
    __nv_bfloat16* Xall_ = nullptr;
    float* Tall_ = nullptr;
    int32_t* perm_ = nullptr;
    int64_t n_data_ = 0;
    // training batch buffers
    int batch_ = 0;
    __nv_bfloat16 *Xb_ = nullptr, *XTb_ = nullptr;
    float* Tb_ = nullptr;
    __nv_bfloat16 *Z1_ = nullptr, *H1_ = nullptr, *H1T_ = nullptr;
    __nv_bfloat16 *Z2_ = nullptr, *H2_ = nullptr, *H2T_ = nullptr;
    __nv_bfloat16 *dZ3_ = nullptr, *dZ3T_ = nullptr, *H3T_ = nullptr;
    __nv_bfloat16 *dZ2_ = nullptr, *dZ2T_ = nullptr, *dZ1_ = nullptr, *dZ1T_ = nullptr;
    float *y_ = nullptr, *dy_ = nullptr;
    float *dW1p_ = nullptr, *dW2p_ = nullptr, *dW3p_ = nullptr;
    float *db1_ = nullptr, *db2_ = nullptr, *db3_ = nullptr, *dw4_ = nullptr, *db4_ = nullptr;
    float* loss_hist_ = nullptr;
    int loss_cap_ = 0;
    cudaGraphExec_t step_graph_ = nullptr;
    // inference buffers
    int64_t pred_rows_ = 0;
    int sm_count_ = 0;
    __nv_bfloat16 *PX_ = nullptr, *PH1_ = nullptr, *PH2_ = nullptr;
    float* Py_ = nullptr;
    float* Pbase_ = nullptr;
};

}  // namespace qkb
