// sur_api.cpp -- extern "C" entry points of the Heston surrogate.
#include "../../include/qk_api.h"

#include <cuda_runtime.h>

#include "qk_error.h"
#include "sur_gemm.cuh"

extern "C" {

int32_t qk_sur_gemm_bf16(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k,
                         int32_t splits, void* stream) {
    if (!a) return qkb::fail_null("a");
    if (!b) return qkb::fail_null("b");
    if (!c) return qkb::fail_null("c");
    if (m <= 0 || n <= 0 || k <= 0 || splits <= 0 || k % 64 != 0 || n % 64 != 0 ||
        k % (64 * splits) != 0)
        return qkb::fail_size(m <= 0 ? m : (n <= 0 ? n : k));
    CUtensorMap ta, tb;
    const int bn = (n % 128 == 0) ? 128 : 64;
    if (!qkb::make_tmap_bf16(&ta, a, (uint64_t)m, (uint64_t)k, 128) ||
        !qkb::make_tmap_bf16(&tb, b, (uint64_t)n, (uint64_t)k, (uint32_t)bn))
        return qkb::fail_cuda(cudaErrorInvalidValue, "qk_sur_gemm_bf16 (tensor map)");
    qkb::GemmArgs g = {};
    g.M = m;
    g.N = n;
    g.K = k;
    g.k_per_split = k / splits;
    g.c_f32 = c;
    static int* err_word[64] = {};  // one device error word per GPU
    int dev = 0;
    cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess || dev < 0 || dev >= 64) return qkb::fail_cuda(de, "qk_sur_gemm_bf16");
    if (!err_word[dev]) {
        cudaError_t e = cudaMalloc(&err_word[dev], sizeof(int));
        if (e != cudaSuccess) return qkb::fail_cuda(e, "qk_sur_gemm_bf16");
        cudaMemset(err_word[dev], 0, sizeof(int));
    }
    g.err = err_word[dev];
    cudaError_t e = qkb::launch_umma_gemm(qkb::kEpiF32, bn, ta, tb, g, splits,
                                          static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? QK_OK : qkb::fail_cuda(e, "qk_sur_gemm_bf16");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The surrogate model.
#include <cmath>
#include <limits>
#include <vector>

#include "sur_mlp.h"

struct qk_sur_model {
    qkb::SurModel m;
};

namespace {

int32_t sur_status(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return QK_OK;
    if (e == cudaErrorInvalidValue) {
        qkb::set_error_fmt("invalid argument in %s", where);
        return QK_ERR_INVALID_INPUT;
    }
    return qkb::fail_cuda(e, where);
}

double smax0(double x) { return (0.0 < x) ? x : 0.0; }

}  // namespace

extern "C" {

int32_t qk_sur_heston_create(const double* box_lo, const double* box_hi, uint64_t seed,
                             qk_sur_model** out_model) {
    if (!box_lo) return qkb::fail_null("box_lo");
    if (!box_hi) return qkb::fail_null("box_hi");
    if (!out_model) return qkb::fail_null("out_model");
    *out_model = nullptr;
    qkb::SurBox box;
    for (int i = 0; i < qkb::kSurIn; ++i) {
        if (!(box_hi[i] >= box_lo[i]) || !std::isfinite(box_lo[i]) || !std::isfinite(box_hi[i])) {
            qkb::set_error_fmt("invalid box dimension %d", i);
            return QK_ERR_INVALID_INPUT;
        }
        box.lo[i] = box_lo[i];
        box.hi[i] = box_hi[i];
    }
    qk_sur_model* p = new qk_sur_model();
    cudaError_t e = p->m.init(seed, box);
    if (e != cudaSuccess) {
        delete p;
        return qkb::fail_cuda(e, "qk_sur_heston_create");
    }
    *out_model = p;
    return QK_OK;
}

int32_t qk_sur_heston_destroy(qk_sur_model* model) {
    delete model;
    return QK_OK;
}

int32_t qk_sur_heston_set_dataset(qk_sur_model* model, const double* features,
                                  const double* target, int64_t n) {
    if (!model) return qkb::fail_null("model");
    if (!features) return qkb::fail_null("features");
    if (!target) return qkb::fail_null("target");
    if (n <= 0 || n > std::numeric_limits<int32_t>::max()) return qkb::fail_size(n);
    return sur_status(model->m.set_dataset(features, target, n), "qk_sur_heston_set_dataset");
}

int32_t qk_sur_heston_train(qk_sur_model* model, int32_t epochs, int32_t batch, double lr,
                            uint64_t shuffle_seed, double* out_epoch_loss) {
    if (!model) return qkb::fail_null("model");
    if (epochs <= 0) return qkb::fail_size(epochs);
    if (batch <= 0 || batch % 128 != 0) return qkb::fail_size(batch);
    std::vector<float> el(static_cast<size_t>(epochs));
    float last = 0.0f;
    cudaError_t e = model->m.train(epochs, batch, static_cast<float>(lr), shuffle_seed, &last, el.data());
    if (e == cudaSuccess && model->m.device_error() != 0) {
        qkb::set_error_fmt("tensor-core pipeline timed out (code %d)", model->m.device_error());
        return QK_ERR_RUNTIME_INIT;
    }
    if (e == cudaSuccess && out_epoch_loss)
        for (int i = 0; i < epochs; ++i) out_epoch_loss[i] = el[static_cast<size_t>(i)];
    return sur_status(e, "qk_sur_heston_train");
}

int32_t qk_sur_heston_predict(qk_sur_model* model, const double* features, int64_t n, double* out) {
    if (!model) return qkb::fail_null("model");
    if (!features) return qkb::fail_null("features");
    if (!out) return qkb::fail_null("out");
    if (n <= 0) return qkb::fail_size(n);
    return sur_status(model->m.predict(features, n, out), "qk_sur_heston_predict");
}

int32_t qk_sur_heston_predict_device(qk_sur_model* model, const void* x_rows, const float* base,
                                     int64_t n, float* y, void* stream) {
    if (!model) return qkb::fail_null("model");
    if (!x_rows) return qkb::fail_null("x_rows");
    if (!base && model->m.base_kind() != qkb::kSurBaseNone) return qkb::fail_null("base");
    if (!y) return qkb::fail_null("y");
    if (n <= 0) return qkb::fail_size(n);
    return sur_status(model->m.predict_device(static_cast<const __nv_bfloat16*>(x_rows), base, n, y,
                                              static_cast<cudaStream_t>(stream)),
                      "qk_sur_heston_predict_device");
}

int32_t qk_sur_heston_predict_device_layered(qk_sur_model* model, const void* x_rows,
                                             const float* base, int64_t n, float* y, void* stream) {
    if (!model) return qkb::fail_null("model");
    if (!x_rows) return qkb::fail_null("x_rows");
    if (!base && model->m.base_kind() != qkb::kSurBaseNone) return qkb::fail_null("base");
    if (!y) return qkb::fail_null("y");
    if (n <= 0) return qkb::fail_size(n);
    return sur_status(model->m.predict_device(static_cast<const __nv_bfloat16*>(x_rows), base, n, y,
                                              static_cast<cudaStream_t>(stream), true),
                      "qk_sur_heston_predict_device_layered");
}

int32_t qk_sur_heston_features(qk_sur_model* model, const double* features, int64_t n,
                               void* out_rows, float* out_base) {
    if (!model) return qkb::fail_null("model");
    if (!features) return qkb::fail_null("features");
    if (!out_rows) return qkb::fail_null("out_rows");
    if (n <= 0) return qkb::fail_size(n);
    model->m.normalise(features, n, static_cast<__nv_bfloat16*>(out_rows));
    if (out_base) model->m.base_host(features, n, out_base);
    return QK_OK;
}

int32_t qk_sur_heston_features_device(qk_sur_model* model, const double* features, int64_t n,
                                      void* rows, float* base, void* stream) {
    if (!model) return qkb::fail_null("model");
    if (!features) return qkb::fail_null("features");
    if (!rows) return qkb::fail_null("rows");
    if (!base) return qkb::fail_null("base");
    if (n <= 0) return qkb::fail_size(n);
    return sur_status(model->m.features_device(features, n, static_cast<__nv_bfloat16*>(rows), base,
                                               static_cast<cudaStream_t>(stream)),
                      "qk_sur_heston_features_device");
}

int32_t qk_sur_heston_gradients(qk_sur_model* model, const double* features, const double* target,
                                int32_t n, double* grads, double* loss) {
    if (!model) return qkb::fail_null("model");
    if (!features) return qkb::fail_null("features");
    if (!target) return qkb::fail_null("target");
    if (!grads) return qkb::fail_null("grads");
    if (n <= 0 || n % 128 != 0) return qkb::fail_size(n);
    return sur_status(model->m.gradients(features, target, n, grads, loss), "qk_sur_heston_gradients");
}

int32_t qk_sur_heston_parameters(qk_sur_model* model, double* out) {
    if (!model) return qkb::fail_null("model");
    if (!out) return qkb::fail_null("out");
    return sur_status(model->m.parameters(out), "qk_sur_heston_parameters");
}

int32_t qk_sur_heston_set_parameters(qk_sur_model* model, const double* in) {
    if (!model) return qkb::fail_null("model");
    if (!in) return qkb::fail_null("in");
    return sur_status(model->m.set_parameters(in), "qk_sur_heston_set_parameters");
}

int32_t qk_sur_heston_save(qk_sur_model* model, const char* path) {
    if (!model) return qkb::fail_null("model");
    if (!path) return qkb::fail_null("path");
    return sur_status(model->m.save(path), "qk_sur_heston_save");
}

int32_t qk_sur_heston_load(qk_sur_model* model, const char* path) {
    if (!model) return qkb::fail_null("model");
    if (!path) return qkb::fail_null("path");
    return sur_status(model->m.load(path), "qk_sur_heston_load");
}

int32_t qk_sur_heston_price_batch(qk_sur_model* model, const double* spot, const double* strike,
                                  const double* t, const double* r, const double* q,
                                  const double* v0, const double* kappa, const double* theta,
                                  const double* sigma, const double* rho,
                                  const int32_t* option_type, int32_t n, int32_t fallback_paths,
                                  int32_t fallback_steps, uint64_t fallback_seed,
                                  double* out_prices, int32_t* out_source) {
    if (!model) return qkb::fail_null("model");
    const void* ptrs[] = {spot, strike, t, r, q, v0, kappa, theta, sigma, rho, option_type, out_prices};
    const char* names[] = {"spot", "strike", "t", "r", "q", "v0", "kappa", "theta", "sigma", "rho",
                           "option_type", "out_prices"};
    for (int i = 0; i < 12; ++i)
        if (!ptrs[i]) return qkb::fail_null(names[i]);
    if (n <= 0) return qkb::fail_size(n);
    const double nan = std::numeric_limits<double>::quiet_NaN();
    std::vector<int32_t> sur_idx, mc_idx;
    std::vector<double> feats;
    for (int32_t i = 0; i < n; ++i) {
        const int32_t ot = option_type[i];
        // entry checks of heston_monte_carlo.cpp:18-26
        const bool bad = !(ot == 0 || ot == 1) || spot[i] <= 0.0 || strike[i] <= 0.0 || t[i] < 0.0 ||
                         v0[i] < 0.0 || kappa[i] < 0.0 || theta[i] < 0.0 || sigma[i] < 0.0 ||
                         rho[i] < -1.0 || rho[i] > 1.0;
        if (bad) {
            out_prices[i] = nan;
            if (out_source) out_source[i] = 2;
            continue;
        }
        if (t[i] <= 1e-12) {
            out_prices[i] = ot == 0 ? smax0(spot[i] - strike[i]) : smax0(strike[i] - spot[i]);
            if (out_source) out_source[i] = 2;
            continue;
        }
        const double f[qkb::kSurIn] = {spot[i] / strike[i], t[i], r[i], q[i], v0[i],
                                       kappa[i], theta[i], sigma[i], rho[i]};
        if (model->m.in_box(f)) {
            sur_idx.push_back(i);
            feats.insert(feats.end(), f, f + qkb::kSurIn);
        } else {
            mc_idx.push_back(i);
        }
    }
    if (!sur_idx.empty()) {
        std::vector<double> y(sur_idx.size());
        int32_t rc = sur_status(model->m.predict(feats.data(), static_cast<int64_t>(sur_idx.size()), y.data()),
                                "qk_sur_heston_price_batch");
        if (rc != QK_OK) return rc;
        for (size_t k = 0; k < sur_idx.size(); ++k) {
            const int32_t i = sur_idx[k];
            const double call = spot[i] * y[k];
            out_prices[i] = option_type[i] == 0
                                ? call
                                : call - spot[i] * std::exp(-q[i] * t[i]) + strike[i] * std::exp(-r[i] * t[i]);
            if (out_source) out_source[i] = 0;
        }
    }
    if (!mc_idx.empty()) {
        const size_t m = mc_idx.size();
        std::vector<double> a[10];
        for (auto& v : a) v.resize(m);
        std::vector<int32_t> ot(m), pp(m, fallback_paths), st(m, fallback_steps);
        std::vector<uint64_t> sd(m);
        const double* src[10] = {spot, strike, t, r, q, v0, kappa, theta, sigma, rho};
        for (size_t k = 0; k < m; ++k) {
            const int32_t i = mc_idx[k];
            for (int c = 0; c < 10; ++c) a[c][k] = src[c][i];
            ot[k] = option_type[i];
            sd[k] = fallback_seed + static_cast<uint64_t>(i);
        }
        std::vector<double> out(m);
        int32_t rc = qk_mcm_heston_monte_carlo_price_batch(
            a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(), a[5].data(), a[6].data(),
            a[7].data(), a[8].data(), a[9].data(), ot.data(), pp.data(), st.data(), sd.data(),
            static_cast<int32_t>(m), out.data());
        if (rc != QK_OK) return rc;
        for (size_t k = 0; k < m; ++k) {
            out_prices[mc_idx[k]] = out[k];
            if (out_source) out_source[mc_idx[k]] = 1;
        }
    }
    return QK_OK;
}

}  // extern "C"
