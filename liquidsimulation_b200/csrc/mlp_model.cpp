// Warm-start network state and optimiser (mlp_model.h) over the kernels of mlp.cu.
#include "mlp_model.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "lsp_kernels.h"
#include "mlp.cuh"
#include "mlp_tc.cuh"

namespace lsp {

#define CK(call) LSP_CK(call)

void MlpModel::init(cudaStream_t s)
{
    s_ = s;
    master_.alloc(kMlpParams);
    m1_.alloc(kMlpParams);
    m2_.alloc(kMlpParams);
    grad_.alloc(kMlpParams);
    loss_.alloc(1);
    packed_.alloc(sizeof(MlpPacked) / 4);
    umma_.alloc(sizeof(MlpUmma) / 4);
    err_.alloc(1);
    CK(cudaMemsetAsync(err_.p, 0, sizeof(uint32_t), s_));
    reset(0);
}

void MlpModel::repack()
{
    launch_mlp_pack(master_.p, reinterpret_cast<MlpPacked*>(packed_.p), s_);
    launch_mlp_pack_umma(master_.p, reinterpret_cast<MlpUmma*>(umma_.p), s_);
    CK(cudaGetLastError());
}

void MlpModel::reset(uint64_t seed)
{
    std::vector<float> w(kMlpParams, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fin, int fout, float scale) {
        std::uniform_real_distribution<float> u(-1.f, 1.f);
        float a = scale * std::sqrt(6.f / (float)(fin + fout));
        for (int i = 0; i < fin * fout; i++) w[off + i] = a * u(rng);
    };
    fill(kOffW1, kMlpIn, kMlpHidden, 1.f);
    fill(kOffW2, kMlpHidden, kMlpHidden, 1.f);
    fill(kOffW3, kMlpHidden, 1, 0.1f);
    set(w.data(), kMlpParams);
}

void MlpModel::set(const float* w, int n)
{
    if (!w || n != kMlpParams) throw Error(LSP_ERR_INVALID, "MLP parameter vector must hold 1377 floats");
    CK(cudaMemcpyAsync(master_.p, w, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, s_));
    CK(cudaMemsetAsync(m1_.p, 0, kMlpParams * sizeof(float), s_));
    CK(cudaMemsetAsync(m2_.p, 0, kMlpParams * sizeof(float), s_));
    step_ = 0;
    repack();
    CK(cudaStreamSynchronize(s_));
}

void MlpModel::get(float* w, int n)
{
    if (!w || n != kMlpParams) throw Error(LSP_ERR_INVALID, "MLP parameter vector must hold 1377 floats");
    CK(cudaMemcpyAsync(w, master_.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
}

void MlpModel::set_over_weight(float w)
{
    if (!(w >= 1.f) || !std::isfinite(w)) throw Error(LSP_ERR_INVALID, "loss asymmetry must be >= 1");
    over_weight_ = w;
}

float MlpModel::train(const float* feat, const float* tgt, int64_t n, int iterations, int batch, float lr,
                      uint64_t seed)
{
    if (iterations <= 0 || batch <= 0) throw Error(LSP_ERR_INVALID, "iterations and batch must be > 0");
    batch = (int)std::min<int64_t>(batch, n);
    const int rows = mlp_grad_rows(batch);
    if (partial_.n < (size_t)rows * kMlpParams) partial_.alloc((size_t)rows * kMlpParams);
    if (loss_part_.n < (size_t)rows) loss_part_.alloc(rows);
    if (idx_.n < (size_t)batch) idx_.alloc(batch);
    for (int it = 0; it < iterations; it++) {
        launch_random_indices(idx_.p, batch, (int)n, seed * 1000003ull + (uint64_t)it, s_);
        launch_mlp_grad(packed(), feat, tgt, idx_.p, batch, over_weight_, partial_.p, loss_part_.p, s_);
        step_++;
        launch_mlp_adam(partial_.p, loss_part_.p, rows, master_.p, m1_.p, m2_.p, nullptr, loss_.p, lr, step_, 1, s_);
        repack();
    }
    CK(cudaGetLastError());
    float loss = 0.f;
    CK(cudaMemcpyAsync(&loss, loss_.p, sizeof(float), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    return loss / (float)batch;
}

void MlpModel::forward(const float* feat, int64_t n, float* out)
{
    if (!feat || !out || n <= 0 || n > (1 << 26)) throw Error(LSP_ERR_INVALID, "mlp_forward: bad arguments");
    if (io_.n < (size_t)n * (kMlpIn + 2)) io_.alloc((size_t)n * (kMlpIn + 2));
    float* df = io_.p;
    float* dout = df + n * kMlpIn;
    CK(cudaMemcpyAsync(df, feat, n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s_));
    launch_mlp_forward_tc(umma(), df, dout, (int)n, err_.p, s_);
    CK(cudaGetLastError());
    uint32_t err = 0;
    CK(cudaMemcpyAsync(out, dout, n * sizeof(float), cudaMemcpyDeviceToHost, s_));
    CK(cudaMemcpyAsync(&err, err_.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    if (err) {
        CK(cudaMemsetAsync(err_.p, 0, sizeof(uint32_t), s_));
        throw Error(LSP_ERR_TIMEOUT, "mlp_forward: a tensor-core accumulator wait gave up");
    }
}

float MlpModel::gradient(const float* feat, const float* target, int64_t n, float* grad)
{
    if (!feat || !target || !grad || n <= 0 || n > (1 << 26)) throw Error(LSP_ERR_INVALID, "mlp_gradient: bad arguments");
    if (io_.n < (size_t)n * (kMlpIn + 2)) io_.alloc((size_t)n * (kMlpIn + 2));
    float* df = io_.p;
    float* dt = df + n * kMlpIn;
    CK(cudaMemcpyAsync(df, feat, n * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, s_));
    CK(cudaMemcpyAsync(dt, target, n * sizeof(float), cudaMemcpyHostToDevice, s_));
    const int rows = mlp_grad_rows((int)n);
    if (partial_.n < (size_t)rows * kMlpParams) partial_.alloc((size_t)rows * kMlpParams);
    if (loss_part_.n < (size_t)rows) loss_part_.alloc(rows);
    launch_mlp_grad(packed(), df, dt, nullptr, (int)n, 1.f, partial_.p, loss_part_.p, s_);
    launch_mlp_adam(partial_.p, loss_part_.p, rows, master_.p, m1_.p, m2_.p, grad_.p, loss_.p, 0.f, 1, 0, s_);
    CK(cudaGetLastError());
    float loss = 0.f;
    CK(cudaMemcpyAsync(grad, grad_.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, s_));
    CK(cudaMemcpyAsync(&loss, loss_.p, sizeof(float), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    return loss / (float)n;
}

}  // namespace lsp
