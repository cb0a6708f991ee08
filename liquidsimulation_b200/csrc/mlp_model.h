// The warm-start network's parameters and optimiser on one device stream: FP32 master
// weights with Adam moments, the fragment-ordered BF16 copy the kernels read (MlpPacked),
// and the training / inference / gradient entry points of lsp_mlp_* and lsp_batch_mlp_*.
#pragma once

#include <cstdint>

#include "host_util.h"

namespace lsp {

struct MlpPacked;
struct MlpUmma;

class MlpModel {
public:
    // Allocates on the current device and sets the Xavier weights of seed 0.
    void init(cudaStream_t s);
    // Uniform(-a, a) weights with a = sqrt(6 / (fan_in + fan_out)), zero biases, the output
    // layer scaled down so an untrained network guesses close to zero.
    void reset(uint64_t seed);
    void set(const float* w, int n);
    void get(float* w, int n);
    // Weight of the squared error of over-estimates in training. With a zero negative-
    // pressure factor PCISPH only ever adds pressure, so a guess that is too high cannot be
    // corrected within the step; weighting those errors up biases the guess low.
    void set_over_weight(float w);
    // `iterations` Adam steps, each on `batch` rows drawn at random from the n device rows
    // feat[n][8] with targets tgt[n]; returns the last step's mean loss.
    float train(const float* feat, const float* tgt, int64_t n, int iterations, int batch, float lr, uint64_t seed);
    // Host rows in, host outputs out.
    void forward(const float* feat, int64_t n, float* out);
    // Gradient of 1/(2n) sum (y - t)^2 at the current parameters (host in, host out).
    float gradient(const float* feat, const float* target, int64_t n, float* grad);
    const MlpPacked* packed() const { return reinterpret_cast<const MlpPacked*>(packed_.p); }
    // The weights as tensor-core (tcgen05) operand images, for inference.
    const MlpUmma* umma() const { return reinterpret_cast<const MlpUmma*>(umma_.p); }

private:
    void repack();
    cudaStream_t s_ = nullptr;
    DevArray<float> master_, m1_, m2_, partial_, loss_part_, grad_, loss_, io_;
    DevArray<int32_t> idx_;
    DevArray<uint32_t> packed_, umma_, err_;
    int step_ = 0;
    float over_weight_ = 1.f;
};

}  // namespace lsp
