// The warm-start network's inference on the 5th-generation tensor cores (tcgen05): a CTA of
// 128 threads evaluates 128 particles per tile. The two hidden layers are single-CTA UMMAs
// (M = 128 rows, N = 32, BF16 operands in shared memory, FP32 accumulators in tensor
// memory); one thread issues them and a tcgen05.commit signals an mbarrier. Each warp then
// reads its 32 rows of the accumulator (tcgen05.ld 32x32b: thread t of warp w holds row
// 32 w + t, all 32 columns), adds the bias, applies SiLU, rounds to BF16 and writes its row
// as the next layer's A operand. The 32 -> 1 output layer is 32 FMAs per thread.
//
// Operands use the K-major, no-swizzle canonical layout of the UMMA shared-memory
// descriptor: 8-row x 16-byte core matrices, element (row, k) at byte
//   (row / 8) * SBO + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,
// so LBO (next 8 k) = 128 B and SBO (next 8 rows) = K * 16 B.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lsp_kernels.h"
#include "mlp.cuh"

namespace lsp {

constexpr int kTcRows = 128;          // particles per tile = threads per CTA
constexpr int kTcCols = 64;           // tensor-memory columns: layer 1 at 0, layer 2 at 32
constexpr uint32_t kTcSpinLimit = 1u << 24;
constexpr int kTcSmemPad = 16 * 1024;   // dynamic shared memory requested only to cap blocks per SM

// Weights as UMMA B operands (W^T, K-major image) plus the FP32 epilogue constants.
struct MlpUmma {
    uint16_t w1t[32 * 16];   // W1^T [32 outputs][16] (8 inputs, zero padded), SBO 256
    uint16_t w2t[32 * 32];   // W2^T [32][32], SBO 512
    float b1[32], b2[32];
    float w3[32];            // BF16-rounded W3
    float b3, pad[3];
};

__host__ __device__ constexpr int umma_kmajor_offset(int row, int k, int sbo)
{
    return (row >> 3) * sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// FP32 master parameters -> MlpUmma (one block).
void launch_mlp_pack_umma(const float* master, MlpUmma* out, cudaStream_t s);

// out[i] = network(features[i]) for i < n (features [n][8]).
void launch_mlp_forward_tc(const MlpUmma* w, const float* feat, float* out, int n, uint32_t* err, cudaStream_t s);

// Learned warm start after iteration 0's density pass (which stored the features, rho* and
// the plain first correction): each particle's pressure becomes the network's guess
// p = y * delta * 0.01 * rho0 and x*.w = p / rho*^2. A wait that gives up raises
// kErrTimeout in the status.
void launch_warm_guess_tc(const MlpUmma* w, const DevParams& P, const StepBuffers& b, const float* feat,
                          cudaStream_t s);
struct BatchItem;
// warm_scene (may be null: every scene): items of scenes with a zero flag keep the plain
// first correction.
void launch_batch_warm_guess_tc(const MlpUmma* w, const DevParams* sp, const BatchItem* items, int items_count,
                                const StepBuffers& b, const float* feat, const int32_t* warm_scene, DevStatus* st,
                                cudaStream_t s);

}  // namespace lsp
