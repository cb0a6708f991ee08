// Per-particle MLP of the learned PCISPH warm start: 8 features -> 32 -> 32 -> 1, SiLU,
// BF16 operands on the tensor cores with FP32 accumulation. This header holds the training
// side (warp-level mma.sync m16n8k16, whose fragments the backward pass reuses); inference
// runs on tcgen05 (mlp_tc.cuh).
//
// A warp evaluates 32 particles as two 16-row tiles. The accumulator fragment of one
// layer (rows g, g+8; columns 2q, 2q+1 of each 8-column tile; g = lane/4, q = lane%4)
// is exactly the A-operand fragment of the next layer's 16-column k-tile, so hidden
// activations never leave registers. Weights live in shared memory already split into
// per-lane B fragments (MlpPacked), one 32-bit word per lane per register.
//
// Parameter vector (FP32 master copy, 1377 floats):
//   W1[8][32] @0, b1[32] @256, W2[32][32] @288, b2[32] @1312, W3[32] @1344, b3 @1376
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace lsp {

constexpr int kMlpIn = 8;
constexpr int kMlpHidden = 32;
constexpr int kMlpParams = 8 * 32 + 32 + 32 * 32 + 32 + 32 + 1;   // 1377
constexpr int kOffW1 = 0, kOffB1 = 256, kOffW2 = 288, kOffB2 = 1312, kOffW3 = 1344, kOffB3 = 1376;

// Fragment-ordered BF16 weights (bf16x2 words) and FP32 biases.
struct MlpPacked {
    uint32_t l1[4][32];          // layer 1 B fragment b0 per n-tile (b1 is the zero padding of K 8->16)
    uint32_t l2[4][2][2][32];    // layer 2 [n-tile][k-tile][reg]
    uint32_t l3[2][2][32];       // layer 3 [k-tile][reg], output column 0 only
    uint32_t l2t[4][2][2][32];   // W2 transposed, for the backward pass dh1 = dz2 W2^T
    float b1[32], b2[32], w3[32], b3, pad[3];   // w3: BF16-rounded W3 as float (backward)
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// D = A * B + D, A 16x16 bf16 (row), B 16x8 bf16 (col), D 16x8 fp32.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// The network's activations use the hardware approximations (__expf, __fdividef): the
// library is compiled for IEEE-exact division and square roots (the physics needs them),
// which the activations do not, and their error (a few ulp) is far below the BF16
// rounding of every activation. For z < -87, __expf(-z) overflows and the quotient is 0.
__device__ __forceinline__ float sigmoidf(float z) { return __fdividef(1.f, 1.f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigmoidf(z); }
__device__ __forceinline__ float silu_grad(float z)
{
    float s = sigmoidf(z);
    return s * (1.f + z * (1.f - s));
}

// Forward of one 16-particle tile. a1: layer-1 A fragment (features). Returns the output
// of rows g (in y[0]) and g+8 (in y[1]), valid in lanes with q == 0. When keep is set,
// pre-activations z1, z2 (fragment layout) are returned for the backward pass.
template <bool kKeep>
__device__ __forceinline__ void mlp_tile_forward(const MlpPacked& w, const uint32_t (&a1)[4], float (&z1)[4][4],
                                                 float (&z2)[4][4], uint32_t (&h1)[2][4], uint32_t (&h2)[2][4],
                                                 float (&y)[2])
{
    const int lane = threadIdx.x & 31, q = lane & 3;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        float c0 = w.b1[8 * t + 2 * q], c1 = w.b1[8 * t + 2 * q + 1];
        z1[t][0] = c0; z1[t][1] = c1; z1[t][2] = c0; z1[t][3] = c1;
        mma16816(z1[t], a1, w.l1[t][lane], 0u);
    }
#pragma unroll
    for (int k = 0; k < 2; k++) {
        h1[k][0] = pack_bf16(silu(z1[2 * k][0]), silu(z1[2 * k][1]));
        h1[k][1] = pack_bf16(silu(z1[2 * k][2]), silu(z1[2 * k][3]));
        h1[k][2] = pack_bf16(silu(z1[2 * k + 1][0]), silu(z1[2 * k + 1][1]));
        h1[k][3] = pack_bf16(silu(z1[2 * k + 1][2]), silu(z1[2 * k + 1][3]));
    }
#pragma unroll
    for (int t = 0; t < 4; t++) {
        float c0 = w.b2[8 * t + 2 * q], c1 = w.b2[8 * t + 2 * q + 1];
        z2[t][0] = c0; z2[t][1] = c1; z2[t][2] = c0; z2[t][3] = c1;
#pragma unroll
        for (int k = 0; k < 2; k++) mma16816(z2[t], h1[k], w.l2[t][k][0][lane], w.l2[t][k][1][lane]);
    }
#pragma unroll
    for (int k = 0; k < 2; k++) {
        h2[k][0] = pack_bf16(silu(z2[2 * k][0]), silu(z2[2 * k][1]));
        h2[k][1] = pack_bf16(silu(z2[2 * k][2]), silu(z2[2 * k][3]));
        h2[k][2] = pack_bf16(silu(z2[2 * k + 1][0]), silu(z2[2 * k + 1][1]));
        h2[k][3] = pack_bf16(silu(z2[2 * k + 1][2]), silu(z2[2 * k + 1][3]));
    }
    float o[4] = {w.b3, 0.f, w.b3, 0.f};
#pragma unroll
    for (int k = 0; k < 2; k++) mma16816(o, h2[k], w.l3[k][0][lane], w.l3[k][1][lane]);
    y[0] = o[0];
    y[1] = o[2];
}


}  // namespace lsp
