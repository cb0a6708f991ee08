// Training and inference kernels of the warm-start MLP (see mlp.cuh for the layout).
//
//   k_mlp_pack   FP32 master parameters -> BF16 fragment-ordered weights + FP32 biases
//   k_mlp_grad   forward + backward on the tensor cores for a batch, MSE loss; the data
//                gradients use the register-resident fragments, the weight gradients
//                (reductions over particles) are MMAs whose operands are the transposed
//                activation tiles read back from shared memory. Each warp writes its own
//                partial gradient row, so the reduction order is fixed.
//   k_mlp_adam   sums the warp partials in order and applies Adam to the FP32 master.
#include "mlp.cuh"
#include "lsp_kernels.h"

namespace lsp {

constexpr int kMlpThreads = 256;
constexpr int kMlpWarps = kMlpThreads / 32;

__device__ __forceinline__ float bf16_to_float(uint16_t b)
{
    return __uint_as_float(((uint32_t)b) << 16);
}
__device__ __forceinline__ uint32_t pack_bits(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

__global__ void k_mlp_pack(const float* __restrict__ m, MlpPacked* __restrict__ out)
{
    const float* W1 = m + kOffW1;
    const float* W2 = m + kOffW2;
    const float* W3 = m + kOffW3;
    for (int idx = threadIdx.x; idx < 32 * 4; idx += blockDim.x) {
        const int t = idx / 32, lane = idx % 32, g = lane >> 2, q = lane & 3;
        out->l1[t][lane] = pack_bf16(W1[(2 * q) * 32 + 8 * t + g], W1[(2 * q + 1) * 32 + 8 * t + g]);
    }
    for (int idx = threadIdx.x; idx < 4 * 2 * 2 * 32; idx += blockDim.x) {
        const int lane = idx % 32, r = (idx / 32) % 2, k = (idx / 64) % 2, t = idx / 128;
        const int g = lane >> 2, q = lane & 3;
        const int kk = 16 * k + 8 * r + 2 * q, n = 8 * t + g;
        out->l2[t][k][r][lane] = pack_bf16(W2[kk * 32 + n], W2[(kk + 1) * 32 + n]);
        // W2 transposed: B'[k = m][n = c] = W2[c][m].
        out->l2t[t][k][r][lane] = pack_bf16(W2[n * 32 + kk], W2[n * 32 + kk + 1]);
    }
    for (int idx = threadIdx.x; idx < 2 * 2 * 32; idx += blockDim.x) {
        const int lane = idx % 32, r = (idx / 32) % 2, k = idx / 64;
        const int g = lane >> 2, q = lane & 3;
        const int kk = 16 * k + 8 * r + 2 * q;
        out->l3[k][r][lane] = g == 0 ? pack_bf16(W3[kk], W3[kk + 1]) : 0u;
    }
    for (int c = threadIdx.x; c < 32; c += blockDim.x) {
        out->b1[c] = m[kOffB1 + c];
        out->b2[c] = m[kOffB2 + c];
        out->w3[c] = bf16_round(W3[c]);
    }
    if (threadIdx.x == 0) {
        out->b3 = m[kOffB3];
        out->pad[0] = out->pad[1] = out->pad[2] = 0.f;
    }
}

__device__ __forceinline__ void load_packed(MlpPacked& s, const MlpPacked* g)
{
    const uint32_t* src = reinterpret_cast<const uint32_t*>(g);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&s);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 4); i += blockDim.x) dst[i] = src[i];
}

// Reads the bf16 element (row, col) of a row-major 16 x 32 tile stored as bf16x2 words.
__device__ __forceinline__ uint16_t tile_el(const uint32_t* t, int row, int col)
{
    uint32_t w = t[row * 16 + (col >> 1)];
    return (col & 1) ? (uint16_t)(w >> 16) : (uint16_t)(w & 0xffffu);
}
// Features tile (16 rows x 8 features) from the per-lane staging words.
__device__ __forceinline__ uint16_t feat_el(const uint32_t* stage, int tile, int row, int f)
{
    uint32_t w = stage[(16 * tile + row) * 4 + (f >> 1)];
    return (f & 1) ? (uint16_t)(w >> 16) : (uint16_t)(w & 0xffffu);
}

// Stores the D-layout fragments of a 16 x 32 activation tile as bf16 words, row-major.
__device__ __forceinline__ void store_tile(uint32_t* t, const uint32_t (&h)[2][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        t[g * 16 + 8 * k + q] = h[k][0];
        t[(g + 8) * 16 + 8 * k + q] = h[k][1];
        t[g * 16 + 8 * k + 4 + q] = h[k][2];
        t[(g + 8) * 16 + 8 * k + 4 + q] = h[k][3];
    }
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_grad(const MlpPacked* __restrict__ wg,
                                                         const float* __restrict__ feat,
                                                         const float* __restrict__ target,
                                                         const int32_t* __restrict__ idx, int nb, float inv_batch,
                                                         float over_w, float* __restrict__ partial,
                                                         float* __restrict__ loss_partial)
{
    __shared__ MlpPacked w;
    __shared__ uint32_t stage[kMlpWarps][32 * 4];
    __shared__ uint32_t th1[kMlpWarps][16 * 16], tdz2[kMlpWarps][16 * 16], tdz1[kMlpWarps][16 * 16];
    load_packed(w, wg);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const int gw = blockIdx.x * kMlpWarps + warp;
    const int nwarps = gridDim.x * kMlpWarps;

    float dW2[2][4][4] = {}, dW1[4][4] = {};
    float dW3[4][2] = {}, db2[4][2] = {}, db1[4][2] = {};
    float db3 = 0.f, loss = 0.f;

    for (int base = gw * 32; base < nb; base += nwarps * 32) {
        const int bi = base + lane;
        const bool valid = bi < nb;
        const int i = valid ? (idx ? idx[bi] : bi) : 0;
        float f[kMlpIn];
#pragma unroll
        for (int c = 0; c < kMlpIn; c++) f[c] = valid ? feat[(int64_t)i * kMlpIn + c] : 0.f;
        const float tgt = valid ? target[i] : 0.f;
        uint32_t* st = stage[warp];
#pragma unroll
        for (int p = 0; p < 4; p++) st[lane * 4 + p] = pack_bf16(f[2 * p], f[2 * p + 1]);
        __syncwarp();
#pragma unroll
        for (int m = 0; m < 2; m++) {
            uint32_t a1[4] = {st[(16 * m + g) * 4 + q], st[(16 * m + g + 8) * 4 + q], 0u, 0u};
            float z1[4][4], z2[4][4], y[2];
            uint32_t h1[2][4], h2[2][4];
            mlp_tile_forward<true>(w, a1, z1, z2, h1, h2, y);
            // Output gradient of rows g and g+8 (valid in lanes q == 0), then broadcast.
            const float t0 = __shfl_sync(0xffffffffu, tgt, 16 * m + g);
            const float t1 = __shfl_sync(0xffffffffu, tgt, 16 * m + g + 8);
            const bool v0 = base + 16 * m + g < nb, v1 = base + 16 * m + g + 8 < nb;
            // Loss 1/(2n) sum w(r) r^2 with r = y - t, w = over_w when the guess is too high.
            const float r0 = y[0] - t0, r1 = y[1] - t1;
            const float w0 = r0 > 0.f ? over_w : 1.f, w1 = r1 > 0.f ? over_w : 1.f;
            float dy0 = v0 ? w0 * r0 * inv_batch : 0.f;
            float dy1 = v1 ? w1 * r1 * inv_batch : 0.f;
            if (q == 0) {
                loss += (v0 ? 0.5f * w0 * r0 * r0 : 0.f) + (v1 ? 0.5f * w1 * r1 * r1 : 0.f);
                db3 += dy0 + dy1;
            }
            dy0 = __shfl_sync(0xffffffffu, dy0, 4 * g);
            dy1 = __shfl_sync(0xffffffffu, dy1, 4 * g);
            // Layer 3: dW3[c] += sum_rows h2[row][c] dy[row]; dz2 = dy W3 silu'(z2).
            float dz2[4][4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const uint32_t r0 = h2[t >> 1][(t & 1) * 2], r1 = h2[t >> 1][(t & 1) * 2 + 1];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int c = 8 * t + 2 * q + j;
                    const float hr0 = bf16_to_float(j ? (uint16_t)(r0 >> 16) : (uint16_t)(r0 & 0xffffu));
                    const float hr1 = bf16_to_float(j ? (uint16_t)(r1 >> 16) : (uint16_t)(r1 & 0xffffu));
                    dW3[t][j] += hr0 * dy0 + hr1 * dy1;
                    dz2[t][j] = dy0 * w.w3[c] * silu_grad(z2[t][j]);
                    dz2[t][2 + j] = dy1 * w.w3[c] * silu_grad(z2[t][2 + j]);
                    db2[t][j] += dz2[t][j] + dz2[t][2 + j];
                }
            }
            uint32_t dz2p[2][4];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                dz2p[k][0] = pack_bf16(dz2[2 * k][0], dz2[2 * k][1]);
                dz2p[k][1] = pack_bf16(dz2[2 * k][2], dz2[2 * k][3]);
                dz2p[k][2] = pack_bf16(dz2[2 * k + 1][0], dz2[2 * k + 1][1]);
                dz2p[k][3] = pack_bf16(dz2[2 * k + 1][2], dz2[2 * k + 1][3]);
            }
            // Layer 2 data gradient: dh1 = dz2 W2^T, dz1 = dh1 silu'(z1).
            float dz1[4][4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < 2; k++) mma16816(acc, dz2p[k], w.l2t[t][k][0][lane], w.l2t[t][k][1][lane]);
#pragma unroll
                for (int e = 0; e < 4; e++) dz1[t][e] = acc[e] * silu_grad(z1[t][e]);
#pragma unroll
                for (int j = 0; j < 2; j++) db1[t][j] += dz1[t][j] + dz1[t][2 + j];
            }
            uint32_t dz1p[2][4];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                dz1p[k][0] = pack_bf16(dz1[2 * k][0], dz1[2 * k][1]);
                dz1p[k][1] = pack_bf16(dz1[2 * k][2], dz1[2 * k][3]);
                dz1p[k][2] = pack_bf16(dz1[2 * k + 1][0], dz1[2 * k + 1][1]);
                dz1p[k][3] = pack_bf16(dz1[2 * k + 1][2], dz1[2 * k + 1][3]);
            }
            // Weight gradients: reductions over the 16 rows as MMAs with K = rows.
            store_tile(th1[warp], h1);
            store_tile(tdz2[warp], dz2p);
            store_tile(tdz1[warp], dz1p);
            __syncwarp();
            // dW2[k][c] = sum_r h1[r][k] dz2[r][c]: A[m = k][kk = r] = h1[r][k], B[kk = r][n = c] = dz2[r][c].
#pragma unroll
            for (int mu = 0; mu < 2; mu++) {
                const int k0 = 16 * mu + g;
                uint32_t a[4] = {
                    pack_bits(tile_el(th1[warp], 2 * q, k0), tile_el(th1[warp], 2 * q + 1, k0)),
                    pack_bits(tile_el(th1[warp], 2 * q, k0 + 8), tile_el(th1[warp], 2 * q + 1, k0 + 8)),
                    pack_bits(tile_el(th1[warp], 2 * q + 8, k0), tile_el(th1[warp], 2 * q + 9, k0)),
                    pack_bits(tile_el(th1[warp], 2 * q + 8, k0 + 8), tile_el(th1[warp], 2 * q + 9, k0 + 8))};
#pragma unroll
                for (int t = 0; t < 4; t++) {
                    const int c = 8 * t + g;
                    uint32_t b0 = pack_bits(tile_el(tdz2[warp], 2 * q, c), tile_el(tdz2[warp], 2 * q + 1, c));
                    uint32_t b1 = pack_bits(tile_el(tdz2[warp], 2 * q + 8, c), tile_el(tdz2[warp], 2 * q + 9, c));
                    mma16816(dW2[mu][t], a, b0, b1);
                }
            }
            // dW1[f][c] = sum_r x[r][f] dz1[r][c] (features padded to 16 rows of A).
            {
                uint32_t a[4] = {pack_bits(feat_el(st, m, 2 * q, g), feat_el(st, m, 2 * q + 1, g)), 0u,
                                 pack_bits(feat_el(st, m, 2 * q + 8, g), feat_el(st, m, 2 * q + 9, g)), 0u};
#pragma unroll
                for (int t = 0; t < 4; t++) {
                    const int c = 8 * t + g;
                    uint32_t b0 = pack_bits(tile_el(tdz1[warp], 2 * q, c), tile_el(tdz1[warp], 2 * q + 1, c));
                    uint32_t b1 = pack_bits(tile_el(tdz1[warp], 2 * q + 8, c), tile_el(tdz1[warp], 2 * q + 9, c));
                    mma16816(dW1[t], a, b0, b1);
                }
            }
            __syncwarp();
        }
        __syncwarp();
    }
    // Reduce the per-lane column partials over the 8 row groups (lanes with equal q).
#pragma unroll
    for (int t = 0; t < 4; t++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int off = 4; off < 32; off <<= 1) {
                dW3[t][j] += __shfl_xor_sync(0xffffffffu, dW3[t][j], off);
                db2[t][j] += __shfl_xor_sync(0xffffffffu, db2[t][j], off);
                db1[t][j] += __shfl_xor_sync(0xffffffffu, db1[t][j], off);
            }
#pragma unroll
    for (int off = 4; off < 32; off <<= 1) {
        db3 += __shfl_xor_sync(0xffffffffu, db3, off);
        loss += __shfl_xor_sync(0xffffffffu, loss, off);
    }
    float* row = partial + (int64_t)gw * kMlpParams;
#pragma unroll
    for (int mu = 0; mu < 2; mu++)
#pragma unroll
        for (int t = 0; t < 4; t++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int k = 16 * mu + g + (e >= 2 ? 8 : 0), c = 8 * t + 2 * q + (e & 1);
                row[kOffW2 + k * 32 + c] = dW2[mu][t][e];
            }
#pragma unroll
    for (int t = 0; t < 4; t++)
#pragma unroll
        for (int e = 0; e < 2; e++) row[kOffW1 + g * 32 + 8 * t + 2 * q + e] = dW1[t][e];
    if (g == 0) {
#pragma unroll
        for (int t = 0; t < 4; t++)
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int c = 8 * t + 2 * q + j;
                row[kOffW3 + c] = dW3[t][j];
                row[kOffB2 + c] = db2[t][j];
                row[kOffB1 + c] = db1[t][j];
            }
    }
    if (lane == 0) {
        row[kOffB3] = db3;
        loss_partial[gw] = loss;
    }
}

// Sums the warp partials (fixed order) and applies one Adam step to the FP32 master.
__global__ void k_mlp_adam(const float* __restrict__ partial, const float* __restrict__ loss_partial, int rows,
                           float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                           float* __restrict__ grad_out, float* __restrict__ loss_out, float lr, float beta1,
                           float beta2, float eps, float bc1, float bc2, int apply)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && loss_out) {
        float l = 0.f;
        for (int r = 0; r < rows; r++) l += loss_partial[r];
        *loss_out = l;
    }
    if (p >= kMlpParams) return;
    float gsum = 0.f;
    for (int r = 0; r < rows; r++) gsum += partial[(int64_t)r * kMlpParams + p];
    if (grad_out) grad_out[p] = gsum;
    if (!apply) return;
    float a = beta1 * m1[p] + (1.f - beta1) * gsum;
    float b = beta2 * m2[p] + (1.f - beta2) * gsum * gsum;
    m1[p] = a;
    m2[p] = b;
    master[p] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
}

// Batch indices drawn uniformly from [0, n) by a counter-based hash of (seed, slot).
__global__ void k_random_indices(int32_t* idx, int nb, int n, uint64_t seed)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(t + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    idx[t] = (int32_t)(z % (uint64_t)n);
}

void launch_random_indices(int32_t* idx, int nb, int n, uint64_t seed, cudaStream_t s)
{
    if (nb > 0 && n > 0) k_random_indices<<<(nb + 255) / 256, 256, 0, s>>>(idx, nb, n, seed);
}

void launch_mlp_pack(const float* master, MlpPacked* packed, cudaStream_t s)
{
    k_mlp_pack<<<1, 256, 0, s>>>(master, packed);
}


int mlp_grad_rows(int nb)
{
    int blocks = (nb + kMlpThreads - 1) / kMlpThreads;
    blocks = blocks < 1 ? 1 : (blocks > 296 ? 296 : blocks);
    return blocks * kMlpWarps;
}

void launch_mlp_grad(const MlpPacked* packed, const float* feat, const float* target, const int32_t* idx, int nb,
                     float over_weight, float* partial, float* loss_partial, cudaStream_t s)
{
    int rows = mlp_grad_rows(nb);
    k_mlp_grad<<<rows / kMlpWarps, kMlpThreads, 0, s>>>(packed, feat, target, idx, nb, 1.f / (float)nb,
                                                         over_weight, partial, loss_partial);
}

void launch_mlp_grad_blocks(const MlpPacked* packed, const float* feat, const float* target, int nb, int blocks,
                            float* partial, float* loss_partial, cudaStream_t s)
{
    k_mlp_grad<<<blocks, kMlpThreads, 0, s>>>(packed, feat, target, nullptr, nb, 1.f / (float)nb, 1.f, partial,
                                               loss_partial);
}

void launch_mlp_adam(const float* partial, const float* loss_partial, int rows, float* master, float* m1, float* m2,
                     float* grad_out, float* loss_out, float lr, int step, int apply, cudaStream_t s)
{
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(partial, loss_partial, rows, master, m1, m2, grad_out,
                                                        loss_out, lr, beta1, beta2, eps, bc1, bc2, apply);
}

}  // namespace lsp
