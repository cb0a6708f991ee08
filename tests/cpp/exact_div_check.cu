// GPU check of recip_rn and div_by (liquidsimulation_b200/csrc/lsp_device.cuh) against the
// IEEE reciprocal (__frcp_rn) and IEEE division (__fdiv_rn) of the same device:
//   1. recip_rn(d) for EVERY float d in [2^-126, 2^126], where 1 / d is normal (above it the
//      approximate reciprocal flushes the subnormal result to zero; callers stay far below);
//   2. div_by(a, d, recip_rn(d)) for 2^32 pseudo-random pairs with 2^-99 <= d <= 2^28 and
//      |a| <= d (a = 0, a = +-d, a a power of two times d, and a one ulp off those included);
//   3. the same for d in [1e-3, 0.1] (neighbour distances) and a the components of random
//      difference vectors of length d;
//   4. sqrt_rn(s) for EVERY float s from 2^-102 up;
//   5. div_by on 2^32 pairs in the non-pressure pass's ranges: d in [2^-20, 2^20] and a 0
//      or of magnitude in [2^-80, 2^87] (counted with 2.).
// Prints the mismatch counts; exit status 0 when all are zero.
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>
#include "lsp_device.cuh"

using lsp::div_by;
using lsp::recip_rn;

__device__ unsigned long long g_bad[3];
__device__ unsigned int g_first[3][2];

__device__ __forceinline__ uint64_t mix(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__global__ void k_recip(uint32_t lo, uint64_t count)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const float d = __uint_as_float(lo + (uint32_t)t);
        const float y = recip_rn(d), z = __frcp_rn(d);
        if (__float_as_uint(y) != __float_as_uint(z)) {
            if (atomicAdd(&g_bad[0], 1ull) == 0) { g_first[0][0] = __float_as_uint(d); g_first[0][1] = 0; }
        }
    }
}

__device__ unsigned long long g_sqrt_bad;
__device__ unsigned int g_sqrt_first;

__global__ void k_sqrt(uint32_t lo, uint64_t count)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const float v = __uint_as_float(lo + (uint32_t)t);
        if (__float_as_uint(lsp::sqrt_rn(v)) != __float_as_uint(__fsqrt_rn(v))) {
            if (atomicAdd(&g_sqrt_bad, 1ull) == 0) g_sqrt_first = __float_as_uint(v);
        }
    }
}

__global__ void k_div(uint64_t seed, uint64_t count, int mode)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < count;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r1 = mix(seed ^ (t * 2)), r2 = mix(seed ^ (t * 2 + 1));
        float d, a;
        if (mode == 0) {
            // d: exponent uniform in [-99, 27], random significand; a: |a| <= d of several kinds.
            const int e = -99 + (int)(r1 % 127);
            d = ldexpf(1.f + (float)((r1 >> 8) & 0x7fffff) * 0x1p-23f, e);
            if (d > 0x1p28f) d = 0x1p28f;
            const uint32_t kind = (uint32_t)(r2 & 7);
            const float u = (float)((r2 >> 8) & 0xffffff) * 0x1p-24f;   // [0, 1)
            if (kind == 0) a = 0.f;
            else if (kind == 1) a = d;
            else if (kind == 2) a = ldexpf(d, -(int)((r2 >> 40) % 70));
            else if (kind == 3) a = __uint_as_float(__float_as_uint(ldexpf(d, -(int)((r2 >> 40) % 70))) + 1);
            else if (kind == 4) a = __uint_as_float(__float_as_uint(d) - 1 - (uint32_t)((r2 >> 40) & 15));
            else a = __fmul_rn(d, u);
            if (fabsf(a) != 0.f && fabsf(a) < 0x1p-99f) a = 0x1p-99f;
            if ((r2 >> 63) & 1) a = -a;
        } else if (mode == 2) {
            // The non-pressure pass's ranges: d (a density) in [2^-20, 2^20], |a| 0 or in
            // [2^-80, 2^87], exponents uniform.
            d = ldexpf(1.f + (float)((r1 >> 8) & 0x7fffff) * 0x1p-23f, -20 + (int)(r1 % 40));
            a = ldexpf(1.f + (float)((r2 >> 8) & 0x7fffff) * 0x1p-23f, -80 + (int)((r2 >> 40) % 167));
            if ((r2 & 63) == 0) a = 0.f;
            if ((r2 >> 63) & 1) a = -a;
        } else {
            // Neighbour-like pairs: a random direction scaled to length d in [1e-3, 0.1].
            const float x = (float)((r1 >> 8) & 0xffffff) * 0x1p-24f - 0.5f;
            const float y = (float)((r2 >> 8) & 0xffffff) * 0x1p-24f - 0.5f;
            const float z = (float)((r1 >> 40) & 0xffffff) * 0x1p-24f - 0.5f;
            const float s = 1e-3f + (float)((r2 >> 40) & 0xffffff) * 0x1p-24f * 0.099f;
            const float px = x * s, py = y * s, pz = z * s;
            d = sqrtf(px * px + py * py + pz * pz);
            if (!(d >= 0x1p-99f)) continue;
            a = (t & 1) ? px : pz;
        }
        const float q = div_by(a, d, recip_rn(d)), w = __fdiv_rn(a, d);
        if (__float_as_uint(q) != __float_as_uint(w) && !(q == 0.f && w == 0.f)) {
            const int slot = mode == 2 ? 1 : 1 + (mode > 0);
            if (atomicAdd(&g_bad[slot], 1ull) == 0) {
                g_first[slot][0] = __float_as_uint(a);
                g_first[slot][1] = __float_as_uint(d);
            }
        }
    }
}

int main()
{
    const uint32_t lo = 0x00800000u, hi = 0x7e800000u;   // 2^-126 .. 2^126
    k_recip<<<148 * 16, 256>>>(lo, (uint64_t)(hi - lo) + 1);
    k_div<<<148 * 16, 256>>>(12345, 1ull << 32, 0);
    k_div<<<148 * 16, 256>>>(777, 1ull << 31, 1);
    k_div<<<148 * 16, 256>>>(4242, 1ull << 32, 2);
    const uint32_t s_lo = 0x0c800000u, s_hi = 0x7f7fffffu;   // 2^-102 .. the largest float
    k_sqrt<<<148 * 16, 256>>>(s_lo, (uint64_t)(s_hi - s_lo) + 1);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        std::printf("cuda error %s\n", cudaGetErrorString(e));
        return 2;
    }
    unsigned long long bad[3];
    unsigned int first[3][2];
    cudaMemcpyFromSymbol(bad, g_bad, sizeof(bad));
    cudaMemcpyFromSymbol(first, g_first, sizeof(first));
    const char* name[3] = {"reciprocal (every float in [2^-126, 2^126])", "division (2^33 random pairs, |a| <= d and the density ranges)",
                           "division (2^31 neighbour-like pairs)"};
    for (int k = 0; k < 3; k++) std::printf("%s: %llu mismatches\n", name[k], bad[k]);
    if (bad[0]) std::printf("  first reciprocal mismatch: d=0x%08x\n", first[0][0]);
    for (int k = 1; k < 3; k++)
        if (bad[k]) std::printf("  first division mismatch: a=0x%08x d=0x%08x\n", first[k][0], first[k][1]);
    unsigned long long sb = 0;
    unsigned int sf = 0;
    cudaMemcpyFromSymbol(&sb, g_sqrt_bad, sizeof(sb));
    cudaMemcpyFromSymbol(&sf, g_sqrt_first, sizeof(sf));
    std::printf("square root (every float from 2^-102 up): %llu mismatches\n", sb);
    if (sb) std::printf("  first square-root mismatch: s=0x%08x\n", sf);
    return (bad[0] || bad[1] || bad[2] || sb) ? 1 : 0;
}
