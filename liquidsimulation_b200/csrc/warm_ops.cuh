// Learned warm start, per particle: the features of iteration 0 and its density pass.
// Shared by the single-scene kernel (pcisph.cu) and the batched one (batch.cu).
#pragma once

#include "lsp_kernels.h"
#include "mlp.cuh"
#include "particle_ops.cuh"

namespace lsp {

// Features of particle i at iteration 0 (all dimensionless):
//   f0 predicted density error at zero pressure, in % of rho0 (clamped to +-50)
//   f1 f2 f3  pressures of the previous three steps / p_scale
//   f4 neighbour count / 32      f5 |v| dt / h * 10      f6 |grad rho| h / rho0
//   f7 distance to the nearest collider surface / (4 h), clamped to [0, 1]
// p_scale = delta * 0.01 * rho0 is the pressure one correction assigns to a 1 % error.

__device__ __forceinline__ float collider_distance(const Collider& o, V3 x)
{
    V3 d = v3(fabsf(x.x - o.cx), fabsf(x.y - o.cy), fabsf(x.z - o.cz));
    if (o.sphere) {
        float r = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        return o.boundary ? o.radius - r : r - o.radius;
    }
    if (o.boundary) return fminf(fminf(o.hx - d.x, o.hy - d.y), o.hz - d.z);
    return fmaxf(fmaxf(d.x - o.hx, d.y - o.hy), d.z - o.hz);
}

__device__ __forceinline__ void warm_features(const DevParams& P, const StepBuffers& b, const float4* hist,
                                              const float* gradrho, float p_scale, int i, float pd, int cnt,
                                              float (&f)[kMlpIn])
{
    const float4 hs = hist[i];
    const float4 v = b.vel[i];
    const V3 x = v3(b.pos[i]);
    f[0] = fminf(fmaxf((pd - P.rho0) / (0.01f * P.rho0), -50.f), 50.f);
    f[1] = hs.x / p_scale;
    f[2] = hs.y / p_scale;
    f[3] = hs.z / p_scale;
    f[4] = (float)cnt * (1.f / 32.f);
    f[5] = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z) * P.dt / P.h * 10.f;
    f[6] = gradrho[i] * P.h / P.rho0;
    float dist = 4.f * P.h;
    for (int c = 0; c < P.ncoll; c++)
        dist = fminf(dist, fmaxf(collider_distance(b.colliders[P.coll_off + c], x), 0.f));
    f[7] = dist / (4.f * P.h);
}

// Iteration 0's density pass for particle i (PCISPHSolver.cpp:100-126 with p starting at 0)
// with the warm-start features (stored when feat is non-null); `valid` marks threads with a
// particle. The network's guess, when used, replaces the stored first correction afterwards
// (mlp_tc.cu). Returns |error| (0 for NaN and for invalid threads).
__device__ __forceinline__ float density_first(const DevParams& P, const StepBuffers& b, float* feat,
                                               const float4* hist, const float* gradrho, float p_scale,
                                               const float* W, const float* TH2, int i, bool valid)
{
    float a = 0.f, pd = 0.f, p = 0.f;
    float f[kMlpIn];
    if (valid) {
        const V3 xi = v3(b.ppos[i]);
        const int cnt = __ldg(b.nbr_count + i);
        float sum = 0.f;
        for_each_neighbor<4>(b.nbr, i, P.nbr_stride, cnt, [&](int j) { return b.ppos[j]; },
                             [&](int, float4 pj) { sum += lookup_sq(W, TH2, sqmag(v3(pj) - xi), P); });
        pd = P.mass * sum;
        float er = pd - P.rho0;
        float pp = P.delta * er;
        if (pp < 0.f) {
            er *= P.neg;
            pp *= P.neg;
        }
        p = 0.f + pp;
        b.prho[i] = pd;
        b.err[i] = er;
        a = fabsf(er);
        a = a == a ? a : 0.f;
        warm_features(P, b, hist, gradrho, p_scale, i, pd, cnt, f);
        if (feat) {
#pragma unroll
            for (int c = 0; c < kMlpIn; c++) feat[(int64_t)i * kMlpIn + c] = f[c];
        }
    }
    if (valid) {
        b.pres[i] = p;
        reinterpret_cast<float*>(b.ppos + i)[3] = p / (pd * pd);
    }
    return a;
}

}  // namespace lsp
