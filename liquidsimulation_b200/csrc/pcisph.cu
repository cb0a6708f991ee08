// PCISPH predict-correct pressure loop (PCISPHSolver::accumulatePressureForces, CPU
// branch, PCISPHSolver.cpp:50-170), one kernel per phase:
//   k_pci_predict  predict v_half*, x* from (F + F_p) / rho, collide, first-step velocity wipe
//   k_pci_density  rho* at x* over the start-of-step lists, error, p += delta * error,
//                  the force factor p / rho*^2, and the max |error| of the iteration
//   k_pci_force    F_p = -m rho_i sum dW(x*) (s_i + s_j) (x*_i - x*_j) / d
#include "lsp_device.cuh"
#include "lsp_kernels.h"

namespace lsp {

constexpr int kThreads = 256;

enum { T_W = 0, T_SPIKY_DW = 3 };

// PCISPHSolver.cpp:67-97 for one particle. Iteration 0 starts from p = 0, F_p = 0
// (:58-62). aproximateVelocity (:96, SPHParticle.cpp:46-49) sets v = (v_half_old + v_half)/2;
// within a step it is idempotent, so it is applied in iteration 0 only, after the
// prediction has read v.
__device__ __forceinline__ void pci_predict_one(const DevParams& P, const StepBuffers& b, int i, int iteration)
{
    float4 v4 = b.vel[i];
    V3 F = v3(b.force[i]);
    V3 Fp = iteration == 0 ? v3(0.f, 0.f, 0.f) : v3(b.pforce[i]);
    const float rho = b.rho[i];
    V3 hv = v3(b.half[i]);
    V3 acc = (F + Fp) / rho;
    if (v4.w != 0.f) hv = v3(v4) - acc * P.dt / 2.f;
    V3 ph = hv + acc * P.dt;
    V3 px = v3(b.pos[i]) + ph * P.dt;
    collide_all(b.colliders, P.ncoll, px, ph, P);
    b.ppos[i] = f4(px, 0.f);
    b.phalf[i] = f4(ph, 0.f);
    if (iteration == 0 && !P.keep_initial_velocity) {
        V3 v = (v3(b.old[i]) + v3(b.half[i])) / 2.f;
        b.vel[i] = f4(v, v4.w);
    }
}

__global__ void __launch_bounds__(kThreads) k_pci_predict(DevParams P, StepBuffers b, int iteration)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) b.status->max_err_bits = 0u;
    if (i >= P.n) return;
    pci_predict_one(P, b, i, iteration);
}

// PCISPHSolver.cpp:100-126 for one particle; returns |error| (0 for NaN, which the
// reference's std::max ignores).
__device__ __forceinline__ float pci_density_one(const DevParams& P, const StepBuffers& b, const float* W, int i,
                                                 int iteration)
{
    const V3 xi = v3(b.ppos[i]);
    const int cnt = b.nbr_count[i];
    float sum = 0.f;
    for (int e = 0; e < cnt; e++) {
        int j = b.nbr[(int64_t)e * P.nbr_stride + i];
        sum += lookup(W, mag(v3(b.ppos[j]) - xi), P);
    }
    float pd = P.mass * sum;
    float er = pd - P.rho0;
    float pp = P.delta * er;
    if (pp < 0.f) {
        er *= P.neg;
        pp *= P.neg;
    }
    float p = (iteration == 0 ? 0.f : b.pres[i]) + pp;
    b.prho[i] = pd;
    b.err[i] = er;
    b.pres[i] = p;
    b.sfac[i] = p / (pd * pd);
    float a = fabsf(er);
    return a == a ? a : 0.f;
}

__global__ void __launch_bounds__(kThreads) k_pci_density(DevParams P, StepBuffers b, int iteration)
{
    __shared__ float W[kTableSize];
    __shared__ float wmax[kThreads / 32];
    for (int t = threadIdx.x; t < kTableSize; t += blockDim.x) W[t] = b.tables[T_W * kTableSize + t];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float a = i < P.n ? pci_density_one(P, b, W, i, iteration) : 0.f;
    // Max of non-negative floats: their bit patterns order like the values.
    uint32_t m = __float_as_uint(a);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = __uint_as_float(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t bm = 0;
        for (int w = 0; w < kThreads / 32; w++) bm = max(bm, __float_as_uint(wmax[w]));
        if (bm) atomicMax(&b.status->max_err_bits, bm);
    }
}

// PCISPHSolver.cpp:129-150 for one particle. s = p / rho*^2 is the per-particle factor the
// reference recomputes per pair; the prefactor uses the current density rho_i.
__device__ __forceinline__ void pci_force_one(const DevParams& P, const StepBuffers& b, const float* SDW, int i)
{
    const V3 xi = v3(b.ppos[i]);
    const float tf = b.sfac[i];
    V3 pf = v3(0.f, 0.f, 0.f);
    const int cnt = b.nbr_count[i];
    for (int e = 0; e < cnt; e++) {
        int j = b.nbr[(int64_t)e * P.nbr_stride + i];
        if (j == i) continue;
        const V3 xj = v3(b.ppos[j]);
        float d = mag(xj - xi);
        V3 dir = (xi - xj) / d;
        pf += dir * lookup(SDW, d, P) * (tf + b.sfac[j]);
    }
    pf *= -(P.mass * b.rho[i]);
    if (isnan(pf.x)) pf = v3(0.f, 0.f, 0.f);
    b.pforce[i] = f4(pf, 0.f);
}

__global__ void __launch_bounds__(kThreads) k_pci_force(DevParams P, StepBuffers b)
{
    __shared__ float SDW[kTableSize];
    for (int t = threadIdx.x; t < kTableSize; t += blockDim.x) SDW[t] = b.tables[T_SPIKY_DW * kTableSize + t];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    pci_force_one(P, b, SDW, i);
}

static inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

void launch_pci_predict(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s)
{
    if (P.n) k_pci_predict<<<blocks_for(P.n), kThreads, 0, s>>>(P, b, iteration);
}
void launch_pci_density(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s)
{
    if (P.n) k_pci_density<<<blocks_for(P.n), kThreads, 0, s>>>(P, b, iteration);
}
void launch_pci_force(const DevParams& P, const StepBuffers& b, cudaStream_t s)
{
    if (P.n) k_pci_force<<<blocks_for(P.n), kThreads, 0, s>>>(P, b);
}

bool launch_pci_loop(const DevParams&, const StepBuffers&, cudaStream_t, int* grid_used)
{
    if (grid_used) *grid_used = 0;
    return false;
}

}  // namespace lsp
