// SPH passes over the start-of-step neighbour lists: density/pressure, non-pressure
// forces (gravity, surface tension, viscosity), the SPH pressure force, and the fused
// leapfrog integration + collision pass.
//
// Thread per particle; each thread walks its own neighbour list in the reference's
// order, so its sums round exactly as the reference CPU solver's do. The lookup tables
// the pass needs are staged in shared memory (4 KB each) once per block.
#include "lsp_device.cuh"
#include "lsp_kernels.h"

namespace lsp {

constexpr int kThreads = 256;

enum { T_W = 0, T_DW = 1, T_D2W = 2, T_SPIKY_DW = 3, T_VISC_D2W = 4, T_THRESH = 5 };

__device__ __forceinline__ void stage_table(float* sm, const float* g, int t)
{
    const int len = t == T_THRESH ? kTableSize + 1 : kTableSize;
    for (int i = threadIdx.x; i < len; i += blockDim.x) sm[i] = g[t * kTableSize + i];
}

// SPHSolver::calcParticleDensityPressure, CPU branch (SPHSolver.cpp:442-463).
__global__ void __launch_bounds__(kThreads) k_density(DevParams P, StepBuffers b)
{
    __shared__ float W[kTableSize], TH[kTableSize + 1];
    stage_table(W, b.tables, T_W);
    stage_table(TH, b.tables, T_THRESH);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const V3 xi = v3(b.pos[i]);
    float sum = 0.f;
    for_each_neighbor<4>(b.nbr + i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return b.pos[j]; },
                         [&](int, float4 pj) { sum += lookup(W, TH, mag(v3(pj) - xi), P); });
    float rho = P.mass * sum;
    float pr = P.stiffness * (rho - P.rho0);
    if (pr < 0.f) pr *= P.neg;
    b.rho[i] = rho;
    b.pres[i] = pr;
}

// SPHSolver::accumulateNonPressureForces, CPU branch (SPHSolver.cpp:201-248). The
// reference walks the list up to three times (normal, colour Laplacian when the normal
// exceeds the threshold, viscosity); each sum is independent, so one walk computes all
// three with the same per-sum rounding.
template <bool kGrad>
__global__ void __launch_bounds__(kThreads) k_nonpressure(DevParams P, StepBuffers b)
{
    __shared__ float DW[kTableSize], D2W[kTableSize], VD2W[kTableSize], TH[kTableSize + 1];
    stage_table(TH, b.tables, T_THRESH);
    stage_table(DW, b.tables, T_DW);
    stage_table(D2W, b.tables, T_D2W);
    stage_table(VD2W, b.tables, T_VISC_D2W);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const V3 xi = v3(b.pos[i]);
    const V3 vi = v3(b.vel[i]);
    const float rhoi = b.rho[i];
    V3 F = v3(0.f, 0.f, 0.f);
    F += v3(P.gx, P.gy, P.gz) * rhoi;
    V3 normal = v3(0.f, 0.f, 0.f);
    V3 visc = v3(0.f, 0.f, 0.f);
    float lap = 0.f;
    V3 grad = v3(0.f, 0.f, 0.f);   // sum (rho_j - rho_i) / rho_j grad W_ij: a warm-start feature only
    struct Rec {
        float4 x, v;
        float rho;
    };
    for_each_neighbor<2>(b.nbr + i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return Rec{b.pos[j], b.vel[j], b.rho[j]}; },
                         [&](int j, const Rec& r) {
                             const V3 xj = v3(r.x);
                             V3 dir = xi - xj;
                             float d = mag(xj - xi);
                             normal += dir * lookup(DW, TH, d, P) / r.rho;
                             lap += lookup(D2W, TH, d, P) / r.rho;
                             if (j != i) visc += ((v3(r.v) - vi) / r.rho) * lookup(VD2W, TH, d, P);
                             if (kGrad) grad += dir * (lookup(DW, TH, d, P) * ((r.rho - rhoi) / r.rho));
                         });
    if (kGrad) b.gradrho[i] = P.mass * mag(grad);
    normal *= P.mass;
    float len = mag(normal);
    if (len > P.sigma_thr) F += (normal / len) * (-P.sigma * lap * P.mass);
    visc *= P.viscosity * P.mass;
    F += visc;
    b.force[i] = f4(F, 0.f);
}

// SPHSolver::accumulatePressureForces, CPU branch (SPHSolver.cpp:268-290).
__global__ void __launch_bounds__(kThreads) k_sph_pressure(DevParams P, StepBuffers b)
{
    __shared__ float SDW[kTableSize], TH[kTableSize + 1];
    stage_table(SDW, b.tables, T_SPIKY_DW);
    stage_table(TH, b.tables, T_THRESH);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const V3 xi = v3(b.pos[i]);
    const float rhoi = b.rho[i];
    const float tf = b.pres[i] / (rhoi * rhoi);
    V3 pf = v3(0.f, 0.f, 0.f);
    struct Rec {
        float4 x;
        float rho, p;
    };
    for_each_neighbor<4>(b.nbr + i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return Rec{b.pos[j], b.rho[j], b.pres[j]}; },
                         [&](int j, const Rec& r) {
                             if (j == i) return;
                             const V3 xj = v3(r.x);
                             float d = mag(xi - xj);
                             V3 dir = (xi - xj) / d;
                             pf += dir * lookup(SDW, TH, d, P) * (tf + r.p / (r.rho * r.rho));
                         });
    pf *= -(P.mass * rhoi);
    V3 F = v3(b.force[i]);
    F += pf;
    b.force[i] = f4(F, 0.f);
}

// SPHParticle::integrate (SPHParticle.cpp:30-44) then SPHSolver::handleCollisions
// (SPHSolver.cpp:337-355) for one particle. With add_pforce the PCISPH pressure force is
// added first (PCISPHSolver.cpp:166-169).
__global__ void __launch_bounds__(kThreads) k_integrate_collide(DevParams P, StepBuffers b, int add_pforce)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    float4 p4 = b.pos[i], v4 = b.vel[i], h4 = b.half[i], o4 = b.old[i];
    V3 F = v3(b.force[i]);
    if (add_pforce) F += v3(b.pforce[i]);
    const float rho = b.rho[i];
    V3 acc = F / rho;
    V3 half = v3(h4);
    float first = v4.w;
    if (first != 0.f) {
        half = v3(v4) - acc * P.dt / 2.f;
        first = 0.f;
    }
    V3 old = half;
    half = v3(half.x + acc.x * P.dt, half.y + acc.y * P.dt, half.z + acc.z * P.dt);
    V3 x = v3(p4);
    x = v3(x.x + half.x * P.dt, x.y + half.y * P.dt, x.z + half.z * P.dt);
    collide_all(b.colliders, P.ncoll, x, half, P);
    V3 v = (old + half) / 2.f;
    b.pos[i] = f4(x, p4.w);
    b.vel[i] = f4(v, first);
    b.half[i] = f4(half, h4.w);
    b.old[i] = f4(old, o4.w);
    if (b.hist) {
        // Warm-start pressure history: (p_n, p_{n-1}, p_{n-2}) for the next step's features.
        float4 hs = b.hist[i];
        b.hist[i] = make_float4(b.pres[i], hs.x, hs.y, 0.f);
    }
}

static inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

void launch_density(const DevParams& P, const StepBuffers& b, cudaStream_t s)
{
    if (P.n) k_density<<<blocks_for(P.n), kThreads, 0, s>>>(P, b);
}
void launch_nonpressure(const DevParams& P, const StepBuffers& b, cudaStream_t s)
{
    if (!P.n) return;
    if (b.gradrho)
        k_nonpressure<true><<<blocks_for(P.n), kThreads, 0, s>>>(P, b);
    else
        k_nonpressure<false><<<blocks_for(P.n), kThreads, 0, s>>>(P, b);
}
void launch_sph_pressure(const DevParams& P, const StepBuffers& b, cudaStream_t s)
{
    if (P.n) k_sph_pressure<<<blocks_for(P.n), kThreads, 0, s>>>(P, b);
}
void launch_integrate_collide(const DevParams& P, const StepBuffers& b, bool add_pforce, cudaStream_t s)
{
    if (P.n) k_integrate_collide<<<blocks_for(P.n), kThreads, 0, s>>>(P, b, add_pforce ? 1 : 0);
}

}  // namespace lsp
