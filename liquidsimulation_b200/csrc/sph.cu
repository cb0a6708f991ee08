// SPH passes over the start-of-step neighbour lists: non-pressure forces (gravity,
// surface tension, viscosity), the SPH pressure force, and the fused leapfrog integration +
// collision pass (the density and pressure are summed in the neighbour build, grid.cu).
//
// Thread per particle; each thread walks its own neighbour list in the reference's
// order, so its sums round exactly as the reference CPU solver's do. The lookup tables
// the pass needs are staged in shared memory once per block.
#include "lsp_device.cuh"
#include "lsp_kernels.h"
#include "particle_ops.cuh"

#include <algorithm>

namespace lsp {

constexpr int kThreads = 256;

// SPHSolver::accumulateNonPressureForces, CPU branch (SPHSolver.cpp:201-248). The
// reference walks the list up to three times (normal, colour Laplacian when the normal
// exceeds the threshold, viscosity); each sum is independent, so one walk computes all
// three with the same per-sum rounding.
template <bool kGrad>
__global__ void __launch_bounds__(kThreads) k_nonpressure(DevParams P, StepBuffers b)
{
    __shared__ float4 NA[kTableSize], NB[kTableSize];
    stage_nonpressure_slots(NA, NB, b.tables);
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x)
        nonpressure_one<kGrad>(P, b, NA, NB, i);
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
    sph_pressure_one(P, b, SDW, TH, i);
}

// SPHParticle::integrate (SPHParticle.cpp:30-44) then SPHSolver::handleCollisions
// (SPHSolver.cpp:337-355) for one particle. With add_pforce the PCISPH pressure force is
// added first (PCISPHSolver.cpp:166-169).
__global__ void __launch_bounds__(kThreads) k_integrate_collide(DevParams P, StepBuffers b, int add_pforce)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    integrate_one(P, b, i, add_pforce);
}

static inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// The non-pressure pass loops over the particles with four blocks per SM, so each block
// stages its tables (32 KB of slot records) once for several particles per thread instead
// of once per 256 particles: 7 % faster at 1M particles.
static inline unsigned stride_grid(int64_t n, int per_sm)
{
    return std::min<unsigned>(blocks_for(n, kThreads), (unsigned)(per_sm * device_sm_count()));
}

void launch_nonpressure(const DevParams& P, const StepBuffers& b, cudaStream_t s)
{
    if (!P.n) return;
    if (b.gradrho)
        k_nonpressure<true><<<stride_grid(P.n, 4), kThreads, 0, s>>>(P, b);
    else
        k_nonpressure<false><<<stride_grid(P.n, 4), kThreads, 0, s>>>(P, b);
}
void launch_sph_pressure(const DevParams& P, const StepBuffers& b, cudaStream_t s)
{
    if (P.n) k_sph_pressure<<<blocks_for(P.n, kThreads), kThreads, 0, s>>>(P, b);
}
void launch_integrate_collide(const DevParams& P, const StepBuffers& b, bool add_pforce, cudaStream_t s)
{
    if (P.n) k_integrate_collide<<<blocks_for(P.n, kThreads), kThreads, 0, s>>>(P, b, add_pforce ? 1 : 0);
}

}  // namespace lsp
