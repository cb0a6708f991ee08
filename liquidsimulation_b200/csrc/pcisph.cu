// PCISPH predict-correct pressure loop (PCISPHSolver::accumulatePressureForces, CPU
// branch, PCISPHSolver.cpp:50-170), one kernel per phase:
//   k_pci_predict  predict v_half*, x* from (F + F_p) / rho, collide, first-step velocity wipe
//   k_pci_density  rho* at x* over the start-of-step lists, error, p += delta * error,
//                  the force factor p / rho*^2, and the max |error| of the iteration
//   k_pci_force    F_p = -m rho_i sum dW(x*) (s_i + s_j) (x*_i - x*_j) / d
#include "lsp_device.cuh"
#include "lsp_kernels.h"

#include <algorithm>

namespace lsp {

constexpr int kThreads = 256;

enum { T_W = 0, T_SPIKY_DW = 3 };

// PCISPHSolver.cpp:67-97 for one particle. Iteration 0 starts from p = 0, F_p = 0
// (:58-62). aproximateVelocity (:96, SPHParticle.cpp:46-49) sets v = (v_half_old + v_half)/2;
// within a step it is idempotent, so it is applied in iteration 0 only, after the
// prediction has read v.
__device__ __forceinline__ void pci_predict_one(const DevParams& P, const StepBuffers& b, int i, int iteration,
                                                float4* ppos)
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
    ppos[i] = f4(px, 0.f);
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
    pci_predict_one(P, b, i, iteration, b.ppos);
}

// PCISPHSolver.cpp:100-126 for one particle; returns |error| (0 for NaN, which the
// reference's std::max ignores).
__device__ __forceinline__ float pci_density_one(const DevParams& P, const StepBuffers& b, const float* W, int i,
                                                 int iteration, float4* ppos)
{
    const V3 xi = v3(ppos[i]);
    const int cnt = __ldg(b.nbr_count + i);
    const int32_t* list = b.nbr + i;
    float sum = 0.f;
    for (int e = 0; e < cnt; e++) {
        int j = __ldg(list);
        list += P.nbr_stride;
        sum += lookup(W, mag(v3(ppos[j]) - xi), P);
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
    // p / rho*^2, the per-particle factor of the pressure force, rides in x*.w so the force
    // pass fetches a neighbour's position and factor in one 16-byte load. Other threads
    // read only x*.xyz of this element during this pass.
    reinterpret_cast<float*>(ppos + i)[3] = p / (pd * pd);
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
    float a = i < P.n ? pci_density_one(P, b, W, i, iteration, b.ppos) : 0.f;
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
__device__ __forceinline__ void pci_force_one(const DevParams& P, const StepBuffers& b, const float* SDW, int i,
                                              const float4* ppos)
{
    const float4 pi4 = ppos[i];
    const V3 xi = v3(pi4);
    const float tf = pi4.w;
    V3 pf = v3(0.f, 0.f, 0.f);
    const int cnt = __ldg(b.nbr_count + i);
    const int32_t* list = b.nbr + i;
    for (int e = 0; e < cnt; e++) {
        int j = __ldg(list);
        list += P.nbr_stride;
        if (j == i) continue;
        const float4 pj4 = ppos[j];
        const V3 xj = v3(pj4);
        float d = mag(xj - xi);
        V3 dir = (xi - xj) / d;
        pf += dir * lookup(SDW, d, P) * (tf + pj4.w);
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
    pci_force_one(P, b, SDW, i, b.ppos);
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

// ------------------------------------------------------------------ persistent loop
//
// k_pci_loop runs the whole predict-correct loop in one cooperative launch (every block
// resident), with grid barriers between the phases:
//
//   predict(0)
//   for k: | barrier | density(k) + block max |error| -> maxerr[k] | barrier |
//          decide (all threads read maxerr[k]): done = (converged && k+1 >= min) || k+1 == max
//          force(k), and when not done predict(k+1) in the same pass
//
// force(k) reads the predicted positions of iteration k while predict(k+1) writes
// those of k+1, so x* is double-buffered (ppos, ppos_alt by iteration parity). Every
// other array a fused pass writes is only read by the same thread before the next
// barrier. Mutable arrays are read with plain coherent loads (no read-only cache path).
//
// The grid barrier spins with a bounded count: past the limit it raises kErrTimeout and
// an abort word that makes every block leave; the host reports LSP_ERR_TIMEOUT.

constexpr unsigned long long kBarrierSpinLimit = 1ull << 25;

struct LoopSync {
    uint32_t count;
    uint32_t gen;
    uint32_t abort;
    uint32_t pad;
};

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// Returns false when the loop must stop (a barrier gave up somewhere).
__device__ bool grid_barrier(LoopSync* sy, DevStatus* st)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const uint32_t g = ld_volatile(&sy->gen);
        __threadfence();
        uint32_t arrived = atomicAdd(&sy->count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&sy->count, 0u);
            __threadfence();
            atomicAdd(&sy->gen, 1u);
        } else {
            unsigned long long spins = 0;
            while (ld_volatile(&sy->gen) == g) {
                if (ld_volatile(&sy->abort)) { ok = 0; break; }
                if (++spins > kBarrierSpinLimit) {
                    atomicExch(&sy->abort, 1u);
                    atomicOr(&st->error_flags, kErrTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (ld_volatile(&sy->abort)) ok = 0;
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__global__ void __launch_bounds__(kThreads) k_pci_loop(DevParams P, StepBuffers b, float4* ppos_alt, LoopSync* sy,
                                                      uint32_t* maxerr)
{
    __shared__ float W[kTableSize], SDW[kTableSize];
    __shared__ float wmax[kThreads / 32];
    for (int t = threadIdx.x; t < kTableSize; t += blockDim.x) {
        W[t] = b.tables[T_W * kTableSize + t];
        SDW[t] = b.tables[T_SPIKY_DW * kTableSize + t];
    }
    __syncthreads();
    float4* pp[2] = {b.ppos, ppos_alt};
    const int stride = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = tid; i < P.n; i += stride) pci_predict_one(P, b, i, 0, pp[0]);
    int k = 0;
    bool conv = false, done = false;
    for (k = 0; k < P.max_it; k++) {
        if (!grid_barrier(sy, b.status)) return;
        float m = 0.f;
        for (int i = tid; i < P.n; i += stride) m = fmaxf(m, pci_density_one(P, b, W, i, k, pp[k & 1]));
        uint32_t mb = __float_as_uint(m);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mb = max(mb, __shfl_xor_sync(0xffffffffu, mb, off));
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = __uint_as_float(mb);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t bm = 0;
            for (int w = 0; w < kThreads / 32; w++) bm = max(bm, __float_as_uint(wmax[w]));
            if (bm) atomicMax(&maxerr[k], bm);
        }
        if (!grid_barrier(sy, b.status)) return;
        // PCISPHSolver.cpp:152-162: ratio = max|e| / rho0 in float, exit when below eta.
        const float me = __uint_as_float(ld_volatile(&maxerr[k]));
        const float ratio = me / P.rho0;
        conv = fabsf(ratio) < P.eta;
        done = (conv && k + 1 >= P.min_it) || (k + 1 >= P.max_it);
        for (int i = tid; i < P.n; i += stride) {
            pci_force_one(P, b, SDW, i, pp[k & 1]);
            if (!done) pci_predict_one(P, b, i, k + 1, pp[(k + 1) & 1]);
        }
        if (done) break;
    }
    if (tid == 0) {
        int it = k < P.max_it ? k + 1 : P.max_it;
        b.status->iterations = it;
        b.status->converged = conv ? 1 : 0;
        b.status->max_err_bits = it > 0 ? ld_volatile(&maxerr[it - 1]) : 0u;
    }
}

static int g_loop_blocks_per_sm = -1;
static int g_sm_count = 0;

bool launch_pci_loop(const DevParams& P, const StepBuffers& b, float4* ppos_alt, void* sync, uint32_t* maxerr,
                     cudaStream_t s, int* grid_used)
{
    if (grid_used) *grid_used = 0;
    if (P.n <= 0 || P.max_it <= 0) return false;
    if (g_loop_blocks_per_sm < 0) {
        int dev = 0, coop = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        int per = 0;
        if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pci_loop, kThreads, 0) == cudaSuccess)
            g_loop_blocks_per_sm = per;
        else
            g_loop_blocks_per_sm = 0;
    }
    if (g_loop_blocks_per_sm <= 0) return false;
    int need = (int)((P.n + kThreads - 1) / kThreads);
    int grid = std::min(need, g_loop_blocks_per_sm * g_sm_count);
    DevParams Pc = P;
    StepBuffers bc = b;
    LoopSync* sy = (LoopSync*)sync;
    void* args[] = {&Pc, &bc, &ppos_alt, &sy, &maxerr};
    if (cudaLaunchCooperativeKernel((const void*)k_pci_loop, dim3(grid), dim3(kThreads), args, 0, s) != cudaSuccess)
        return false;
    if (grid_used) *grid_used = grid;
    return true;
}

}  // namespace lsp
