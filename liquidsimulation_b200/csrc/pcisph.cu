// PCISPH predict-correct pressure loop (PCISPHSolver::accumulatePressureForces, CPU
// branch, PCISPHSolver.cpp:50-170), one kernel per phase:
//   k_pci_predict  predict v_half*, x* from (F + F_p) / rho, collide, first-step velocity wipe
//   k_pci_density  rho* at x* over the start-of-step lists, error, p += delta * error,
//                  the force factor p / rho*^2, and the max |error| of the iteration
//   k_pci_force    F_p = -m rho_i sum dW(x*) (s_i + s_j) (x*_i - x*_j) / d
#include "lsp_device.cuh"
#include "lsp_kernels.h"
#include "mlp.cuh"
#include "loop_sync.cuh"
#include "particle_ops.cuh"
#include "warm_ops.cuh"
#include "host_util.h"

#include <algorithm>
#include <mutex>
#include <string>

namespace lsp {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_pci_predict(DevParams P, StepBuffers b, int iteration)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) b.status->max_err_bits = 0u;
    if (i >= P.n) return;
    pci_predict_one(P, b, i, iteration, b.ppos);
}

__global__ void __launch_bounds__(kThreads) k_pci_density(DevParams P, StepBuffers b, int iteration)
{
    __shared__ float W[kTableSize], TH2[kTableSize + 1];
    __shared__ float wmax[kThreads / 32];
    stage_table(W, b.tables, T_W);
    stage_table(TH2, b.tables, T_THRESH2);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float a = i < P.n ? pci_density_one(P, b, W, TH2, i, iteration, b.ppos) : 0.f;
    // Max of non-negative floats: their bit patterns order like the values.
    uint32_t m = __float_as_uint(a);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = __uint_as_float(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t bm = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) bm = max(bm, __float_as_uint(wmax[w]));
        if (bm) atomicMax(&b.status->max_err_bits, bm);
    }
}

__global__ void __launch_bounds__(kThreads) k_pci_force(DevParams P, StepBuffers b)
{
    __shared__ float SDW[kTableSize], TH[kTableSize + 1];
    stage_table(SDW, b.tables, T_SPIKY_DW);
    stage_table(TH, b.tables, T_THRESH);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    pci_force_one(P, b, SDW, TH, i, b.ppos);
}

static inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

void launch_pci_predict(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s)
{
    if (P.n) k_pci_predict<<<blocks_for(P.n, kThreads), kThreads, 0, s>>>(P, b, iteration);
}
void launch_pci_density(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s)
{
    if (P.n) k_pci_density<<<blocks_for(P.n, kThreads), kThreads, 0, s>>>(P, b, iteration);
}
void launch_pci_force(const DevParams& P, const StepBuffers& b, cudaStream_t s)
{
    if (P.n) k_pci_force<<<blocks_for(P.n, kThreads), kThreads, 0, s>>>(P, b);
}

// ------------------------------------------------------------------ learned warm start

// Iteration 0's density pass (PCISPHSolver.cpp:100-126 with p starting at 0) that also
// stores the warm-start features (warm_ops.cuh); its pressures are those of the plain pass
// until the network's guess replaces them (mlp_tc.cu).
__global__ void __launch_bounds__(kThreads) k_pci_density_first(DevParams P, StepBuffers b, WarmArgs w)
{
    __shared__ float W[kTableSize], TH2[kTableSize + 1];
    __shared__ float wmax[kThreads / 32];
    stage_table(W, b.tables, T_W);
    stage_table(TH2, b.tables, T_THRESH2);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const float a = density_first(P, b, w.feat, w.hist, w.gradrho, w.p_scale, W, TH2, i, i < P.n);
    uint32_t m = __float_as_uint(a);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = __uint_as_float(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t bm = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) bm = max(bm, __float_as_uint(wmax[k]));
        if (bm) {
            atomicMax(w.maxerr0, bm);
            atomicMax(&b.status->max_err_bits, bm);
        }
    }
}

void launch_pci_density_first(const DevParams& P, const StepBuffers& b, const WarmArgs& w, cudaStream_t s)
{
    if (P.n) k_pci_density_first<<<blocks_for(P.n, kThreads), kThreads, 0, s>>>(P, b, w);
}

// ------------------------------------------------------------------ persistent loop
//
// k_pci_loop runs the whole predict-correct loop in one cooperative launch (every block
// resident), with grid barriers between the phases:
//
//   predict(0)
//   for k: | barrier | density(k) + block max |error| -> maxerr[k] | barrier |
//          decide (all threads read maxerr[k]): done = (converged && k+1 >= min) || k+1 == max
//          force(k), and when not done predict(k+1) in the same pass, else the
//          integration and collisions of the step
//
// force(k) reads the predicted positions of iteration k while predict(k+1) writes
// those of k+1, so x* is double-buffered (ppos, ppos_alt by iteration parity). Every
// other array a fused pass writes is only read by the same thread before the next
// barrier. Mutable arrays are read with plain coherent loads (no read-only cache path).
//
// The grid barrier spins with a bounded count: past the limit it raises kErrTimeout and
// an abort word that makes every block leave; the host reports LSP_ERR_TIMEOUT.

// One 1024-thread block per SM at 64 registers: measured about 10 % faster than the
// unconstrained allocation (79 registers, 768 threads per SM; 1280 threads per SM are
// slower too), and one block of 1024 beats two of 512 by 3.5 % and four of 256 by 4 % (a
// grid barrier with 148 arrivals, one table copy per SM).
constexpr int kLoopThreads = 1024;
template <bool kTail0>   // DevParams::density_tail0 && DevParams::force_tail0
__global__ void __launch_bounds__(kLoopThreads, 1) k_pci_loop(DevParams P, StepBuffers b, float4* ppos_alt,
                                                             LoopSync* sy, uint32_t* maxerr, int first_done, int warm)
{
    __shared__ float W[kTableSize], SDW[kTableSize], TH[kTableSize + 1], TH2[kTableSize + 1];
    __shared__ float wmax[kLoopThreads / 32];
    stage_table(W, b.tables, T_W);
    stage_table(SDW, b.tables, T_SPIKY_DW);
    stage_table(TH, b.tables, T_THRESH);
    stage_table(TH2, b.tables, T_THRESH2);
    __syncthreads();
    // x* of iteration parity 0 / 1. A select, not a two-pointer array: an array indexed by
    // the iteration lives in local memory, and reading it per particle cost the loop 3.8 %.
    auto pp = [&](int parity) { return parity ? ppos_alt : b.ppos; };
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    // The particles of a pass: full rounds of one contiguous blockDim.x chunk per block,
    // then the partial last round split evenly over all blocks (in whole warps), so that no
    // SM runs a whole extra round while the others wait at the next grid barrier. Every pass
    // maps particles to threads the same way (the bounds are recomputed per pass so that
    // they hold no registers across the loop).
    auto for_particles = [&](auto&& f) {
        const int per_round = (int)(gridDim.x * blockDim.x);
        const int full_end = (P.n / per_round) * per_round;
        const int chunk = ((P.n - full_end + (int)gridDim.x - 1) / (int)gridDim.x + 31) & ~31;
        const int j = full_end + (int)blockIdx.x * chunk + (int)threadIdx.x;
        const int last = ((int)threadIdx.x < chunk && j < P.n) ? j : -1;
        for (int i = tid;; i += per_round) {
            const int q = i < full_end ? i : last;   // past the full rounds: the last-round particle
            if (q < 0) break;
            f(q);
            if (i >= full_end) break;
        }
    };

    // density(k) over all particles; the block maximum of |error| goes to maxerr[slot].
    auto density_pass = [&](int k, int slot) {
        float m = 0.f;
        for_particles([&](int i) { m = fmaxf(m, pci_density_one<kTail0>(P, b, W, TH2, i, k, pp(k & 1))); });
        uint32_t mb = __float_as_uint(m);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mb = max(mb, __shfl_xor_sync(0xffffffffu, mb, off));
        if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = __uint_as_float(mb);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t bm = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) bm = max(bm, __float_as_uint(wmax[w]));
            if (bm) atomicMax(&maxerr[slot], bm);
        }
        __syncthreads();
    };

    int k = 0, kp = 0;
    bool conv = false, rejected = false;
    if (!first_done) {
        for_particles([&](int i) { pci_predict_one(P, b, i, 0, pp(0)); });
        if (!grid_barrier(sy, b.status)) return;
        density_pass(0, 0);
        if (!grid_barrier(sy, b.status)) return;
    }
    for (;;) {
        const float me = __uint_as_float(ld_volatile(&maxerr[kp]));
        if (warm && !rejected && k == 1 && me > __uint_as_float(ld_volatile(&maxerr[kp - 1]))) {
            // The learned guess raised the error: restart from zero pressure (the plain loop).
            rejected = true;
            k = 0;
            kp++;
            for_particles([&](int i) { pci_predict_one(P, b, i, 0, pp(0)); });
            if (!grid_barrier(sy, b.status)) return;
            density_pass(0, kp);
            if (!grid_barrier(sy, b.status)) return;
            continue;
        }
        // PCISPHSolver.cpp:152-162: ratio = max|e| / rho0 in float, exit when below eta.
        const float ratio = me / P.rho0;
        conv = fabsf(ratio) < P.eta;
        // A learned guess is only checked at iteration 1, so a warm step cannot stop at 0.
        const bool unverified = warm && !rejected && k == 0;
        const bool done = (conv && k + 1 >= P.min_it && !unverified) || (k + 1 >= P.max_it);
        for_particles([&](int i) {
            pci_force_one<kTail0>(P, b, SDW, TH, i, pp(k & 1));
            // The last pass also integrates and collides the particle (SPHParticle::integrate
            // after the loop, PCISPHSolver.cpp:166-169): it reads only the particle's own
            // state and pressure force, which this thread has just written, and no thread of
            // this pass reads what it writes (the force pass reads predicted positions).
            if (!done) pci_predict_one(P, b, i, k + 1, pp((k + 1) & 1));
            else integrate_one(P, b, i, 1);
        });
        if (done) break;
        if (!grid_barrier(sy, b.status)) return;
        k++;
        kp++;
        density_pass(k, kp);
        if (!grid_barrier(sy, b.status)) return;
    }
    if (tid == 0) {
        b.status->iterations = kp + 1;
        b.status->converged = conv ? 1 : 0;
        b.status->max_err_bits = ld_volatile(&maxerr[kp]);
        b.status->warm_used = (warm && !rejected) ? 1 : 0;
        b.status->last_k = k;
    }
}

// Per device, instance (kTail0) and block size (1024 / 512 / 256 / 128 threads): resident
// blocks of k_pci_loop per SM (0: no cooperative launch).
constexpr int kMaxDevices = 64;
constexpr int kLoopShapes = 4;
// Filled once per device under a lock (solvers on different host threads may launch at once).
static int g_loop_blocks_per_sm[kMaxDevices][2][kLoopShapes];
static bool g_loop_ready[kMaxDevices];
static std::mutex g_loop_mutex;

// Block size of the loop for n particles: the largest of 1024, 512, 256 and 128 that still
// gives every SM a block (one 1024-thread block per SM is fastest at 1M particles; a
// 12,000-particle scene in blocks of 1024 would run on 12 SMs).
static int loop_shape(int64_t n, int sms)
{
    int k = 0;
    while (k + 1 < kLoopShapes && (n + (kLoopThreads >> k) - 1) / (kLoopThreads >> k) < sms) k++;
    return k;
}

bool launch_pci_loop(const DevParams& P, const StepBuffers& b, float4* ppos_alt, void* sync, uint32_t* maxerr,
                     int first_done, int warm, cudaStream_t s, int* grid_used)
{
    if (grid_used) *grid_used = 0;
    if (P.n <= 0 || P.max_it <= 0) return false;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return false;
    std::unique_lock<std::mutex> lock(g_loop_mutex);
    if (!g_loop_ready[dev]) {
        int coop = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        for (int t = 0; t < 2; t++)
            for (int k = 0; k < kLoopShapes; k++) {
                int per = 0;
                const void* fn = t ? (const void*)k_pci_loop<true> : (const void*)k_pci_loop<false>;
                if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kLoopThreads >> k, 0) !=
                                 cudaSuccess)
                    per = 0;
                g_loop_blocks_per_sm[dev][t][k] = per;
            }
        g_loop_ready[dev] = true;
    }
    const int sms = device_sm_count();
    const int shape = loop_shape(P.n, sms);
    const int threads = kLoopThreads >> shape;
    const int tail0 = (P.density_tail0 && P.force_tail0) ? 1 : 0;
    const int per_sm = g_loop_blocks_per_sm[dev][tail0][shape];
    lock.unlock();
    if (per_sm <= 0) return false;
    int need = (int)((P.n + threads - 1) / threads);
    int grid = std::min(need, per_sm * sms);
    DevParams Pc = P;
    StepBuffers bc = b;
    LoopSync* sy = (LoopSync*)sync;
    void* args[] = {&Pc, &bc, &ppos_alt, &sy, &maxerr, &first_done, &warm};
    const void* fn = tail0 ? (const void*)k_pci_loop<true> : (const void*)k_pci_loop<false>;
    if (cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, 0, s) != cudaSuccess)
        return false;
    if (grid_used) *grid_used = grid;
    return true;
}

// ------------------------------------------------------------------ barrier probe
//
// One grid barrier with `parties` arrivals per round and a short spin limit, for the test
// of the bounded wait: with fewer blocks than parties nothing completes the round, the
// waiting blocks give up, raise kErrTimeout and leave, and the device stays usable.
__global__ void k_barrier_probe(LoopSync* sy, DevStatus* st, uint32_t parties, unsigned long long limit, int* done)
{
    const bool ok = grid_barrier(sy, st, parties, limit);
    if (threadIdx.x == 0 && ok) atomicAdd(done, 1);
}

void barrier_probe(int blocks, int parties, int* completed, uint32_t* error_flags)
{
    struct Probe {
        LoopSync sync;
        DevStatus status;
        int done;
    };
    Probe* d = nullptr;
    cudaStream_t s = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, sizeof(Probe));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, sizeof(Probe), s);
    if (e == cudaSuccess) {
        LoopSync* sy = &d->sync;
        DevStatus* st = &d->status;
        uint32_t np = (uint32_t)parties;
        unsigned long long limit = 1ull << 16;
        int* done = &d->done;
        void* args[] = {&sy, &st, &np, &limit, &done};
        e = cudaLaunchCooperativeKernel((const void*)k_barrier_probe, dim3(blocks), dim3(32), args, 0, s);
    }
    Probe h{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(Probe), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (s) cudaStreamDestroy(s);
    if (d) cudaFree(d);
    if (e != cudaSuccess) throw Error(LSP_ERR_CUDA, std::string("barrier probe: ") + cudaGetErrorString(e));
    *completed = h.done;
    *error_flags = h.status.error_flags;
}

}  // namespace lsp
