// Batched scenes: the step's per-particle kernels over many independent scenes at once,
// and the PCISPH loop of every scene in one cooperative persistent launch.
//
// Scene s owns the slots [base_s, base_s + n_s). An item is a run of at most T particles
// of one scene and the per-item kernels run one item per block, so a block stages exactly
// one scene's constants (DevParams) and kernel tables in shared memory, as the single-scene
// kernels do. Every particle runs the same per-particle function (particle_ops.cuh) with
// its scene's constants, so each scene's results are bit-identical to stepping it alone.
//
// The persistent loop (kb_pci_loop) advances all scenes in lockstep rounds:
//
//   decide   every block reads each scene's maximum |error| of its last density pass and
//            applies the single-scene rules (restart after a rejected warm start, converge,
//            stop at max_it); all blocks reach the same decisions
//   phase A  for every active scene: force(k) and predict(k+1), or force(k) alone when it
//            has finished, or predict(0) when it restarts
//   barrier
//   phase B  density(k+1) of every scene that predicted, per-scene maximum |error|
//   barrier
//
// The active items of a phase are split evenly over the blocks (contiguous ranges of the
// per-scene item prefix), so scenes that converge early stop costing time. The loop ends
// when no scene predicted in phase A.
#include "batch_kernels.h"
#include "loop_sync.cuh"
#include "particle_ops.cuh"
#include "warm_ops.cuh"

#include <algorithm>

namespace lsp {

static_assert(sizeof(DevParams) % 4 == 0, "DevParams is staged as 32-bit words");

__device__ __forceinline__ void stage_params(DevParams* sm, const DevParams* sp, int s)
{
    const uint32_t* src = reinterpret_cast<const uint32_t*>(sp + s);
    uint32_t* dst = reinterpret_cast<uint32_t*>(sm);
    for (int w = threadIdx.x; w < (int)(sizeof(DevParams) / 4); w += blockDim.x) dst[w] = src[w];
}

__device__ __forceinline__ const float* scene_tables(const BatchArgs& a, int s)
{
    return a.tables + (size_t)s * kSceneTableStride;
}

// ------------------------------------------------------------------ per-item kernels

template <int T>
__global__ void __launch_bounds__(T) kb_keys(BatchArgs a, const float4* __restrict__ pos, uint32_t* __restrict__ key,
                                             uint32_t* __restrict__ slot, uint32_t* __restrict__ hist)
{
    __shared__ DevParams P;
    const BatchItem it = a.items[blockIdx.x];
    stage_params(&P, a.sp, it.scene);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    const bool valid = i < it.end;
    uint32_t k = 0xffffffffu;
    bool escaped = false, bad = false;
    if (valid) k = cell_key(P, pos[i], escaped, bad);
    const uint32_t sl = hist_slot(k, valid, hist);
    if (valid) {
        key[i] = k;
        slot[i] = sl;
    }
    record_key_flags(valid, escaped, bad, a.st + it.scene);
}

// The lists plus the start-of-step density and pressure (k_neighbors_density in grid.cu),
// per item with the item's scene constants and tables.
template <int T>
__global__ void __launch_bounds__(T) kb_neighbors_density(BatchArgs a, const float4* __restrict__ pos,
                                                          const uint32_t* __restrict__ cell_start,
                                                          int32_t* __restrict__ nbr, int32_t* __restrict__ count,
                                                          float* __restrict__ rho, float* __restrict__ pres,
                                                          const float4* __restrict__ vel, float4* __restrict__ vrho)
{
    __shared__ DevParams P;
    __shared__ float W[kTableSize], TH2[kTableSize + 1];
    const BatchItem it = a.items[blockIdx.x];
    const float* tb = scene_tables(a, it.scene);
    stage_params(&P, a.sp, it.scene);
    stage_table(W, tb, T_W);
    stage_table(TH2, tb, T_THRESH2);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    const bool valid = i < it.end;
    int c = 0;
    if (valid) {
        float sum;
        c = neighbors_one<true>(P, pos, cell_start, nbr, i, W, TH2, &sum);
        count[i] = min(c, P.nbr_cap);
        const float r = P.mass * sum;
        float pr = P.stiffness * (r - P.rho0);
        if (pr < 0.f) pr *= P.neg;
        rho[i] = r;
        pres[i] = pr;
        const float4 v = vel[i];
        vrho[i] = make_float4(v.x, v.y, v.z, r);
        // Batch-wide, like the rest of the non-pressure pass's range checks (k_rank_gather).
        if (!exact_div_density(r)) atomicOr(&a.st[a.scenes].np_unsafe, 1u);
    }
    record_neighbor_count(P, c, valid, a.st + it.scene);
}

template <int T, bool kGrad>
__global__ void __launch_bounds__(T) kb_nonpressure(BatchArgs a, StepBuffers b)
{
    __shared__ DevParams P;
    __shared__ float4 NA[kTableSize], NB[kTableSize];
    const BatchItem it = a.items[blockIdx.x];
    const float* tb = scene_tables(a, it.scene);
    stage_params(&P, a.sp, it.scene);
    stage_nonpressure_slots(NA, NB, tb);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    if (i >= it.end) return;
    nonpressure_one<kGrad>(P, b, NA, NB, i);
}

template <int T>
__global__ void __launch_bounds__(T) kb_sph_pressure(BatchArgs a, StepBuffers b)
{
    __shared__ DevParams P;
    __shared__ float SDW[kTableSize], TH[kTableSize + 1];
    const BatchItem it = a.items[blockIdx.x];
    const float* tb = scene_tables(a, it.scene);
    stage_params(&P, a.sp, it.scene);
    stage_table(SDW, tb, T_SPIKY_DW);
    stage_table(TH, tb, T_THRESH);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    if (i >= it.end) return;
    sph_pressure_one(P, b, SDW, TH, i);
}

template <int T>
__global__ void __launch_bounds__(T) kb_integrate(BatchArgs a, StepBuffers b, int add_pforce)
{
    __shared__ DevParams P;
    const BatchItem it = a.items[blockIdx.x];
    stage_params(&P, a.sp, it.scene);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    if (i >= it.end) return;
    integrate_one(P, b, i, add_pforce);
}

// ------------------------------------------------------------------ learned warm start

template <int T>
__global__ void __launch_bounds__(T) kb_pci_predict0(BatchArgs a, StepBuffers b)
{
    __shared__ DevParams P;
    const BatchItem it = a.items[blockIdx.x];
    stage_params(&P, a.sp, it.scene);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    if (i >= it.end) return;
    pci_predict_one(P, b, i, 0, b.ppos);
}

// Iteration 0's density with the warm-start features (density_first); p_scale = delta *
// 0.01 * rho0 of the item's scene. The scene's maximum |error| goes to
// maxerr[scene * mstride].
template <int T>
__global__ void __launch_bounds__(T) kb_density_first(BatchArgs a, StepBuffers b, BatchWarmArgs w)
{
    __shared__ DevParams P;
    __shared__ float W[kTableSize], TH2[kTableSize + 1];
    const BatchItem it = a.items[blockIdx.x];
    const float* tb = scene_tables(a, it.scene);
    stage_params(&P, a.sp, it.scene);
    stage_table(W, tb, T_W);
    stage_table(TH2, tb, T_THRESH2);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    const float p_scale = P.delta * 0.01f * P.rho0;
    const float e = density_first(P, b, w.feat, b.hist, b.gradrho, p_scale, W, TH2, i, i < it.end);
    uint32_t m = __float_as_uint(e);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(w.maxerr + (size_t)it.scene * w.mstride, m);
}

// Training targets: final pressure / p_scale of the particle's scene.
template <int T>
__global__ void __launch_bounds__(T) kb_targets(BatchArgs a, const float* __restrict__ pres, float* __restrict__ tgt)
{
    __shared__ DevParams P;
    const BatchItem it = a.items[blockIdx.x];
    stage_params(&P, a.sp, it.scene);
    __syncthreads();
    const int i = it.begin + (int)threadIdx.x;
    if (i >= it.end) return;
    const float p_scale = P.delta * 0.01f * P.rho0;
    tgt[i] = pres[i] * (1.f / p_scale);
}

// ------------------------------------------------------------------ persistent loop

enum { ACT_NONE = 0, ACT_RESTART = 1, ACT_STEP = 2, ACT_FINAL = 3 };

// Scene state word: k (bits 0-10), kp (11-21), rejected (22), finished (23), action (24-25).
__device__ __forceinline__ int pack_state(int k, int kp, bool rej, bool fin, int act)
{
    return k | (kp << 11) | ((int)rej << 22) | ((int)fin << 23) | (act << 24);
}
__device__ __forceinline__ int st_k(int w) { return w & 0x7ff; }
__device__ __forceinline__ int st_kp(int w) { return (w >> 11) & 0x7ff; }
__device__ __forceinline__ bool st_rej(int w) { return (w >> 22) & 1; }
__device__ __forceinline__ bool st_fin(int w) { return (w >> 23) & 1; }
__device__ __forceinline__ int st_act(int w) { return (w >> 24) & 3; }

// In-place exclusive scan of a[0..n-1] by one block; a[n] receives the total.
template <int T>
__device__ void block_scan_counts(int* a, int n, int* warp_sums)
{
    const int per = (n + T - 1) / T;
    const int lo = min((int)threadIdx.x * per, n), hi = min(lo + per, n);
    int s = 0;
    for (int q = lo; q < hi; q++) s += a[q];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < T / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < T / 32) warp_sums[lane] = w;
    }
    __syncthreads();
    int run = (warp ? warp_sums[warp - 1] : 0) + x - s;
    for (int q = lo; q < hi; q++) {
        int v = a[q];
        a[q] = run;
        run += v;
    }
    if (threadIdx.x == T - 1) a[n] = warp_sums[T / 32 - 1];
    __syncthreads();
}

template <int T>
// 64 registers (four 256-thread blocks per SM): measured faster than the unconstrained
// allocation (about 112 registers, two blocks per SM) despite a few spilled words.
__global__ void __launch_bounds__(T, 1024 / T) kb_pci_loop(BatchArgs a, StepBuffers b, BatchLoopArgs l)
{
    extern __shared__ int dyn[];
    const int S = a.scenes;
    int* sst = dyn;                // scene state words
    int* sitems = dyn + S;         // items per scene
    int* preA = dyn + 2 * S;       // phase A item prefix (S + 1)
    int* preB = dyn + 3 * S + 1;   // phase B item prefix (S + 1)
    __shared__ DevParams P;
    __shared__ float W[kTableSize], SDW[kTableSize], TH[kTableSize + 1], TH2[kTableSize + 1];
    __shared__ int staged;
    __shared__ int warp_sums[32];
    LoopSync* sy = reinterpret_cast<LoopSync*>(l.sync);
    DevStatus* gst = a.st + S;
    // Predicted positions of iteration k live in buffer k & 1 (selected, not indexed, so the
    // pair stays in registers).
    auto pp = [&](int k) { return (k & 1) ? l.ppos_alt : b.ppos; };

    for (int s = threadIdx.x; s < S; s += T) {
        const int n = a.sp[s].n;
        sitems[s] = (n + T - 1) / T;
        // Without a precomputed iteration 0, every scene starts with predict(0) + density(0).
        sst[s] = pack_state(0, 0, false, false, l.first_done ? ACT_NONE : ACT_RESTART);
        preA[s] = preB[s] = l.first_done ? 0 : sitems[s];
    }
    if (threadIdx.x == 0) staged = -1;
    __syncthreads();
    block_scan_counts<T>(preA, S, warp_sums);
    block_scan_counts<T>(preB, S, warp_sums);

    // Block-uniform: every thread of the block calls it with the same scene.
    auto stage_scene = [&](int s) {
        if (s == staged) return;
        __syncthreads();
        const float* tb = scene_tables(a, s);
        stage_params(&P, a.sp, s);
        stage_table(W, tb, T_W);
        stage_table(SDW, tb, T_SPIKY_DW);
        stage_table(TH, tb, T_THRESH);
        stage_table(TH2, tb, T_THRESH2);
        if (threadIdx.x == 0) staged = s;
        __syncthreads();
    };
    // This block's share of a phase: items [q0, q1) of the prefix `pre` (pre[S] = total).
    auto for_items = [&](const int* pre, auto&& f) {
        const int total = pre[S];
        const int q0 = (int)(((long long)total * blockIdx.x) / gridDim.x);
        const int q1 = (int)(((long long)total * (blockIdx.x + 1)) / gridDim.x);
        if (q0 >= q1) return;
        int lo = 0, hi = S;   // largest s with pre[s] <= q0
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (pre[mid] <= q0) lo = mid; else hi = mid;
        }
        int s = lo;
        for (int q = q0; q < q1; q++) {
            while (q >= pre[s + 1]) s++;
            f(s, q - pre[s]);
        }
    };

    bool first = !l.first_done;
    for (;;) {
        if (!first) {
            // decide: the single-scene loop's rules (pcisph.cu k_pci_loop), per scene.
            for (int s = threadIdx.x; s < S; s += T) {
                const int w = sst[s];
                int k = st_k(w), kp = st_kp(w);
                bool rej = st_rej(w), fin = st_fin(w);
                int act = ACT_NONE;
                if (!fin) {
                    const DevParams* ps = a.sp + s;
                    const uint32_t* me_s = l.maxerr + (size_t)s * l.mstride;
                    const float me = __uint_as_float(ld_volatile(me_s + kp));
                    const bool warm = l.warm && (!l.warm_scene || l.warm_scene[s]);
                    if (warm && !rej && k == 1 && me > __uint_as_float(ld_volatile(me_s + kp - 1))) {
                        rej = true;
                        k = 0;
                        kp++;
                        act = ACT_RESTART;
                    } else {
                        const float ratio = me / ps->rho0;
                        const bool conv = fabsf(ratio) < ps->eta;
                        const bool unverified = warm && !rej && k == 0;
                        const bool done = (conv && k + 1 >= ps->min_it && !unverified) || (k + 1 >= ps->max_it);
                        if (done) {
                            act = ACT_FINAL;
                            fin = true;
                            if (blockIdx.x == 0) {
                                DevStatus* st = a.st + s;
                                st->iterations = kp + 1;
                                st->converged = conv ? 1 : 0;
                                st->max_err_bits = ld_volatile(me_s + kp);
                                st->warm_used = (warm && !rej) ? 1 : 0;
                                st->last_k = k;
                            }
                        } else {
                            act = ACT_STEP;
                            k++;
                            kp++;
                        }
                    }
                }
                sst[s] = pack_state(k, kp, rej, fin, act);
                preA[s] = act != ACT_NONE ? sitems[s] : 0;
                preB[s] = (act == ACT_RESTART || act == ACT_STEP) ? sitems[s] : 0;
            }
            __syncthreads();
            block_scan_counts<T>(preA, S, warp_sums);
            block_scan_counts<T>(preB, S, warp_sums);
        }
        first = false;
        if (preA[S] == 0) break;

        // phase A
        for_items(preA, [&](int s, int j) {
            stage_scene(s);
            const int w = sst[s];
            const int act = st_act(w), k = st_k(w);
            const int i = P.base + j * T + (int)threadIdx.x;
            if (i >= P.base + P.n) return;
            // One call site each for the force walk and the prediction (separate call sites
            // per action spilled 148 bytes; this form 84, batched step 2 % faster). A restart
            // (k = 0) only predicts iteration 0; a step adds force(k - 1) before predict(k);
            // the scene's last pass is force(k), then the integration and collisions (own
            // data only; the scenes never read each other's particles).
            const bool restart = act == ACT_RESTART, last = act == ACT_FINAL;
            if (!restart) pci_force_one(P, b, SDW, TH, i, pp(last ? k : k - 1));
            if (!last) pci_predict_one(P, b, i, k, pp(k));
            else integrate_one(P, b, i, 1);
        });
        if (preB[S] == 0) break;
        if (!grid_barrier(sy, gst)) return;

        // phase B
        for_items(preB, [&](int s, int j) {
            stage_scene(s);
            const int w = sst[s];
            const int k = st_k(w), kp = st_kp(w);
            const int i = P.base + j * T + (int)threadIdx.x;
            float m = 0.f;
            if (i < P.base + P.n) m = pci_density_one(P, b, W, TH2, i, k, pp(k));
            // Max of non-negative floats: their bit patterns order like the values.
            uint32_t mb = __float_as_uint(m);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) mb = max(mb, __shfl_xor_sync(0xffffffffu, mb, off));
            if ((threadIdx.x & 31) == 0 && mb) atomicMax(l.maxerr + (size_t)s * l.mstride + kp, mb);
        });
        if (!grid_barrier(sy, gst)) return;
    }
}

// ------------------------------------------------------------------ launchers

bool batch_threads_supported(int threads)
{
    return threads == 128 || threads == 256 || threads == 512 || threads == 1024;
}

#define LSP_BATCH_DISPATCH(threads, BODY)                                                     \
    switch (threads) {                                                                         \
    case 128: { constexpr int T = 128; BODY; } break;                                         \
    case 256: { constexpr int T = 256; BODY; } break;                                         \
    case 512: { constexpr int T = 512; BODY; } break;                                         \
    case 1024: { constexpr int T = 1024; BODY; } break;                                       \
    default: return 0;                                                                         \
    }

int launch_batch_keys(const BatchArgs& a, const float4* pos, uint32_t* key, uint32_t* slot, uint32_t* hist,
                      cudaStream_t s)
{
    if (!a.items_count) return 0;
    LSP_BATCH_DISPATCH(a.threads, (kb_keys<T><<<a.items_count, T, 0, s>>>(a, pos, key, slot, hist)));
    return 1;
}

int launch_batch_neighbors_density(const BatchArgs& a, const float4* pos, const uint32_t* cell_start, int32_t* nbr,
                                   int32_t* count, float* rho, float* pres, const float4* vel, float4* vrho,
                                   cudaStream_t s)
{
    if (!a.items_count) return 0;
    LSP_BATCH_DISPATCH(a.threads, (kb_neighbors_density<T><<<a.items_count, T, 0, s>>>(a, pos, cell_start, nbr,
                                                                                      count, rho, pres, vel, vrho)));
    return 1;
}

int launch_batch_nonpressure(const BatchArgs& a, const StepBuffers& b, cudaStream_t s)
{
    if (!a.items_count) return 0;
    if (b.gradrho) {
        LSP_BATCH_DISPATCH(a.threads, (kb_nonpressure<T, true><<<a.items_count, T, 0, s>>>(a, b)));
    } else {
        LSP_BATCH_DISPATCH(a.threads, (kb_nonpressure<T, false><<<a.items_count, T, 0, s>>>(a, b)));
    }
    return 1;
}

int launch_batch_sph_pressure(const BatchArgs& a, const StepBuffers& b, cudaStream_t s)
{
    if (!a.items_count) return 0;
    LSP_BATCH_DISPATCH(a.threads, (kb_sph_pressure<T><<<a.items_count, T, 0, s>>>(a, b)));
    return 1;
}

int launch_batch_integrate(const BatchArgs& a, const StepBuffers& b, bool add_pforce, cudaStream_t s)
{
    if (!a.items_count) return 0;
    LSP_BATCH_DISPATCH(a.threads, (kb_integrate<T><<<a.items_count, T, 0, s>>>(a, b, add_pforce ? 1 : 0)));
    return 1;
}

int launch_batch_pci_predict0(const BatchArgs& a, const StepBuffers& b, cudaStream_t s)
{
    if (!a.items_count) return 0;
    LSP_BATCH_DISPATCH(a.threads, (kb_pci_predict0<T><<<a.items_count, T, 0, s>>>(a, b)));
    return 1;
}

int launch_batch_density_first(const BatchArgs& a, const StepBuffers& b, const BatchWarmArgs& w, cudaStream_t s)
{
    if (!a.items_count) return 0;
    LSP_BATCH_DISPATCH(a.threads, (kb_density_first<T><<<a.items_count, T, 0, s>>>(a, b, w)));
    return 1;
}

int launch_batch_targets(const BatchArgs& a, const float* pres, float* tgt, cudaStream_t s)
{
    if (!a.items_count) return 0;
    LSP_BATCH_DISPATCH(a.threads, (kb_targets<T><<<a.items_count, T, 0, s>>>(a, pres, tgt)));
    return 1;
}

static size_t loop_smem(int scenes) { return (size_t)(4 * scenes + 2) * sizeof(int); }

template <int T>
static const void* loop_kernel()
{
    return reinterpret_cast<const void*>(&kb_pci_loop<T>);
}

int batch_loop_max_blocks(int threads, int scenes)
{
    int dev = 0, coop = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (!coop) return 0;
    const void* fn = nullptr;
    switch (threads) {
    case 128: fn = loop_kernel<128>(); break;
    case 256: fn = loop_kernel<256>(); break;
    case 512: fn = loop_kernel<512>(); break;
    case 1024: fn = loop_kernel<1024>(); break;
    default: return 0;
    }
    const size_t smem = loop_smem(scenes);
    if (smem > 48 * 1024) {
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem) != cudaSuccess) return 0;
    return per * sms;
}

bool launch_batch_pci_loop(const BatchArgs& a, const StepBuffers& b, const BatchLoopArgs& l, int grid, cudaStream_t s)
{
    if (a.scenes <= 0 || grid <= 0) return false;
    const void* fn = nullptr;
    switch (a.threads) {
    case 128: fn = loop_kernel<128>(); break;
    case 256: fn = loop_kernel<256>(); break;
    case 512: fn = loop_kernel<512>(); break;
    case 1024: fn = loop_kernel<1024>(); break;
    default: return false;
    }
    BatchArgs ac = a;
    StepBuffers bc = b;
    BatchLoopArgs lc = l;
    void* args[] = {&ac, &bc, &lc};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(a.threads);
    cfg.dynamicSmemBytes = loop_smem(a.scenes);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args) == cudaSuccess;
}

}  // namespace lsp
