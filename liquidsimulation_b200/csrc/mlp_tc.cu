// tcgen05 inference of the warm-start network (mlp_tc.cuh).
#include "mlp_tc.cuh"
#include "batch_kernels.h"

namespace lsp {

// ------------------------------------------------------------------ tcgen05 / mbarrier

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address, leading / stride byte offsets (all >> 4),
// descriptor version 1 (bits 46-47), no swizzle (layout type 0, bits 61-63).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B
// (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(dst_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, one UMMA issued by the calling thread.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// Arrives on the mbarrier once every UMMA the thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint64_t* mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_addr(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(mbar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Bounded wait for the phase with the given parity; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity)
{
    const uint32_t a = smem_addr(mbar);
    for (uint32_t spin = 0; spin < kTcSpinLimit; spin++) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 32 consecutive accumulator columns of this warp's 32 rows: thread t gets row 32 w + t.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int c = 0; c < 32; c++) v[c] = __uint_as_float(r[c]);
}

__device__ __forceinline__ uint16_t bf16_of(float x)
{
    __nv_bfloat16 b = __float2bfloat16_rn(x);
    return *reinterpret_cast<uint16_t*>(&b);
}

// ------------------------------------------------------------------ kernels

__global__ void k_mlp_pack_umma(const float* __restrict__ m, MlpUmma* __restrict__ out)
{
    const float* W1 = m + kOffW1;   // W1[i][j]: input i, output j
    const float* W2 = m + kOffW2;   // W2[k][n]
    for (int idx = threadIdx.x; idx < 32 * 16; idx += blockDim.x) {
        const int n = idx / 16, k = idx % 16;
        out->w1t[umma_kmajor_offset(n, k, 256) / 2] = k < kMlpIn ? bf16_of(W1[k * 32 + n]) : (uint16_t)0;
    }
    for (int idx = threadIdx.x; idx < 32 * 32; idx += blockDim.x) {
        const int n = idx / 32, k = idx % 32;
        out->w2t[umma_kmajor_offset(n, k, 512) / 2] = bf16_of(W2[k * 32 + n]);
    }
    for (int c = threadIdx.x; c < 32; c += blockDim.x) {
        out->b1[c] = m[kOffB1 + c];
        out->b2[c] = m[kOffB2 + c];
        out->w3[c] = bf16_round(m[kOffW3 + c]);
    }
    if (threadIdx.x == 0) {
        out->b3 = m[kOffB3];
        out->pad[0] = out->pad[1] = out->pad[2] = 0.f;
    }
}

// Per-block state of the tensor-core evaluation: shared operand tiles, the staged weights,
// the accumulator mbarrier and the tensor-memory columns.
struct TcShared {
    __align__(128) uint16_t a1[kTcRows * 16];   // layer-1 A: [128][16] BF16
    __align__(128) uint16_t a2[kTcRows * 32];   // layer-2 A: [128][32] BF16
    __align__(128) MlpUmma w;
    __align__(8) uint64_t mbar;
    uint32_t tmem;
};

// Stages the weights, allocates the accumulators (warp 0) and initialises the mbarrier.
__device__ __forceinline__ void tc_begin(TcShared& sh, const MlpUmma* wg)
{
    const int tid = threadIdx.x;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(wg);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sh.w);
    for (int q = tid; q < (int)(sizeof(MlpUmma) / 4); q += kTcRows) dst[q] = src[q];
    if ((tid >> 5) == 0) tmem_alloc(&sh.tmem, kTcCols);
    if (tid == 0) mbar_init(&sh.mbar, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// Frees the accumulators once every thread has finished reading them.
__device__ __forceinline__ void tc_end(TcShared& sh)
{
    tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc_fence_after();
        tmem_dealloc(sh.tmem, kTcCols);
    }
}

// The network for one tile of 128 rows; every thread of the block calls it with its row's
// features and gets its row's output. parity: the mbarrier phase, advanced twice; ok is
// cleared if an accumulator wait gave up.
__device__ __forceinline__ float tc_tile(TcShared& sh, const float (&f)[kMlpIn], uint32_t& parity, bool& ok)
{
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t row_lane = (uint32_t)(warp * 32) << 16;   // this warp's lane quarter
    const uint32_t idesc = umma_idesc_bf16(kTcRows, 32);
    const uint32_t a1 = smem_addr(sh.a1), a2 = smem_addr(sh.a2);
    const uint32_t b1 = smem_addr(sh.w.w1t), b2 = smem_addr(sh.w.w2t);
    // Layer-1 A row: 8 BF16 features, 8 zeros (K padded to 16).
    *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sh.a1) + umma_kmajor_offset(tid, 0, 256)) =
        make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
    *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sh.a1) + umma_kmajor_offset(tid, 8, 256)) =
        make_uint4(0u, 0u, 0u, 0u);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
        umma_bf16(sh.tmem, umma_desc(a1, 128, 256), umma_desc(b1, 128, 256), idesc, 0u);
        umma_commit(&sh.mbar);
    }
    ok &= mbar_wait(&sh.mbar, parity);
    parity ^= 1u;
    tc_fence_after();
    float z[32];
    tmem_ld32(sh.tmem + row_lane, z);
    // Hidden layer 1 -> layer-2 A row (BF16, K = 32).
#pragma unroll
    for (int c = 0; c < 4; c++) {
        uint32_t q[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int k = 8 * c + 2 * e;
            q[e] = pack_bf16(silu(z[k] + sh.w.b1[k]), silu(z[k + 1] + sh.w.b1[k + 1]));
        }
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sh.a2) + umma_kmajor_offset(tid, 8 * c, 512)) =
            make_uint4(q[0], q[1], q[2], q[3]);
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
        tc_fence_after();
        umma_bf16(sh.tmem + 32, umma_desc(a2, 128, 512), umma_desc(b2, 128, 512), idesc, 0u);
        umma_bf16(sh.tmem + 32, umma_desc(a2 + 256, 128, 512), umma_desc(b2 + 256, 128, 512), idesc, 1u);
        umma_commit(&sh.mbar);
    }
    ok &= mbar_wait(&sh.mbar, parity);
    parity ^= 1u;
    tc_fence_after();
    tmem_ld32(sh.tmem + row_lane + 32, z);
    float y = 0.f;
#pragma unroll
    for (int k = 0; k < 32; k++) y += bf16_round(silu(z[k] + sh.w.b2[k])) * sh.w.w3[k];
    y += sh.w.b3;
    tc_fence_before();
    __syncthreads();   // the next tile rewrites the A tiles and the accumulators
    return y;
}

__device__ __forceinline__ void load_features(const float* feat, int64_t i, bool valid, float (&f)[kMlpIn])
{
    if (valid) {
        const float4 lo = *reinterpret_cast<const float4*>(feat + i * kMlpIn);
        const float4 hi = *reinterpret_cast<const float4*>(feat + i * kMlpIn + 4);
        f[0] = lo.x; f[1] = lo.y; f[2] = lo.z; f[3] = lo.w;
        f[4] = hi.x; f[5] = hi.y; f[6] = hi.z; f[7] = hi.w;
    } else {
#pragma unroll
        for (int c = 0; c < kMlpIn; c++) f[c] = 0.f;
    }
}

// The guess replaces iteration 0's pressure correction: p = y * p_scale (clamped at zero
// when negative pressure is switched off), and the force factor p / rho*^2 in x*.w, as the
// fused iteration-0 pass would store them (warm_ops.cuh).
__device__ __forceinline__ void store_guess(const DevParams& P, const StepBuffers& b, int i, float y, float p_scale)
{
    float p = y * p_scale;
    if (P.neg == 0.f && p < 0.f) p = 0.f;
    const float pd = b.prho[i];
    b.pres[i] = p;
    reinterpret_cast<float*>(b.ppos + i)[3] = p / (pd * pd);
}

// features[n][8] -> out[n] (lsp_mlp_forward). Tiles of 128 rows in a grid-stride loop.
__global__ void __launch_bounds__(kTcRows) k_mlp_forward_tc(const MlpUmma* __restrict__ wg,
                                                           const float* __restrict__ feat, float* __restrict__ out,
                                                           int n, uint32_t* err)
{
    __shared__ TcShared sh;
    tc_begin(sh, wg);
    uint32_t parity = 0;
    bool ok = true;
    for (int tile = blockIdx.x; (int64_t)tile * kTcRows < n; tile += gridDim.x) {
        const int i = tile * kTcRows + (int)threadIdx.x;
        float f[kMlpIn];
        load_features(feat, i, i < n, f);
        const float y = tc_tile(sh, f, parity, ok);
        if (i < n) out[i] = y;
    }
    if (!ok && err && threadIdx.x == 0) atomicOr(err, 1u);
    tc_end(sh);
}

// Warm-start guess of one scene: rows [0, P.n), features from iteration 0's density pass.
__global__ void __launch_bounds__(kTcRows) k_warm_guess_tc(const MlpUmma* __restrict__ wg, DevParams P,
                                                          StepBuffers b, const float* __restrict__ feat)
{
    __shared__ TcShared sh;
    tc_begin(sh, wg);
    const float p_scale = P.delta * 0.01f * P.rho0;
    uint32_t parity = 0;
    bool ok = true;
    for (int tile = blockIdx.x; (int64_t)tile * kTcRows < P.n; tile += gridDim.x) {
        const int i = tile * kTcRows + (int)threadIdx.x;
        float f[kMlpIn];
        load_features(feat, i, i < P.n, f);
        const float y = tc_tile(sh, f, parity, ok);
        if (i < P.n) store_guess(P, b, i, y, p_scale);
    }
    if (!ok && threadIdx.x == 0) atomicOr(&b.status->error_flags, kErrTimeout);
    tc_end(sh);
}

// Warm-start guess of a batch: block k evaluates item k (one scene) in tiles of 128 rows.
__global__ void __launch_bounds__(kTcRows) kb_warm_guess_tc(const MlpUmma* __restrict__ wg,
                                                           const DevParams* __restrict__ sp,
                                                           const BatchItem* __restrict__ items, StepBuffers b,
                                                           const float* __restrict__ feat,
                                                           const int32_t* __restrict__ warm_scene, DevStatus* st)
{
    __shared__ TcShared sh;
    const BatchItem it = items[blockIdx.x];
    if (warm_scene && !warm_scene[it.scene]) return;   // block-uniform: one scene per item
    tc_begin(sh, wg);
    const DevParams& P = sp[it.scene];
    const float p_scale = P.delta * 0.01f * P.rho0;
    uint32_t parity = 0;
    bool ok = true;
    for (int base = it.begin; base < it.end; base += kTcRows) {
        const int i = base + (int)threadIdx.x;
        float f[kMlpIn];
        load_features(feat, i, i < it.end, f);
        const float y = tc_tile(sh, f, parity, ok);
        if (i < it.end) store_guess(P, b, i, y, p_scale);
    }
    if (!ok && threadIdx.x == 0) atomicOr(&st->error_flags, kErrTimeout);
    tc_end(sh);
}

void launch_mlp_pack_umma(const float* master, MlpUmma* out, cudaStream_t s)
{
    k_mlp_pack_umma<<<1, 256, 0, s>>>(master, out);
}

void launch_mlp_forward_tc(const MlpUmma* w, const float* feat, float* out, int n, uint32_t* err, cudaStream_t s)
{
    if (n <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (n + kTcRows - 1) / kTcRows;
    const int blocks = tiles < 4 * sms ? tiles : 4 * sms;
    // Padding shared memory so that at most 7 blocks share an SM: 7 x 64 tensor-memory
    // columns fit in the SM's 512, so no block waits in tcgen05.alloc.
    k_mlp_forward_tc<<<blocks, kTcRows, kTcSmemPad, s>>>(w, feat, out, n, err);
}

void launch_warm_guess_tc(const MlpUmma* w, const DevParams& P, const StepBuffers& b, const float* feat,
                          cudaStream_t s)
{
    if (P.n <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (P.n + kTcRows - 1) / kTcRows;
    const int blocks = tiles < 4 * sms ? tiles : 4 * sms;
    k_warm_guess_tc<<<blocks, kTcRows, kTcSmemPad, s>>>(w, P, b, feat);
}

void launch_batch_warm_guess_tc(const MlpUmma* w, const DevParams* sp, const BatchItem* items, int items_count,
                                const StepBuffers& b, const float* feat, const int32_t* warm_scene, DevStatus* st,
                                cudaStream_t s)
{
    if (items_count <= 0) return;
    kb_warm_guess_tc<<<items_count, kTcRows, kTcSmemPad, s>>>(w, sp, items, b, feat, warm_scene, st);
}

}  // namespace lsp
