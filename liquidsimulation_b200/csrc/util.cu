// Caller-order read-back and write-back: the device keeps particles sorted by cell and
// slot_of_id[id] tells where caller particle `id` sits. These kernels replace the
// reference's blocking sorted read-back (SPHSolver::onEndUpdate, SPHSolver.cpp:400-427)
// and its full re-upload on change (SPHSolver::initParallelBuffers, :791-886).
#include "lsp_device.cuh"
#include "lsp_kernels.h"

#include <atomic>

namespace lsp {

constexpr int kThreads = 256;
static inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__global__ void k_gather_vec(const float4* __restrict__ src, const int32_t* __restrict__ slot_of_id,
                             float* __restrict__ out, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    float4 v = src[slot_of_id[id]];
    out[3 * id] = v.x;
    out[3 * id + 1] = v.y;
    out[3 * id + 2] = v.z;
}

__global__ void k_gather_w(const float4* __restrict__ src, const int32_t* __restrict__ slot_of_id,
                           float* __restrict__ out, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    out[id] = src[slot_of_id[id]].w;
}

__global__ void k_gather_sqlen(const float4* __restrict__ src, const int32_t* __restrict__ slot_of_id,
                               float* __restrict__ out, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    out[id] = sqmag(v3(src[slot_of_id[id]]));
}

__global__ void k_gather_scalar(const float* __restrict__ src, const int32_t* __restrict__ slot_of_id,
                                float* __restrict__ out, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    out[id] = src[slot_of_id[id]];
}

__global__ void k_gather_count(const int32_t* __restrict__ count, const int32_t* __restrict__ slot_of_id,
                               float* __restrict__ out, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    out[id] = (float)count[slot_of_id[id]];
}

void launch_gather_field(const void* src, int comps, int mode, const int32_t* slot_of_id, float* out, int64_t n,
                         cudaStream_t s)
{
    if (!n) return;
    if (comps == 3)
        k_gather_vec<<<blocks_for(n), kThreads, 0, s>>>((const float4*)src, slot_of_id, out, n);
    else if (mode == 1)
        k_gather_w<<<blocks_for(n), kThreads, 0, s>>>((const float4*)src, slot_of_id, out, n);
    else if (mode == 2)
        k_gather_sqlen<<<blocks_for(n), kThreads, 0, s>>>((const float4*)src, slot_of_id, out, n);
    else
        k_gather_scalar<<<blocks_for(n), kThreads, 0, s>>>((const float*)src, slot_of_id, out, n);
}

void launch_gather_count(const int32_t* count, const int32_t* slot_of_id, float* out, int64_t n, cudaStream_t s)
{
    if (n) k_gather_count<<<blocks_for(n), kThreads, 0, s>>>(count, slot_of_id, out, n);
}

__global__ void k_scatter_state(const float* __restrict__ x, const float* __restrict__ v,
                                const float* __restrict__ h, const float* __restrict__ o,
                                const int32_t* __restrict__ first, const int32_t* __restrict__ slot_of_id,
                                float4* pos, float4* vel, float4* hv, float4* ov, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    int32_t s = slot_of_id[id];
    pos[s] = make_float4(x[3 * id], x[3 * id + 1], x[3 * id + 2], __int_as_float((int)id));
    vel[s] = make_float4(v[3 * id], v[3 * id + 1], v[3 * id + 2], first[id] ? 1.f : 0.f);
    float4 a = hv[s], b = ov[s];
    hv[s] = make_float4(h[3 * id], h[3 * id + 1], h[3 * id + 2], a.w);
    ov[s] = make_float4(o[3 * id], o[3 * id + 1], o[3 * id + 2], b.w);
}

void launch_scatter_state(const float* x, const float* v, const float* half, const float* old, const int32_t* first,
                          const int32_t* slot_of_id, float4* pos, float4* vel, float4* hvel, float4* oldv,
                          int64_t n, cudaStream_t s)
{
    if (n) k_scatter_state<<<blocks_for(n), kThreads, 0, s>>>(x, v, half, old, first, slot_of_id, pos, vel, hvel,
                                                               oldv, n);
}

__global__ void k_scatter_vec(const float* __restrict__ in, const int32_t* __restrict__ slot_of_id,
                              float4* __restrict__ dst, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    dst[slot_of_id[id]] = make_float4(in[3 * id], in[3 * id + 1], in[3 * id + 2], 0.f);
}

void launch_scatter_vec(const float* in, const int32_t* slot_of_id, float4* dst, int64_t n, cudaStream_t s)
{
    if (n) k_scatter_vec<<<blocks_for(n), kThreads, 0, s>>>(in, slot_of_id, dst, n);
}

__global__ void k_gather_state(const float4* __restrict__ pos, const float4* __restrict__ vel,
                               const float4* __restrict__ hv, const float4* __restrict__ ov,
                               const int32_t* __restrict__ slot_of_id, float* x, float* v, float* h, float* o,
                               int32_t* first, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    int32_t s = slot_of_id[id];
    float4 a = pos[s], b = vel[s], c = hv[s], d = ov[s];
    x[3 * id] = a.x; x[3 * id + 1] = a.y; x[3 * id + 2] = a.z;
    v[3 * id] = b.x; v[3 * id + 1] = b.y; v[3 * id + 2] = b.z;
    h[3 * id] = c.x; h[3 * id + 1] = c.y; h[3 * id + 2] = c.z;
    o[3 * id] = d.x; o[3 * id + 1] = d.y; o[3 * id + 2] = d.z;
    first[id] = b.w != 0.f ? 1 : 0;
}

void launch_gather_state(const float4* pos, const float4* vel, const float4* hvel, const float4* oldv,
                         const int32_t* slot_of_id, float* x, float* v, float* half, float* old, int32_t* first,
                         int64_t n, cudaStream_t s)
{
    if (n) k_gather_state<<<blocks_for(n), kThreads, 0, s>>>(pos, vel, hvel, oldv, slot_of_id, x, v, half, old,
                                                              first, n);
}

__global__ void k_neighbor_export(const int32_t* __restrict__ nbr, const int32_t* __restrict__ count, int64_t stride,
                                  const float4* __restrict__ pos, const int32_t* __restrict__ slot_of_id,
                                  const int64_t* __restrict__ offsets, int32_t* __restrict__ out, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    int32_t s = slot_of_id[id];
    int c = count[s];
    int64_t o = offsets[id];
    for (int e = 0; e < c; e++) out[o + e] = id_of(pos[list_entry(nbr, stride, s, e)]);
}

void launch_neighbor_export(const int32_t* nbr, const int32_t* count, int64_t stride, const float4* pos,
                            const int32_t* slot_of_id, const int64_t* offsets, int32_t* out, int64_t n,
                            cudaStream_t s)
{
    if (n) k_neighbor_export<<<blocks_for(n), kThreads, 0, s>>>(nbr, count, stride, pos, slot_of_id, offsets, out, n);
}

__global__ void k_scale(const float* __restrict__ src, float* __restrict__ dst, int64_t n, float f)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i] * f;
}

void launch_scale(const float* src, float* dst, int64_t n, float factor, cudaStream_t s)
{
    if (n) k_scale<<<blocks_for(n), kThreads, 0, s>>>(src, dst, n, factor);
}

__global__ void k_gather_rows(const float* __restrict__ src, int width, const int32_t* __restrict__ slot_of_id,
                              float* __restrict__ out, int64_t n)
{
    const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const int64_t s = slot_of_id[id];
    for (int c = 0; c < width; c++) out[id * width + c] = src[s * width + c];
}

void launch_gather_rows(const float* src, int width, const int32_t* slot_of_id, float* out, int64_t n, cudaStream_t s)
{
    if (n) k_gather_rows<<<blocks_for(n), kThreads, 0, s>>>(src, width, slot_of_id, out, n);
}

// Float min/max through order-preserving integer images (atomicMin/Max on ints).
__device__ __forceinline__ int32_t ordered(float f)
{
    int32_t i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}

__global__ void k_bounds(const float4* __restrict__ pos, int64_t n, int32_t* out)
{
    int32_t lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float4 p = pos[i];
        float c[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (!isfinite(c[a])) continue;
            int32_t o = ordered(c[a]);
            lo[a] = min(lo[a], o);
            hi[a] = max(hi[a], o);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        for (int off = 16; off > 0; off >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; a++) {
            atomicMin(&out[a], lo[a]);
            atomicMax(&out[3 + a], hi[a]);
        }
    }
}

void launch_bounds(const float4* pos, int64_t n, int32_t* out, cudaStream_t s)
{
    if (n) k_bounds<<<148 * 4, kThreads, 0, s>>>(pos, n, out);
}

int device_sm_count()
{
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cached[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        v = sms > 0 ? sms : 148;
        cached[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

}  // namespace lsp
