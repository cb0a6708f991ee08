// lsp_mlp_gradient_static: the warm-start MLP's loss gradient on caller-supplied device
// buffers, with no device memory allocated by the call.
//
// Who needs it: callers that are not allowed to allocate device memory while they run.
// A training loop embedded in another framework that owns the GPU's memory through its
// own pool (a cudaMalloc from here would bypass and fragment that pool), code that runs
// between the points where a host application is allowed to allocate, or a process with
// a hard device-memory budget, can still compute gradients: they hand over inputs and
// outputs they already own, and the per-warp partial sums go to a fixed scratch array
// that lives in this library's module for the lifetime of the process.
//
// Limits: the kernel runs on a fixed grid of kStaticBlocks blocks (one partial row per
// warp), so the scratch is kStaticRows * (1377 + 1) floats = 2.7 MiB on every device
// that loads the library; batches larger than kStaticMaxBatch particles are refused.
// Every call shares that one array: calls that overlap on the GPU (two streams, two
// solvers on the same device) race and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/lsp.h"
#include "lsp_handle.h"
#include "lsp_kernels.h"
#include "mlp.cuh"

namespace lsp {
namespace {

constexpr int kStaticBlocks = 64;
constexpr int kStaticRows = kStaticBlocks * 8;              // one row per warp of 256-thread blocks
constexpr int64_t kStaticMaxBatch = int64_t(1) << 24;        // 16,777,216 particles
constexpr int kMaxDevices = 64;

// Per-warp partial gradients (kStaticRows x kMlpParams) followed by per-warp losses.
static __device__ __align__(256) float g_static_grad_scratch[kStaticRows * kMlpParams + kStaticRows];

}  // namespace

// Device address of the scratch array, looked up once per device with that device current:
// in host code the array's name is only a host-side stand-in, never a device address.
// lsp_create calls it for the solver's device, so the lookup (and the loading of this
// file's module with the array, which CUDA's lazy module loading defers to the first use of
// a symbol) happens when the solver is created, not inside lsp_mlp_gradient_static.
float* scratch_on(int device)
{
    static std::mutex mu;
    static float* addr[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) throw Error(LSP_ERR_NO_DEVICE, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        int current = -1;
        cudaGetDevice(&current);
        if (current != device) throw Error(LSP_ERR_STATE, "scratch set-up needs the solver's device current");
        float* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_static_grad_scratch);
        if (e != cudaSuccess || !p)
            throw Error(LSP_ERR_CUDA, std::string("cudaGetSymbolAddress of the gradient scratch: ") +
                                          cudaGetErrorString(e));
        addr[device] = p;
    }
    return addr[device];
}

namespace {

// Sums the partial rows in a fixed order: grad[p] = sum_r partial[r][p], loss = sum_r loss[r] / n.
__global__ void k_static_reduce(const float* __restrict__ scratch, int rows, float inv_n, float* __restrict__ grad,
                                float* __restrict__ loss)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const float* loss_part = scratch + (int64_t)rows * kMlpParams;
    if (p == 0) {
        float l = 0.f;
        for (int r = 0; r < rows; r++) l += loss_part[r];
        *loss = l * inv_n;
    }
    if (p >= kMlpParams) return;
    float g = 0.f;
    for (int r = 0; r < rows; r++) g += scratch[(int64_t)r * kMlpParams + p];
    grad[p] = g;
}

// Device memory of `device` itself, or managed memory (reachable from every device). Memory
// of another GPU is refused: the kernels would read it from this device, which faults without
// peer access and crosses NVLink silently with it.
bool on_device(const void* p, int device)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

}  // namespace
}  // namespace lsp

extern "C" int lsp_mlp_gradient_static(lsp_solver* s, const float* features, const float* targets, int64_t n,
                                       float* grad, float* loss)
{
    try {
        if (!s || !s->e) throw lsp::Error(LSP_ERR_INVALID, "null solver handle");
        if (!features || !targets || !grad || !loss) throw lsp::Error(LSP_ERR_INVALID, "null buffer");
        if (n <= 0) throw lsp::Error(LSP_ERR_INVALID, "n must be > 0");
        if (n > lsp::kStaticMaxBatch)
            throw lsp::Error(LSP_ERR_CAPACITY, "lsp_mlp_gradient_static takes at most 16777216 particles per call "
                                               "(fixed scratch); split the batch or use lsp_mlp_gradient");
        lsp::Engine& e = *s->e;
        if (cudaSetDevice(e.device()) != cudaSuccess) throw lsp::Error(LSP_ERR_CUDA, "cudaSetDevice failed");
        for (const void* p : {(const void*)features, (const void*)targets, (const void*)grad, (const void*)loss})
            if (!lsp::on_device(p, e.device()))
                throw lsp::Error(LSP_ERR_INVALID, "buffers must be device memory of the solver's GPU");
        float* scratch = lsp::scratch_on(e.device());
        cudaStream_t st = e.stream();
        // Every partial row and loss slot the reduction reads is written by this launch
        // first, so nothing in the scratch has to be cleared between calls.
        lsp::launch_mlp_grad_blocks(reinterpret_cast<const lsp::MlpPacked*>(e.mlp_packed_device()), features,
                                    targets, (int)n, lsp::kStaticBlocks, scratch,
                                    scratch + (int64_t)lsp::kStaticRows * lsp::kMlpParams, st);
        lsp::k_static_reduce<<<(lsp::kMlpParams + 255) / 256, 256, 0, st>>>(scratch, lsp::kStaticRows,
                                                                          1.f / (float)n, grad, loss);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) throw lsp::Error(LSP_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(err));
        return LSP_OK;
    } catch (const lsp::Error& x) {
        lsp::set_last_error(x.what());
        return x.code;
    } catch (const std::exception& x) {
        lsp::set_last_error(x.what());
        return LSP_ERR_INVALID;
    }
}
