// Grid-wide barrier of the cooperative persistent kernels (the PCISPH loop of one scene
// and of a batch of scenes). Every block of the grid is resident (cooperative launch).
// The spin is bounded: past the limit it raises kErrTimeout and an abort word that makes
// every block leave, and the host reports LSP_ERR_TIMEOUT.
#pragma once

#include "lsp_device.cuh"

namespace lsp {

constexpr unsigned long long kBarrierSpinLimit = 1ull << 25;

struct LoopSync {
    uint32_t count;
    uint32_t gen;
    uint32_t abort;
    uint32_t pad;
};

static __device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// Returns false when the loop must stop (a barrier gave up somewhere).
static __device__ bool grid_barrier(LoopSync* sy, DevStatus* st)
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

}  // namespace lsp
