// Grid-wide barrier of the cooperative persistent kernels (the PCISPH loop of one scene
// and of a batch of scenes). Every block of the grid is resident (cooperative launch).
// The spin is bounded: past the limit it raises kErrTimeout and an abort word that makes
// every block leave, and the host reports LSP_ERR_TIMEOUT.
#pragma once

#include "lsp_device.cuh"

namespace lsp {

constexpr unsigned long long kBarrierSpinLimit = 1ull << 25;

struct LoopSync {
    uint32_t count;   // barrier arrivals since the launch
    uint32_t unused;
    uint32_t abort;
    uint32_t pad;
};

static __device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// Returns false when the loop must stop (a barrier gave up somewhere). The arrival counter
// only grows during a launch (the host clears it before each one): the block that arrives
// as the a-th waits until the counter reaches the next multiple of the number of parties
// (the grid size), so one atomic per block and barrier is all the traffic (measured 1.2 %
// faster loop than a counter reset by the last arrival plus a generation word).
static __device__ bool grid_barrier(LoopSync* sy, DevStatus* st, uint32_t parties = 0,
                                    unsigned long long spin_limit = kBarrierSpinLimit)
{
    if (parties == 0) parties = gridDim.x;
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();
        const uint32_t arrived = atomicAdd(&sy->count, 1u);
        const uint32_t target = (arrived / parties + 1u) * parties;
        unsigned long long spins = 0;
        while ((int)(ld_volatile(&sy->count) - target) < 0) {
            if (ld_volatile(&sy->abort)) { ok = 0; break; }
            if (++spins > spin_limit) {
                atomicExch(&sy->abort, 1u);
                atomicOr(&st->error_flags, kErrTimeout);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        if (ld_volatile(&sy->abort)) ok = 0;
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace lsp
