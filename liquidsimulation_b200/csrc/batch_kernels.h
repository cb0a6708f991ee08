// Host-side launch interface of the batched-scene kernels (batch.cu).
//
// A batch holds many independent scenes in one set of particle arrays: scene s owns the
// slots [base_s, base_s + n_s) in every step (the sort keys of different scenes never
// mix, because each scene's cells occupy their own range of the batch's cell table), so
// the per-particle kernels run over "items": runs of at most `threads` particles of one
// scene, one item per block. Per-scene constants (DevParams, kernel tables, colliders)
// are arrays in device memory, so a captured CUDA graph of the step stays valid when dt
// or a collider changes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lsp_kernels.h"

namespace lsp {

constexpr int kMaxBatchScenes = 4096;
// Per-scene kernel tables: the single-scene table block (5 tables of kTableSize, the slot
// thresholds on d and on d^2), padded to a multiple of 64 floats.
constexpr int kSceneTableFloats = kTableFloats;
constexpr int kSceneTableStride = (kSceneTableFloats + 63) / 64 * 64;

struct BatchItem {
    int scene;
    int begin;   // first slot
    int end;     // one past the last slot
    int pad;
};

struct BatchArgs {
    const DevParams* sp;     // [scenes]
    const float* tables;     // [scenes][kSceneTableStride]
    const BatchItem* items;  // [items]
    int items_count;
    int scenes;
    int threads;             // particles per item = threads per block of the per-item kernels
    DevStatus* st;           // [scenes + 1]; the last one holds batch-wide errors
};

// Supported item sizes (threads per block of the per-item kernels).
bool batch_threads_supported(int threads);

int launch_batch_keys(const BatchArgs& a, const float4* pos, uint32_t* key, uint32_t* slot, uint32_t* hist,
                      cudaStream_t s);
// Lists plus the start-of-step density and pressure (rho, pres), per item.
int launch_batch_neighbors_density(const BatchArgs& a, const float4* pos, const uint32_t* cell_start, int32_t* nbr,
                                   int32_t* count, float* rho, float* pres, const float4* vel, float4* vrho,
                                   cudaStream_t s);
int launch_batch_nonpressure(const BatchArgs& a, const StepBuffers& b, cudaStream_t s);
int launch_batch_sph_pressure(const BatchArgs& a, const StepBuffers& b, cudaStream_t s);
int launch_batch_integrate(const BatchArgs& a, const StepBuffers& b, bool add_pforce, cudaStream_t s);

// Learned warm start of a batch: iteration 0's predict, then its density pass with the
// features (b.hist, b.gradrho); per-scene maximum |error| to maxerr[scene * mstride].
// Training targets p / p_scale per scene. (The network's guess: mlp_tc.cuh.)
struct BatchWarmArgs {
    float* feat;             // [n][8] features, written
    uint32_t* maxerr;
    int mstride;
};
int launch_batch_pci_predict0(const BatchArgs& a, const StepBuffers& b, cudaStream_t s);
int launch_batch_density_first(const BatchArgs& a, const StepBuffers& b, const BatchWarmArgs& w, cudaStream_t s);
int launch_batch_targets(const BatchArgs& a, const float* pres, float* tgt, cudaStream_t s);

// The PCISPH loop of every scene in one cooperative launch of `grid` blocks of a.threads
// threads (grid <= batch_loop_max_blocks). Scenes iterate in lockstep rounds separated by
// grid barriers, each with its own iteration count, convergence test and warm-start check.
// sync: 16 zeroed bytes; maxerr: [scenes][mstride] zeroed words (mstride >= max_it + 2).
struct BatchLoopArgs {
    float4* ppos_alt;
    void* sync;
    uint32_t* maxerr;
    int mstride;
    int first_done;
    int warm;
    const int32_t* warm_scene;   // per-scene use of the guess (LSP_WARM_AUTO); null: every scene
};
// Blocks of a.threads threads that can be co-resident (0: no cooperative launch).
int batch_loop_max_blocks(int threads, int scenes);
bool launch_batch_pci_loop(const BatchArgs& a, const StepBuffers& b, const BatchLoopArgs& l, int grid,
                           cudaStream_t s);

}  // namespace lsp
