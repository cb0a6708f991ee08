// Host-side launch interface of the device kernels (no kernel bodies here).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lsp_device.cuh"

namespace lsp {

struct GridBuildArgs {
    DevParams P;
    const float4* pos_in;
    const float4* vel_in;
    const float4* half_in;
    const float4* old_in;
    float4* pos_out;
    float4* vel_out;
    float4* half_out;
    float4* old_out;
    uint32_t* key;
    uint32_t* slot;
    uint32_t* hist;        // cells + 1 counters, zero on entry, left zero on exit
    uint32_t* tile_sums;
    uint32_t* cell_start;  // cells + 1 entries
    int2* tmp;
    int32_t* slot_of_id;
    uint32_t* sorted_key;
    int32_t* nbr;
    int32_t* nbr_count;
    DevStatus* status;
};

// Per-step particle buffers in device (sorted) order.
struct StepBuffers {
    float4* pos;
    float4* vel;
    float4* half;
    float4* old;
    float4* force;
    float* rho;
    float* pres;
    // PCISPH
    float4* ppos;
    float4* phalf;
    float4* pforce;
    float* prho;
    float* err;
    // neighbours
    const int32_t* nbr;
    const int32_t* nbr_count;
    // tables (5 x 1001) and colliders
    const float* tables;
    const Collider* colliders;
    DevStatus* status;
};

// Both return the number of kernels launched.
int launch_grid_sort(const GridBuildArgs& a, cudaStream_t s);
int launch_neighbors(const GridBuildArgs& a, cudaStream_t s);

void launch_density(const DevParams& P, const StepBuffers& b, cudaStream_t s);
void launch_nonpressure(const DevParams& P, const StepBuffers& b, cudaStream_t s);
void launch_sph_pressure(const DevParams& P, const StepBuffers& b, cudaStream_t s);
void launch_integrate_collide(const DevParams& P, const StepBuffers& b, bool add_pforce, cudaStream_t s);

void launch_pci_predict(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s);
void launch_pci_density(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s);
void launch_pci_force(const DevParams& P, const StepBuffers& b, cudaStream_t s);
// Whole predict-correct loop in one cooperative persistent launch; returns false when the
// device cannot co-schedule the grid (the caller then uses the per-phase launches).
// ppos_alt: second predicted-position buffer; sync: 16 zeroed bytes; maxerr: max_it zeroed words.
bool launch_pci_loop(const DevParams& P, const StepBuffers& b, float4* ppos_alt, void* sync, uint32_t* maxerr,
                     cudaStream_t s, int* grid_used);

// Gathers a per-particle field from device order into caller order.
// comps: 1 (float) or 3 (xyz of a float4); src is float* or float4* accordingly.
void launch_gather_field(const void* src, int comps, int w_as_flag, const int32_t* slot_of_id, float* out,
                         int64_t n, cudaStream_t s);
void launch_gather_count(const int32_t* count, const int32_t* slot_of_id, float* out, int64_t n, cudaStream_t s);
// Scatters caller-order state (x, v, v_half, v_half_old, first) into device slots.
void launch_scatter_state(const float* x, const float* v, const float* half, const float* old,
                          const int32_t* first, const int32_t* slot_of_id, float4* pos, float4* vel,
                          float4* hvel, float4* oldv, int64_t n, cudaStream_t s);
// Writes caller-order x, v, v_half, v_half_old, first from device slots.
void launch_gather_state(const float4* pos, const float4* vel, const float4* hvel, const float4* oldv,
                         const int32_t* slot_of_id, float* x, float* v, float* half, float* old, int32_t* first,
                         int64_t n, cudaStream_t s);
// Neighbour lists in caller order and caller ids.
void launch_neighbor_export(const int32_t* nbr, const int32_t* count, int64_t stride, const float4* pos,
                            const int32_t* slot_of_id, const int64_t* offsets, int32_t* out, int64_t n,
                            cudaStream_t s);
// Axis-aligned bounds of the positions: out[0..2] = min, out[3..5] = max (as ordered ints).
void launch_bounds(const float4* pos, int64_t n, int32_t* out, cudaStream_t s);

}  // namespace lsp
