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
    const float4* hist_in;   // optional fifth persistent array (warm-start history)
    float4* hist_out;
    int32_t* nbr;
    int32_t* nbr_count;
    DevStatus* status;
    // The start-of-step density is computed in the neighbour build (rho, p written;
    // tables = the kernel table block).
    const float* tables;
    float* rho;
    float* pres;
    float4* vrho;          // {v, rho} per particle for the non-pressure pass's gathers
};

struct MlpPacked;

// Learned warm start inputs (device order). Features of particle i: feat[8*i .. 8*i+7].
struct WarmArgs {
    float* feat;            // written when non-null (recording or warm start)
    const float4* hist;     // (p_{n-1}, p_{n-2}, p_{n-3}, -) per particle
    const float* gradrho;   // |grad rho| from the non-pressure pass
    float p_scale;          // pressure of one correction at 1 % density error: delta * 0.01 * rho0
    uint32_t* maxerr0;      // max |error| of iteration 0 (float bits)
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
    float4* hist;             // warm-start pressure history, null when off
    float* gradrho;           // |grad rho|, null when off
    // neighbours: the lists in list_entry's grouped layout (nbr), read by every walk after
    // the non-pressure pass. The neighbour build writes them plain column-major (nbr_src,
    // entry k of particle i at nbr_src[k * stride + i]: one 4-byte store per entry, the
    // cheapest for its accept branch), and the non-pressure pass, which walks every list
    // first, regroups them into nbr_out (the same memory as nbr) with 16-byte stores.
    const int32_t* nbr;
    const int32_t* nbr_count;
    const int32_t* nbr_src;
    int32_t* nbr_out;
    // {v.x, v.y, v.z, rho} of each particle, written by the neighbour build once rho is known:
    // the non-pressure pass gathers a neighbour's velocity and density with one 16-byte load.
    const float4* vrho;
    // tables (5 x 1001) and colliders
    const float* tables;
    const Collider* colliders;
    DevStatus* status;
};

// Entries of the histogram and cell-table buffers for `n` live entries: the scan moves them
// 8 at a time, so both are padded to a multiple of 8 (the padding stays zero); and the scan's
// tiles of 2048 entries.
inline int64_t scan_entries(int64_t n) { return (n + 7) / 8 * 8; }
inline int64_t scan_tiles(int64_t n) { return (scan_entries(n) + 2047) / 2048; }

// All return the number of kernels launched.
int launch_grid_sort(const GridBuildArgs& a, cudaStream_t s);
// The part of the grid build after the keys: scan of a.hist (a.P.cells + 1 counters) into
// the cell table, scatter, rank by caller id and gather of a.P.n particles.
int launch_grid_order(const GridBuildArgs& a, cudaStream_t s);
int launch_neighbors(const GridBuildArgs& a, cudaStream_t s);
// The grid build's four passes one by one (launch_grid_sort = all four in order): cell keys
// and histogram, scan into the cell table, scatter, rank + gather.
int launch_grid_keys(const GridBuildArgs& a, cudaStream_t s);
int launch_grid_scan(const GridBuildArgs& a, cudaStream_t s);
int launch_grid_scatter(const GridBuildArgs& a, cudaStream_t s);
int launch_grid_gather(const GridBuildArgs& a, cudaStream_t s);

// With b.gradrho set, also stores |grad rho| (a warm-start feature).
void launch_nonpressure(const DevParams& P, const StepBuffers& b, cudaStream_t s);
void launch_sph_pressure(const DevParams& P, const StepBuffers& b, cudaStream_t s);
void launch_integrate_collide(const DevParams& P, const StepBuffers& b, bool add_pforce, cudaStream_t s);

void launch_pci_predict(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s);
void launch_pci_density(const DevParams& P, const StepBuffers& b, int iteration, cudaStream_t s);
void launch_pci_force(const DevParams& P, const StepBuffers& b, cudaStream_t s);
// Whole predict-correct loop in one cooperative persistent launch; returns false when the
// device cannot co-schedule the grid (the caller then uses the per-phase launches).
// ppos_alt: second predicted-position buffer; sync: 16 zeroed bytes; maxerr: max_it zeroed words.
// first_done: iteration 0's predict and density already ran (launch_pci_density_first).
// warm: iteration 0 carried a learned pressure guess, rejected at iteration 1 if it raised
// the maximum density error (the loop then restarts from zero pressure).
bool launch_pci_loop(const DevParams& P, const StepBuffers& b, float4* ppos_alt, void* sync, uint32_t* maxerr,
                     int first_done, int warm, cudaStream_t s, int* grid_used);
// Iteration 0's density pass with the warm-start features.
void launch_pci_density_first(const DevParams& P, const StepBuffers& b, const WarmArgs& w, cudaStream_t s);

// MLP (mlp.cu).
void launch_mlp_pack(const float* master, MlpPacked* packed, cudaStream_t s);
int mlp_grad_rows(int nb);
void launch_mlp_grad(const MlpPacked* packed, const float* feat, const float* target, const int32_t* idx, int nb,
                     float over_weight, float* partial, float* loss_partial, cudaStream_t s);
// k_mlp_grad on exactly `blocks` blocks of 256 threads: writes blocks * 8 partial rows.
void launch_mlp_grad_blocks(const MlpPacked* packed, const float* feat, const float* target, int nb, int blocks,
                            float* partial, float* loss_partial, cudaStream_t s);
void launch_mlp_adam(const float* partial, const float* loss_partial, int rows, float* master, float* m1, float* m2,
                     float* grad_out, float* loss_out, float lr, int step, int apply, cudaStream_t s);
void launch_random_indices(int32_t* idx, int nb, int n, uint64_t seed, cudaStream_t s);

// Gathers a per-particle field from device order into caller order.
// comps: 1 (float) or 3 (xyz of a float4); src is float* or float4* accordingly.
void launch_gather_field(const void* src, int comps, int w_as_flag, const int32_t* slot_of_id, float* out,
                         int64_t n, cudaStream_t s);
void launch_gather_count(const int32_t* count, const int32_t* slot_of_id, float* out, int64_t n, cudaStream_t s);
// Scatters caller-order state (x, v, v_half, v_half_old, first) into device slots.
void launch_scatter_state(const float* x, const float* v, const float* half, const float* old,
                          const int32_t* first, const int32_t* slot_of_id, float4* pos, float4* vel,
                          float4* hvel, float4* oldv, int64_t n, cudaStream_t s);
// dst[slot_of_id[id]] = (in[3 id], in[3 id + 1], in[3 id + 2], 0) for caller-order rows.
void launch_scatter_vec(const float* in, const int32_t* slot_of_id, float4* dst, int64_t n, cudaStream_t s);

// SM count of the current device (cached per device).
int device_sm_count();
// One bounded grid barrier of `blocks` blocks waiting for `parties` arrivals (test of the
// loops' timeout path); throws Error on a CUDA failure.
void barrier_probe(int blocks, int parties, int* completed, uint32_t* error_flags);
// Writes caller-order x, v, v_half, v_half_old, first from device slots.
void launch_gather_state(const float4* pos, const float4* vel, const float4* hvel, const float4* oldv,
                         const int32_t* slot_of_id, float* x, float* v, float* half, float* old, int32_t* first,
                         int64_t n, cudaStream_t s);
// Neighbour lists in caller order and caller ids.
void launch_neighbor_export(const int32_t* nbr, const int32_t* count, int64_t stride, const float4* pos,
                            const int32_t* slot_of_id, const int64_t* offsets, int32_t* out, int64_t n,
                            cudaStream_t s);
void launch_scale(const float* src, float* dst, int64_t n, float factor, cudaStream_t s);
// out[id][c] = src[slot_of_id[id]][c] for rows of `width` floats.
void launch_gather_rows(const float* src, int width, const int32_t* slot_of_id, float* out, int64_t n, cudaStream_t s);
// Axis-aligned bounds of the positions: out[0..2] = min, out[3..5] = max (as ordered ints).
void launch_bounds(const float4* pos, int64_t n, int32_t* out, cudaStream_t s);

}  // namespace lsp
