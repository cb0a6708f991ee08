// Test infrastructure (the oracle), not product code.
//
// CPU restatement of LiquidPhysics' sequential SPH / PCISPH step
// (LiquidPhysics/src/SPHSolver.cpp, PCISPHSolver.cpp, SPHSpatialGrid.cpp,
// Kernels/*.cpp, Collision/*.cpp, Particles/SPHParticle.cpp) in structure-of-arrays
// form, with every floating-point operation in the reference's order so that the
// FP32 instantiation reproduces the compiled reference bit for bit. It adds what
// the reference lacks and the parity tests need: a minimum PCISPH iteration count,
// an FP64 instantiation, the per-step statistics, and a restatement of the device
// grid build (cell keys, sorted order, dense cell table).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
#pragma once

#include "../include/lsp.h"

#ifdef __cplusplus
extern "C" {
#endif

void* orc_create(const lsp_params* p, int fp64);
void orc_destroy(void* h);
int orc_set_params(void* h, const lsp_params* p);
int orc_add_particles(void* h, const float* xyz, const float* vel, int64_t n);
int orc_add_box(void* h, const float center[3], const float half_extent[3], int kind);
int orc_add_sphere(void* h, const float center[3], float radius, int kind);
int orc_update_box(void* h, int index, const float center[3], const float half_extent[3]);
int orc_update_sphere(void* h, int index, const float center[3], float radius);
int64_t orc_count(void* h);
int orc_step(void* h, float dt, lsp_step_stats* stats);
// Next step only: iteration 0 takes this pressure (caller order, n = particle count) in
// place of its own correction, as the device's learned warm start does; checked at
// iteration 1 and dropped for the zero start if the maximum density error rose.
int orc_set_initial_pressure(void* h, const float* pressure, int64_t n);
// PCISPH pressure scaling used instead of the derived one (0: derive it, the default).
int orc_set_delta_override(void* h, double delta);
int orc_get(void* h, int field, float* out);
int orc_get_f64(void* h, int field, double* out);
int orc_set_state(void* h, const float* x, const float* v, const float* half, const float* old_half, const int32_t* first);
float orc_mass(void* h);
float orc_kernel_radius(void* h);
float orc_delta(void* h, float dt);
void orc_tables(void* h, float* out);
int64_t orc_neighbor_total(void* h);
void orc_neighbor_lists(void* h, int64_t* offsets, int32_t* index);
void orc_set_threads(int threads);

// Device grid-build specification (see the comment at its definition).
int orc_grid_build(const float* xyz, int64_t n, float h, const int32_t origin[3], const int32_t dims[3],
                   uint32_t* keys_sorted, int32_t* ids_sorted, uint32_t* cell_start, int64_t* escaped);

#ifdef __cplusplus
}
#endif
