// Host engine behind the C ABI: owns one scene's device memory and CUDA stream and
// sequences the per-step kernels (PhysicSolver::update, PhysicSolver.cpp:12-21).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lsp.h"
#include "host_util.h"
#include "lsp_kernels.h"
#include "mlp_model.h"

namespace lsp {

// Reference-identical host arithmetic (compiled with -ffp-contract=off).
struct HostKernels {
    float h = 0, step = 0, mass = 0;
    float cut2 = 0;              // smallest float s with sqrt(s) >= h
    std::vector<float> tables;   // 5 x 1001 tables, then the slot thresholds on d and on d^2
    // Every entry of the non-pressure pass's tables (poly6 gradient and Laplacian, viscosity
    // Laplacian) is 0 or within [2^-29, 2^60]: the pass may then divide by the neighbour
    // density with div_by (DevParams::exact_tables).
    bool exact_tables = false;
    // The W table's last entry (slot 1000) is +0 and every s >= cut2 takes that slot
    // (thr2[1000] <= cut2): the density lookups may then skip the cutoff's select
    // (DevParams::density_tail0), since the slot already gives the cutoff's 0.
    bool density_tail0 = false;
    // The same for the spiky gradient table and the distance cutoff: its last entry is a zero
    // and every d >= h takes slot 1000 (thr[1000] <= h) (DevParams::force_tail0).
    bool force_tail0 = false;
    void build(const lsp_params& p);
    float delta(const lsp_params& p, float dt) const;
    float look(int t, float d) const;

private:
    float lattice_denominator(const lsp_params& p) const;
    // calcDelta's lattice sum, computed on the first delta() after build() (build resets it).
    mutable float denom_ = 0.f, denom_radius_ = 0.f;
    mutable bool denom_ready_ = false;
};

// Parameter checks shared by single scenes and batches (LSP_ERR_INVALID on failure).
void validate_params(const lsp_params& p);
// Union of the boundary colliders' boxes; false when there is none.
bool boundary_box(const std::vector<Collider>& cols, float lo[3], float hi[3]);
// Grid origin and dimensions (cells of size h, c = (int)(x / h)) covering [lo, hi]; returns
// the cell count (LSP_ERR_CAPACITY above 2^30).
int64_t grid_from_box(const float lo[3], const float hi[3], float h, int32_t org[3], int32_t dim[3]);
// DevParams fields that follow from the parameters, the derived kernel constants and dt
// (everything except the particle count, grid, colliders and neighbour-list layout).
DevParams physics_params(const lsp_params& p, const HostKernels& hk, float dt);
// First neighbour-list capacity: twice the lattice estimate of the neighbour count.
int initial_neighbor_capacity(const lsp_params& p);
// Neighbour-list capacity after an overflow of `needed` entries with `current` allocated.
int grown_neighbor_capacity(int needed, int current);
// LSP_WARM_AUTO switch point: warm_auto_iterations, or max(12, pci_max_iterations / 2) for 0.
int warm_auto_switch(const lsp_params& p);

class Engine {
public:
    Engine(const lsp_params& p, int device);
    ~Engine();

    void set_params(const lsp_params& p);
    // params.warm_start alone (no table rebuild); LSP_WARM_AUTO starts from the zero start.
    void set_warm_start(int mode);
    const lsp_params& params() const { return prm_; }
    float mass() const { return hk_.mass; }
    float kernel_radius() const { return hk_.h; }
    float delta(float dt) const { return hk_.delta(prm_, dt); }
    const std::vector<float>& tables() const { return hk_.tables; }
    int64_t count() const { return n_; }

    void add_particles(const float* xyz, const float* vel, int64_t m);
    void remove_particles();
    int add_collider(const Collider& c);
    void update_collider(int index, const Collider& c);
    void remove_colliders();
    const std::vector<Collider>& colliders() const { return cols_; }
    void set_domain(const float lo[3], const float hi[3]);
    // The user grid box, if one was set (lsp_set_domain); clear_domain returns to the
    // boundary-collider / particle-bounds rule.
    bool domain(float lo[3], float hi[3]) const;
    void clear_domain()
    {
        domain_user_ = false;
        grid_valid_ = false;
    }
    // Warm-start pressure history (p_{n-1}, p_{n-2}, p_{n-3}) in caller order, float[3n];
    // has_history is false while the warm-start buffers do not exist (all zero then).
    bool has_history() const { return phist_[cur_].p != nullptr; }
    void read_history(float* out, int64_t n);
    void write_history(const float* in, int64_t n);

    void step(float dt, lsp_step_stats* st);
    void step_many(float dt, int steps, lsp_step_stats* st);
    void synchronize();

    void read_field(int field, float* out, int64_t n);
    void read_state(float* x, float* v, float* half, float* old, int32_t* first, int64_t n);
    void write_state(const float* x, const float* v, const float* half, const float* old, const int32_t* first,
                     int64_t n);
    void read_neighbors(int64_t* offsets, int32_t* index, int64_t n, int64_t capacity);
    void grid_info(int32_t dims[3], int32_t origin[3], int64_t* cells) const;
    void read_grid(uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start, int64_t cells_plus_one);

    // Measurement (lsp_timer_*, lsp_profile*, lsp_launch_count).
    void timer_mark(int slot);
    float timer_elapsed(int a, int b);
    void profile(bool on);
    void profile_read(double* ms, int64_t* launches, int capacity);
    int64_t launch_count() const { return launches_; }

    // Learned warm start (lsp_mlp_*).
    void mlp_reset(uint64_t seed);
    void mlp_set(const float* w, int n);
    void mlp_get(float* w, int n);
    void mlp_record(bool on);
    void mlp_set_loss_asymmetry(float w);
    float mlp_train(int iterations, int batch, float lr, uint64_t seed);
    void mlp_forward(const float* feat, int64_t n, float* out);
    float mlp_gradient(const float* feat, const float* target, int64_t n, float* grad);
    void read_features(float* out, int64_t n);

    // Device copy of the fragment-ordered MLP weights (MlpPacked).
    const void* mlp_packed_device() const { return mlp_.packed(); }

    cudaStream_t stream() const { return stream_; }
    int device() const { return dev_; }
    // Device order view for in-library callers (kernel timing, the MLP).
    StepBuffers buffers();
    DevParams device_params(float dt) const;

private:
    void activate() const;
    void derive();
    void ensure_capacity(int64_t n);
    void ensure_grid();
    void ensure_neighbors(int cap);
    void upload_colliders();
    void run_step(float dt, lsp_step_stats* st);
    // Returns true when the persistent device loop ran (its stats arrive with the status).
    bool pcisph_loop(const DevParams& P, const StepBuffers& b, lsp_step_stats* st);
    void stage(size_t floats);

    lsp_params prm_{};
    HostKernels hk_;
    int dev_ = 0;
    cudaStream_t stream_ = nullptr;

    int64_t n_ = 0, cap_ = 0;
    int cur_ = 0;
    DevArray<float4> pos_[2], vel_[2], half_[2], old_[2];
    DevArray<float4> force_, ppos_, ppos_alt_, phalf_, pforce_;
    const float4* ppos_final_ = nullptr;   // buffer holding the last iteration's x*
    DevArray<uint32_t> loop_sync_, maxerr_;
    DevArray<float> rho_, pres_, prho_, err_;
    DevArray<float4> vrho_;   // {v, rho} for the non-pressure pass (StepBuffers::vrho)
    DevArray<uint32_t> key_, slot_, sorted_key_;
    DevArray<int2> tmp_;
    DevArray<int32_t> slot_of_id_, nbr_, nbr_src_, nbr_count_;   // nbr_: grouped lists; nbr_src_: the build's plain lists
    int nbr_cap_ = 0;
    int64_t nbr_stride_ = 0;

    DevArray<uint32_t> hist_, cell_start_, tile_sums_;
    int64_t cells_alloc_ = 0;
    bool grid_valid_ = false, domain_user_ = false, domain_from_particles_ = false;
    float dom_lo_[3] = {0, 0, 0}, dom_hi_[3] = {0, 0, 0};
    int32_t org_[3] = {0, 0, 0}, dim_[3] = {1, 1, 1};
    int64_t cells_ = 1;

    DevArray<float> tables_;
    DevArray<Collider> dcols_;
    std::vector<Collider> cols_;
    bool cols_dirty_ = true, tables_dirty_ = true;

    DevArray<DevStatus> status_;
    DevStatus* hstatus_ = nullptr;   // pinned
    DevArray<float> stage_;

    // Launch bracketing for the per-class profile.
    template <typename F>
    void timed(int cls, F&& launch);
    void collect_profile();
    cudaEvent_t marks_[16] = {};
    bool profile_ = false;
    std::vector<cudaEvent_t> evpool_;
    size_t evnext_ = 0;
    std::vector<std::pair<int, size_t>> pending_;   // (class, first event index)
    double prof_ms_[LSP_PROF_COUNT] = {};
    int64_t prof_n_[LSP_PROF_COUNT] = {};
    int64_t launches_ = 0;
    DevArray<int32_t> bounds_;
    bool stepped_ = false;   // a step has run on the current particle set (lists, grid, features valid)

    // Learned warm start state.
    bool features_on() const;
    bool warm_on() const;      // this step starts from the learned guess
    bool history_on() const;   // the pressure history is kept
    void ensure_warm_buffers();
    bool record_ = false, features_valid_ = false;
    bool auto_on_ = false;  // LSP_WARM_AUTO has switched the learned guess on
    float last_p_scale_ = 1.f;
    DevArray<float4> phist_[2];   // pressure history (p_{n-1}, p_{n-2}, p_{n-3})
    DevArray<float> feat_, gradrho_, tgt_;
    MlpModel mlp_;
};

}  // namespace lsp
