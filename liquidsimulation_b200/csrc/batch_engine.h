// Host engine of a batch of independent scenes (lsp_batch_* in include/lsp.h): one set of
// device arrays for all scenes, one stream, and a step that is one CUDA graph (grid build,
// neighbour lists, density, non-pressure forces, the persistent PCISPH loop of every
// scene, integration) per buffer parity.
#pragma once

#include <cstdint>
#include <vector>

#include "batch_kernels.h"
#include "engine.h"

namespace lsp {

class BatchEngine {
public:
    explicit BatchEngine(int device);
    ~BatchEngine();

    int add_scene(const lsp_params& p, const float* xyz, const float* vel, int64_t n, const float* lo,
                  const float* hi);
    int add_collider(int scene, const Collider& c);
    void update_collider(int scene, int index, const Collider& c);

    int scenes() const { return (int)sc_.size(); }
    int64_t total() const { return n_; }
    int64_t scene_count(int scene) const { return at(scene).n; }
    const lsp_params& scene_params(int scene) const { return at(scene).prm; }
    float scene_mass(int scene) const { return at(scene).hk.mass; }
    void grid_info(int scene, int32_t dims[3], int32_t origin[3], int64_t* cells) const;

    void step(float dt, lsp_step_stats* stats);

    void read_particles(int scene, float* x, float* v, int64_t n);
    void read_field(int scene, int field, float* out, int64_t n);
    void read_neighbors(int scene, int64_t* offsets, int32_t* index, int64_t n, int64_t capacity);
    void read_grid(int scene, uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start, int64_t cells_plus_one);
    // Whole batch in caller order, scene after scene.
    void read_state(float* x, float* v, float* half, float* old, int32_t* first, int64_t n);
    void write_state(const float* x, const float* v, const float* half, const float* old, const int32_t* first,
                     int64_t n);

    void set_launch(int use_graph, int threads, int loop_blocks);
    void get_launch(int* use_graph, int* threads, int* loop_blocks, int* graph_active) const;
    void autotune(float dt, int repeats, lsp_batch_tuning* out, lsp_step_stats* stats);

    void timer_mark(int slot);
    float timer_elapsed(int a, int b);
    int64_t launch_count() const { return launches_; }

    // Learned warm start of every PCISPH scene (one network for the batch; features are
    // normalised per scene).
    void set_warm_start(int mode);
    void mlp_reset(uint64_t seed);
    void mlp_set(const float* w, int n);
    void mlp_get(float* w, int n);
    void mlp_record(bool on);
    void mlp_set_loss_asymmetry(float w);
    // Adam steps on the features and final pressures of the last recorded step.
    float mlp_train(int iterations, int batch, float lr, uint64_t seed);
    void read_features(int scene, float* out, int64_t n);

private:
    struct Scene {
        lsp_params prm{};
        HostKernels hk;
        std::vector<Collider> cols;
        bool user_domain = false;
        float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        int64_t n = 0, base = 0;
        int32_t org[3] = {0, 0, 0}, dim[3] = {1, 1, 1};
        int64_t cells = 1, cell_base = 0;
        int coll_off = 0;
        int last_k = 0;
    };
    const Scene& at(int scene) const;
    Scene& at(int scene);
    void activate() const;
    void build();                   // lays out the device arrays at the first step
    void upload_params(float dt);   // DevParams of every scene (dt-dependent delta)
    void upload_colliders();
    void build_items();
    void ensure_neighbors(int cap);
    void drop_graphs();
    int loop_grid() const;
    int enqueue_step(int c, int grid);   // returns the number of kernels launched
    void run_once(int c);           // one step attempt from buffer parity c (graph or direct)
    // Runs the step from parity cur_ until no list overflows; false if it still overflowed.
    bool run_checked();
    void finish_step(lsp_step_stats* stats);
    StepBuffers buffers(int c);
    BatchArgs args();
    void stage(size_t floats);
    void check_scene(int scene) const;
    // The guess runs for every scene (LSP_WARM_MLP) or for the scenes LSP_WARM_AUTO has
    // switched on; features are computed whenever some scene uses the guess or recording is
    // on, and the pressure history is kept from the start in LSP_WARM_AUTO.
    bool guess_on() const { return pcisph_ && (warm_ == LSP_WARM_MLP || (warm_ == LSP_WARM_AUTO && auto_any_)); }
    bool features_on() const { return pcisph_ && (record_ || guess_on()); }
    bool history_on() const { return pcisph_ && (record_ || warm_ != LSP_WARM_ZERO); }
    void upload_auto();
    void ensure_warm_buffers();

    int dev_ = 0;
    cudaStream_t stream_ = nullptr;
    std::vector<Scene> sc_;
    std::vector<float4> init_pos_, init_vel_;   // host copies until the first step
    bool built_ = false, pcisph_ = true;
    int64_t n_ = 0, cells_ = 0;
    int cur_ = 0;
    int mstride_ = 0;
    float dt_ = -1.f;
    bool params_dirty_ = true, cols_dirty_ = true;

    DevArray<float4> pos_[2], vel_[2], half_[2], old_[2];
    DevArray<float4> force_, ppos_, ppos_alt_, phalf_, pforce_;
    DevArray<float> rho_, pres_, prho_, err_;
    DevArray<float4> vrho_;   // {v, rho} for the non-pressure pass (StepBuffers::vrho)
    DevArray<uint32_t> key_, slot_, sorted_key_, hist_, cell_start_, tile_sums_, loop_sync_, maxerr_;
    DevArray<int2> tmp_;
    DevArray<int32_t> slot_of_id_, nbr_, nbr_src_, nbr_count_;   // nbr_: grouped lists; nbr_src_: the build's plain lists
    DevArray<float> tables_, stage_;
    DevArray<Collider> dcols_;
    DevArray<DevParams> dparams_;
    DevArray<BatchItem> items_;
    DevArray<DevStatus> status_;
    DevParams* hparams_ = nullptr;   // pinned
    DevStatus* hstatus_ = nullptr;   // pinned
    int items_count_ = 0;
    int nbr_cap_ = 0;
    int64_t nbr_stride_ = 0;

    int threads_ = 256, loop_blocks_ = 0;
    bool use_graph_ = true, graph_ok_ = true;
    cudaGraphExec_t graph_[2] = {nullptr, nullptr};
    int graph_launches_[2] = {0, 0};

    cudaEvent_t marks_[16] = {};
    int64_t launches_ = 0;

    int warm_ = LSP_WARM_ZERO;
    bool record_ = false, features_valid_ = false;
    std::vector<int32_t> auto_on_;    // LSP_WARM_AUTO: scenes whose guess is switched on
    bool auto_any_ = false;
    DevArray<int32_t> warm_scene_;    // device copy of auto_on_
    DevArray<float4> phist_[2];   // pressure history (p_{n-1}, p_{n-2}, p_{n-3})
    DevArray<float> feat_, gradrho_, tgt_;
    MlpModel mlp_;
};

}  // namespace lsp
