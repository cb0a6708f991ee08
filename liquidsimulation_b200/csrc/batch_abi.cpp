// extern "C" entry points of the batch section of include/lsp.h over lsp::BatchEngine.
// Same error convention as abi.cpp: every call returns a status code and leaves a message
// for lsp_last_error() on failure.
#include <cstring>
#include <string>

#include "../../include/lsp.h"
#include "batch_engine.h"
#include "lsp_handle.h"

struct lsp_batch {
    lsp::BatchEngine* e;
};

namespace {

lsp::BatchEngine& B(lsp_batch* b)
{
    if (!b || !b->e) throw lsp::Error(LSP_ERR_INVALID, "null batch handle");
    return *b->e;
}
const lsp::BatchEngine& B(const lsp_batch* b)
{
    if (!b || !b->e) throw lsp::Error(LSP_ERR_INVALID, "null batch handle");
    return *b->e;
}
void need(const void* p, const char* what)
{
    if (!p) throw lsp::Error(LSP_ERR_INVALID, std::string("null pointer: ") + what);
}
lsp::Collider collider(int sphere, const float c[3], const float h[3], float r, int kind)
{
    if (kind != LSP_OBSTACLE && kind != LSP_BOUNDARY)
        throw lsp::Error(LSP_ERR_INVALID, "kind must be LSP_OBSTACLE or LSP_BOUNDARY");
    lsp::Collider o{};
    o.sphere = sphere;
    o.boundary = kind == LSP_BOUNDARY;
    o.cx = c[0]; o.cy = c[1]; o.cz = c[2];
    if (h) { o.hx = h[0]; o.hy = h[1]; o.hz = h[2]; }
    o.radius = r;
    return o;
}

}  // namespace

extern "C" {

int lsp_batch_create(int device, lsp_batch** out)
{
    return lsp::guard([&] {
        need(out, "out");
        *out = nullptr;
        lsp_batch* b = new lsp_batch{nullptr};
        try {
            b->e = new lsp::BatchEngine(device);
        } catch (...) {
            delete b;
            throw;
        }
        *out = b;
    });
}

int lsp_batch_destroy(lsp_batch* b)
{
    return lsp::guard([&] {
        if (!b) return;
        delete b->e;
        delete b;
    });
}

int lsp_batch_add_scene(lsp_batch* b, const lsp_params* params, const float* xyz, const float* vel, int64_t n,
                        const float* domain_lo, const float* domain_hi, int32_t* scene)
{
    return lsp::guard([&] {
        need(params, "params");
        int s = B(b).add_scene(*params, xyz, vel, n, domain_lo, domain_hi);
        if (scene) *scene = s;
    });
}

int lsp_batch_add_box(lsp_batch* b, int32_t scene, const float center[3], const float half_extent[3], int kind)
{
    return lsp::guard([&] {
        need(center, "center");
        need(half_extent, "half_extent");
        B(b).add_collider(scene, collider(0, center, half_extent, 0.f, kind));
    });
}

int lsp_batch_add_sphere(lsp_batch* b, int32_t scene, const float center[3], float radius, int kind)
{
    return lsp::guard([&] {
        need(center, "center");
        B(b).add_collider(scene, collider(1, center, nullptr, radius, kind));
    });
}

int lsp_batch_update_box(lsp_batch* b, int32_t scene, int32_t index, const float center[3],
                         const float half_extent[3])
{
    return lsp::guard([&] {
        need(center, "center");
        need(half_extent, "half_extent");
        B(b).update_collider(scene, index, collider(0, center, half_extent, 0.f, LSP_OBSTACLE));
    });
}

int lsp_batch_update_sphere(lsp_batch* b, int32_t scene, int32_t index, const float center[3], float radius)
{
    return lsp::guard([&] {
        need(center, "center");
        B(b).update_collider(scene, index, collider(1, center, nullptr, radius, LSP_OBSTACLE));
    });
}

int lsp_batch_info(const lsp_batch* b, int32_t* scenes, int64_t* particles)
{
    return lsp::guard([&] {
        if (scenes) *scenes = B(b).scenes();
        if (particles) *particles = B(b).total();
    });
}

int lsp_batch_scene_count(const lsp_batch* b, int32_t scene, int64_t* n)
{
    return lsp::guard([&] {
        need(n, "n");
        *n = B(b).scene_count(scene);
    });
}

int lsp_batch_particle_mass(const lsp_batch* b, int32_t scene, float* mass)
{
    return lsp::guard([&] {
        need(mass, "mass");
        *mass = B(b).scene_mass(scene);
    });
}

int lsp_batch_step(lsp_batch* b, float dt, lsp_step_stats* stats)
{
    return lsp::guard([&] { B(b).step(dt, stats); });
}

int lsp_batch_read_particles(lsp_batch* b, int32_t scene, float* xyz, float* vel, int64_t n)
{
    return lsp::guard([&] { B(b).read_particles(scene, xyz, vel, n); });
}

int lsp_batch_read_field(lsp_batch* b, int32_t scene, int field, float* out, int64_t n)
{
    return lsp::guard([&] { B(b).read_field(scene, field, out, n); });
}

int lsp_batch_read_neighbors(lsp_batch* b, int32_t scene, int64_t* offsets, int32_t* index, int64_t n,
                             int64_t capacity)
{
    return lsp::guard([&] { B(b).read_neighbors(scene, offsets, index, n, capacity); });
}

int lsp_batch_grid_info(const lsp_batch* b, int32_t scene, int32_t dims[3], int32_t origin[3], int64_t* cells)
{
    return lsp::guard([&] { B(b).grid_info(scene, dims, origin, cells); });
}

int lsp_batch_read_grid(lsp_batch* b, int32_t scene, uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start,
                        int64_t cells_plus_one)
{
    return lsp::guard([&] { B(b).read_grid(scene, keys, ids, n, cell_start, cells_plus_one); });
}

int lsp_batch_read_state(lsp_batch* b, float* x, float* v, float* v_half, float* v_half_old, int32_t* first_step,
                         int64_t n)
{
    return lsp::guard([&] { B(b).read_state(x, v, v_half, v_half_old, first_step, n); });
}

int lsp_batch_write_state(lsp_batch* b, const float* x, const float* v, const float* v_half,
                          const float* v_half_old, const int32_t* first_step, int64_t n)
{
    return lsp::guard([&] { B(b).write_state(x, v, v_half, v_half_old, first_step, n); });
}

int lsp_batch_set_launch(lsp_batch* b, int use_graph, int threads, int loop_blocks)
{
    return lsp::guard([&] { B(b).set_launch(use_graph, threads, loop_blocks); });
}

int lsp_batch_get_launch(const lsp_batch* b, int* use_graph, int* threads, int* loop_blocks, int* graph_active)
{
    return lsp::guard([&] { B(b).get_launch(use_graph, threads, loop_blocks, graph_active); });
}

int lsp_batch_autotune(lsp_batch* b, float dt, int repeats, lsp_batch_tuning* result, lsp_step_stats* stats)
{
    return lsp::guard([&] { B(b).autotune(dt, repeats, result, stats); });
}

int lsp_batch_set_warm_start(lsp_batch* b, int mode)
{
    return lsp::guard([&] { B(b).set_warm_start(mode); });
}

int lsp_batch_mlp_reset(lsp_batch* b, uint64_t seed)
{
    return lsp::guard([&] { B(b).mlp_reset(seed); });
}

int lsp_batch_mlp_set_weights(lsp_batch* b, const float* w, int n)
{
    return lsp::guard([&] { B(b).mlp_set(w, n); });
}

int lsp_batch_mlp_get_weights(lsp_batch* b, float* w, int n)
{
    return lsp::guard([&] { B(b).mlp_get(w, n); });
}

int lsp_batch_mlp_record(lsp_batch* b, int on)
{
    return lsp::guard([&] { B(b).mlp_record(on != 0); });
}

int lsp_batch_mlp_set_loss_asymmetry(lsp_batch* b, float over_weight)
{
    return lsp::guard([&] { B(b).mlp_set_loss_asymmetry(over_weight); });
}

int lsp_batch_mlp_train(lsp_batch* b, int iterations, int batch, float lr, uint64_t seed, float* loss)
{
    return lsp::guard([&] {
        float l = B(b).mlp_train(iterations, batch, lr, seed);
        if (loss) *loss = l;
    });
}

int lsp_batch_read_features(lsp_batch* b, int32_t scene, float* out, int64_t n)
{
    return lsp::guard([&] { B(b).read_features(scene, out, n); });
}

int lsp_batch_timer_mark(lsp_batch* b, int slot)
{
    return lsp::guard([&] { B(b).timer_mark(slot); });
}

int lsp_batch_timer_elapsed(lsp_batch* b, int slot_a, int slot_b, float* ms)
{
    return lsp::guard([&] {
        need(ms, "ms");
        *ms = B(b).timer_elapsed(slot_a, slot_b);
    });
}

int lsp_batch_launch_count(const lsp_batch* b, int64_t* launches)
{
    return lsp::guard([&] {
        need(launches, "launches");
        *launches = B(b).launch_count();
    });
}

}  // extern "C"
