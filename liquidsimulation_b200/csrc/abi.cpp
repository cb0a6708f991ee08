// extern "C" entry points of include/lsp.h over lsp::Engine. Every call catches
// lsp::Error (and std::exception) and turns it into a status code plus a per-thread
// message for lsp_last_error().
#include <cstring>
#include <string>

#include "../../include/lsp.h"
#include "engine.h"
#include "lsp_handle.h"

namespace {
thread_local std::string g_last_error;

lsp::Engine& E(lsp_solver* s)
{
    if (!s || !s->e) throw lsp::Error(LSP_ERR_INVALID, "null solver handle");
    return *s->e;
}
const lsp::Engine& E(const lsp_solver* s)
{
    if (!s || !s->e) throw lsp::Error(LSP_ERR_INVALID, "null solver handle");
    return *s->e;
}
void need(const void* p, const char* what)
{
    if (!p) throw lsp::Error(LSP_ERR_INVALID, std::string("null pointer: ") + what);
}
}  // namespace

namespace lsp {
void set_last_error(const std::string& message) { g_last_error = message; }
}  // namespace lsp

extern "C" {

void lsp_params_default(lsp_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gravity[0] = 0.f;
    p->gravity[1] = -9.81f;
    p->gravity[2] = 0.f;
    p->particle_radius = 0.017f;
    p->kernel_radius_factor = 2.688f;
    p->rest_density = 998.29f;
    p->viscosity = 3.5f;
    p->stiffness = 3.f;
    p->negative_pressure_factor = 0.f;
    p->surface_tension = 0.0728f;
    p->surface_tension_threshold = 7.065f;
    p->restitution = 0.5f;
    p->friction = 1.f;
    p->mass_override = 0.f;
    p->solver = LSP_SOLVER_SPH;
    p->pci_max_iterations = 4;
    p->pci_min_iterations = 1;
    p->pci_eta = 0.1f;
    p->warm_start = LSP_WARM_ZERO;
}

const char* lsp_last_error(void) { return g_last_error.c_str(); }

int lsp_barrier_probe(int device, int blocks, int parties, int32_t* completed, uint32_t* error_flags)
{
    return lsp::guard([&] {
        if (!completed || !error_flags || blocks < 1 || blocks > 8 || parties < 1 || parties > 16)
            throw lsp::Error(LSP_ERR_INVALID, "barrier probe: blocks in [1, 8], parties in [1, 16], non-null outputs");
        int prev = 0;
        LSP_CK(cudaGetDevice(&prev));
        if (device >= 0) LSP_CK(cudaSetDevice(device));
        int done = 0;
        uint32_t flags = 0;
        try {
            lsp::barrier_probe(blocks, parties, &done, &flags);
        } catch (...) {
            cudaSetDevice(prev);
            throw;
        }
        LSP_CK(cudaSetDevice(prev));
        *completed = done;
        *error_flags = flags;
    });
}

int lsp_device_info(int* sm_count, int* cc_major, int* cc_minor)
{
    return lsp::guard([&] {
        int dev = 0, n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw lsp::Error(LSP_ERR_NO_DEVICE, "no CUDA device");
        cudaGetDevice(&dev);
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) throw lsp::Error(LSP_ERR_CUDA, "device query failed");
        if (sm_count) *sm_count = p.multiProcessorCount;
        if (cc_major) *cc_major = p.major;
        if (cc_minor) *cc_minor = p.minor;
    });
}

int lsp_create(const lsp_params* params, int device, lsp_solver** out)
{
    return lsp::guard([&] {
        need(params, "params");
        need(out, "out");
        *out = nullptr;
        lsp_solver* s = new lsp_solver{nullptr};
        try {
            s->e = new lsp::Engine(*params, device);
            // The allocation-free gradient's scratch is set up with the solver, so that
            // lsp_mlp_gradient_static itself never loads a module or looks a symbol up.
            lsp::scratch_on(s->e->device());
        } catch (...) {
            delete s->e;
            delete s;
            throw;
        }
        *out = s;
    });
}

int lsp_destroy(lsp_solver* s)
{
    return lsp::guard([&] {
        if (!s) return;
        delete s->e;
        delete s;
    });
}

int lsp_set_params(lsp_solver* s, const lsp_params* p)
{
    return lsp::guard([&] { need(p, "params"); E(s).set_params(*p); });
}
int lsp_get_params(const lsp_solver* s, lsp_params* out)
{
    return lsp::guard([&] { need(out, "out"); *out = E(s).params(); });
}
int lsp_particle_mass(const lsp_solver* s, float* m)
{
    return lsp::guard([&] { need(m, "mass"); *m = E(s).mass(); });
}
int lsp_kernel_radius(const lsp_solver* s, float* h)
{
    return lsp::guard([&] { need(h, "h"); *h = E(s).kernel_radius(); });
}
int lsp_particle_count(const lsp_solver* s, int64_t* n)
{
    return lsp::guard([&] { need(n, "n"); *n = E(s).count(); });
}
int lsp_pcisph_delta(const lsp_solver* s, float dt, float* delta)
{
    return lsp::guard([&] { need(delta, "delta"); *delta = E(s).delta(dt); });
}
int lsp_kernel_tables(const lsp_solver* s, float* out, int capacity)
{
    return lsp::guard([&] {
        need(out, "out");
        const auto& t = E(s).tables();
        const int n = 5 * lsp::kTableSize;
        if (capacity < n) throw lsp::Error(LSP_ERR_INVALID, "capacity below 5*1001");
        std::memcpy(out, t.data(), n * sizeof(float));
    });
}

int lsp_add_particles(lsp_solver* s, const float* xyz, const float* vel, int64_t n)
{
    return lsp::guard([&] { E(s).add_particles(xyz, vel, n); });
}
int lsp_remove_particles(lsp_solver* s)
{
    return lsp::guard([&] { E(s).remove_particles(); });
}

static lsp::Collider box_of(const float c[3], const float h[3], int kind)
{
    if (kind != LSP_OBSTACLE && kind != LSP_BOUNDARY) throw lsp::Error(LSP_ERR_INVALID, "kind must be LSP_OBSTACLE or LSP_BOUNDARY");
    lsp::Collider o{};
    o.sphere = 0;
    o.boundary = kind == LSP_BOUNDARY;
    o.cx = c[0]; o.cy = c[1]; o.cz = c[2];
    o.hx = h[0]; o.hy = h[1]; o.hz = h[2];
    return o;
}
static lsp::Collider sphere_of(const float c[3], float r, int kind)
{
    if (kind != LSP_OBSTACLE && kind != LSP_BOUNDARY) throw lsp::Error(LSP_ERR_INVALID, "kind must be LSP_OBSTACLE or LSP_BOUNDARY");
    lsp::Collider o{};
    o.sphere = 1;
    o.boundary = kind == LSP_BOUNDARY;
    o.cx = c[0]; o.cy = c[1]; o.cz = c[2];
    o.radius = r;
    return o;
}

int lsp_add_box(lsp_solver* s, const float center[3], const float half_extent[3], int kind)
{
    return lsp::guard([&] {
        need(center, "center");
        need(half_extent, "half_extent");
        E(s).add_collider(box_of(center, half_extent, kind));
    });
}
int lsp_add_sphere(lsp_solver* s, const float center[3], float radius, int kind)
{
    return lsp::guard([&] {
        need(center, "center");
        E(s).add_collider(sphere_of(center, radius, kind));
    });
}
int lsp_remove_colliders(lsp_solver* s)
{
    return lsp::guard([&] { E(s).remove_colliders(); });
}
int lsp_update_box(lsp_solver* s, int index, const float center[3], const float half_extent[3])
{
    return lsp::guard([&] {
        need(center, "center");
        need(half_extent, "half_extent");
        E(s).update_collider(index, box_of(center, half_extent, LSP_OBSTACLE));
    });
}
int lsp_update_sphere(lsp_solver* s, int index, const float center[3], float radius)
{
    return lsp::guard([&] {
        need(center, "center");
        E(s).update_collider(index, sphere_of(center, radius, LSP_OBSTACLE));
    });
}
int lsp_set_domain(lsp_solver* s, const float lo[3], const float hi[3])
{
    return lsp::guard([&] {
        need(lo, "lo");
        need(hi, "hi");
        E(s).set_domain(lo, hi);
    });
}

int lsp_step(lsp_solver* s, float dt, lsp_step_stats* stats)
{
    return lsp::guard([&] { E(s).step(dt, stats); });
}
int lsp_step_many(lsp_solver* s, float dt, int steps, lsp_step_stats* stats)
{
    return lsp::guard([&] { E(s).step_many(dt, steps, stats); });
}
int lsp_synchronize(lsp_solver* s)
{
    return lsp::guard([&] { E(s).synchronize(); });
}

int lsp_read_particles(lsp_solver* s, float* xyz, float* vel, int64_t n)
{
    return lsp::guard([&] {
        if (xyz) E(s).read_field(LSP_FIELD_POSITION, xyz, n);
        if (vel) E(s).read_field(LSP_FIELD_VELOCITY, vel, n);
    });
}
int lsp_read_field(lsp_solver* s, int field, float* out, int64_t n)
{
    return lsp::guard([&] { E(s).read_field(field, out, n); });
}
int lsp_read_state(lsp_solver* s, float* x, float* v, float* half, float* old_half, int32_t* first, int64_t n)
{
    return lsp::guard([&] { E(s).read_state(x, v, half, old_half, first, n); });
}
int lsp_write_state(lsp_solver* s, const float* x, const float* v, const float* half, const float* old_half,
                    const int32_t* first, int64_t n)
{
    return lsp::guard([&] { E(s).write_state(x, v, half, old_half, first, n); });
}
int lsp_read_neighbors(lsp_solver* s, int64_t* offsets, int32_t* index, int64_t n, int64_t capacity)
{
    return lsp::guard([&] { E(s).read_neighbors(offsets, index, n, capacity); });
}
int lsp_grid_info(lsp_solver* s, int32_t dims[3], int32_t origin[3], int64_t* cells)
{
    return lsp::guard([&] { E(s).grid_info(dims, origin, cells); });
}
int lsp_read_grid(lsp_solver* s, uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start, int64_t cells_plus_one)
{
    return lsp::guard([&] { E(s).read_grid(keys, ids, n, cell_start, cells_plus_one); });
}

int lsp_mlp_reset(lsp_solver* s, uint64_t seed)
{
    return lsp::guard([&] { E(s).mlp_reset(seed); });
}
int lsp_mlp_set_weights(lsp_solver* s, const float* w, int n)
{
    return lsp::guard([&] { E(s).mlp_set(w, n); });
}
int lsp_mlp_get_weights(lsp_solver* s, float* w, int n)
{
    return lsp::guard([&] { E(s).mlp_get(w, n); });
}
int lsp_mlp_record(lsp_solver* s, int enable)
{
    return lsp::guard([&] { E(s).mlp_record(enable != 0); });
}
int lsp_set_warm_start(lsp_solver* s, int mode)
{
    return lsp::guard([&] { E(s).set_warm_start(mode); });
}
int lsp_mlp_set_loss_asymmetry(lsp_solver* s, float over_weight)
{
    return lsp::guard([&] { E(s).mlp_set_loss_asymmetry(over_weight); });
}
int lsp_mlp_train(lsp_solver* s, int iterations, int batch, float learning_rate, uint64_t seed, float* loss)
{
    return lsp::guard([&] {
        float l = E(s).mlp_train(iterations, batch, learning_rate, seed);
        if (loss) *loss = l;
    });
}
int lsp_mlp_forward(lsp_solver* s, const float* features, int64_t n, float* out)
{
    return lsp::guard([&] { E(s).mlp_forward(features, n, out); });
}
int lsp_mlp_gradient(lsp_solver* s, const float* features, const float* targets, int64_t n, float* grad, float* loss)
{
    return lsp::guard([&] {
        float l = E(s).mlp_gradient(features, targets, n, grad);
        if (loss) *loss = l;
    });
}
int lsp_read_features(lsp_solver* s, float* out, int64_t n)
{
    return lsp::guard([&] { E(s).read_features(out, n); });
}

int lsp_timer_mark(lsp_solver* s, int slot)
{
    return lsp::guard([&] { E(s).timer_mark(slot); });
}
int lsp_timer_elapsed(lsp_solver* s, int slot_a, int slot_b, float* ms)
{
    return lsp::guard([&] { need(ms, "ms"); *ms = E(s).timer_elapsed(slot_a, slot_b); });
}
int lsp_profile(lsp_solver* s, int enable)
{
    return lsp::guard([&] { E(s).profile(enable != 0); });
}
int lsp_profile_read(lsp_solver* s, double* ms, int64_t* launches, int capacity)
{
    return lsp::guard([&] { E(s).profile_read(ms, launches, capacity); });
}
int lsp_launch_count(const lsp_solver* s, int64_t* launches)
{
    return lsp::guard([&] { need(launches, "launches"); *launches = E(s).launch_count(); });
}
int lsp_host_alloc(size_t bytes, void** out)
{
    return lsp::guard([&] {
        need(out, "out");
        *out = nullptr;
        cudaError_t e = cudaMallocHost(out, bytes);
        if (e != cudaSuccess) throw lsp::Error(LSP_ERR_CUDA, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
    });
}
int lsp_host_free(void* p)
{
    return lsp::guard([&] {
        if (p) cudaFreeHost(p);
    });
}

}  // extern "C"
