// Host engine: device memory, grid box, step sequencing. See engine.h.
#include "engine.h"
#include "mlp.cuh"
#include "mlp_tc.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>

namespace lsp {

#define CK(call) LSP_CK(call)

// ------------------------------------------------------------------ host kernels
// SPHKernel::setRadius / recalcCachedWeights (SPHKernel.cpp:93-137) with the poly6,
// spiky and viscosity formulas (DefaultKernel.cpp:12-42, PressureKernel.cpp:12-42,
// ViscosityKernel.cpp:12-40); SPHSolver::recalcKernelRadius / recalcParticleMass
// (SPHSolver.cpp:480-523). Coefficients are formed in double, as M_PI makes them in the
// reference, and rounded to float.
void HostKernels::build(const lsp_params& p)
{
    denom_ready_ = false;
    const int sub = kTableSize - 1;
    h = p.kernel_radius_factor * p.particle_radius;
    float r2 = h * h, r3 = r2 * h, r4 = r3 * h, r5 = r4 * h, r6 = r5 * h, r9 = r6 * r3;
    (void)r4;
    step = h / sub;
    const double pi = 3.14159265358979323846;
    float poly_k = (float)(315.0 / (64.0 * pi * (double)r9));
    float poly_d1 = (float)(-945.0 / (32.0 * pi * (double)r9));
    float poly_d2 = (float)(-945.0 / (32.0 * pi * (double)r9));
    float spiky_d1 = (float)(-45.0 / (pi * (double)r6));
    float visc_d2 = (float)(45.0 / (pi * (double)r6));
    // Five lookup tables, then the kTableSize + 1 slot thresholds of the device lookup on
    // the distance, then the same thresholds on the squared distance.
    tables.assign(kTableFloats, 0.f);
    for (int i = 0; i <= sub; i++) {
        float d = i * step;
        float t = r2 - d * d;
        tables[0 * kTableSize + i] = poly_k * t * t * t;
        tables[1 * kTableSize + i] = poly_d1 * t * t;
        tables[2 * kTableSize + i] = poly_d2 * (r2 - d * d) * (3.f * r2 - 7.f * d * d);
        float s = h - d;
        tables[3 * kTableSize + i] = spiky_d1 * s * s;
        tables[4 * kTableSize + i] = visc_d2 * (h - d);
    }
    // thr[k] = smallest float d >= 0 with (int)(d / step) >= k, by bisection over the
    // ordered bit patterns of non-negative floats; thr[1001] = +inf.
    float* thr = tables.data() + 5 * kTableSize;
    thr[0] = 0.f;
    const float hi_d = 2.f * h;
    uint32_t hi_bits;
    std::memcpy(&hi_bits, &hi_d, 4);
    for (int k = 1; k <= sub; k++) {
        uint32_t lo = 0, hi = hi_bits;
        while (lo < hi) {
            uint32_t mid = lo + (hi - lo) / 2;
            float d;
            std::memcpy(&d, &mid, 4);
            if ((int)(d / step) >= k) hi = mid; else lo = mid + 1;
        }
        std::memcpy(&thr[k], &lo, 4);
    }
    thr[kTableSize] = std::numeric_limits<float>::infinity();
    // thr2[k] = smallest float s >= 0 whose rounded square root reaches thr[k]: since the
    // IEEE square root is monotone, sqrt(s) >= thr[k] exactly when s >= thr2[k], so a pass
    // that needs the distance only for the table compares squared distances instead.
    float* thr2 = tables.data() + kThresh2Offset;
    auto sq_bound = [](float t) {
        const float hi_s = 4.f * t * t + 1.f;
        uint32_t lo = 0, hi;
        std::memcpy(&hi, &hi_s, 4);
        while (lo < hi) {
            uint32_t mid = lo + (hi - lo) / 2;
            float s;
            std::memcpy(&s, &mid, 4);
            if (std::sqrt(s) >= t) hi = mid; else lo = mid + 1;
        }
        float s;
        std::memcpy(&s, &lo, 4);
        return s;
    };
    thr2[0] = 0.f;
    for (int k = 1; k <= sub; k++) thr2[k] = sq_bound(thr[k]);
    thr2[kTableSize] = std::numeric_limits<float>::infinity();
    cut2 = sq_bound(h);
    uint32_t w_last;
    std::memcpy(&w_last, &tables[0 * kTableSize + sub], 4);   // W at slot 1000
    density_tail0 = w_last == 0u && thr2[sub] <= cut2;
    uint32_t sdw_last;
    std::memcpy(&sdw_last, &tables[3 * kTableSize + sub], 4);   // spiky gradient at slot 1000
    force_tail0 = (sdw_last & 0x7fffffffu) == 0u && thr[sub] <= h;
    float stepSize = 1.6f * p.particle_radius;
    float sum = 0.f;
    for (int i = -3; i <= 3; i++)
        for (int j = -3; j <= 3; j++)
            for (int k = -3; k <= 3; k++) {
                float x = i * stepSize, y = j * stepSize, z = k * stepSize;
                sum += look(0, std::sqrt(x * x + y * y + z * z));
            }
    mass = p.rest_density / sum;
    if (p.mass_override > 0.f) mass = p.mass_override;
    exact_tables = true;
    for (int t : {1, 2, 4})
        for (int i = 0; i <= sub; i++) {
            const float a = std::fabs(tables[t * kTableSize + i]);
            if (!(a == 0.f || (a >= 0x1p-29f && a <= 0x1p60f))) exact_tables = false;
        }
}

float HostKernels::look(int t, float d) const
{
    if (d >= h) return 0.f;
    int key = (int)(d / step);
    return tables[t * kTableSize + key];
}

// PCISPHSolver::calcDelta (PCISPHSolver.cpp:286-328). The lattice sum depends on the
// parameters only, so it is kept for the particle radius it was summed for (the engine asks
// for delta every step); beta and delta follow per time step, in the reference's order.
float HostKernels::delta(const lsp_params& p, float dt) const
{
    if (!(denom_ready_ && denom_radius_ == p.particle_radius)) {
        denom_ = lattice_denominator(p);
        denom_radius_ = p.particle_radius;
        denom_ready_ = true;
    }
    const float denom = denom_;
    float beta = dt * mass / p.rest_density;
    beta = 2.f * beta * beta;
    float delta = 0.f;
    if (std::fabs(denom) > 0.f) delta = -1.f / (beta * denom);
    return delta;
}

float HostKernels::lattice_denominator(const lsp_params& p) const
{
    float stepSize = 1.6f * p.particle_radius;
    float d1x = 0.f, d1y = 0.f, d1z = 0.f, d2 = 0.f;
    for (int i = -3; i <= 3; i++)
        for (int j = -3; j <= 3; j++)
            for (int k = -3; k <= 3; k++) {
                float x = i * stepSize, y = j * stepSize, z = k * stepSize;
                float dist = std::sqrt(x * x + y * y + z * z);
                if (dist > 0.f) {
                    float dx = x / dist, dy = y / dist, dz = z / dist;
                    float w = look(3, dist);
                    float gx = dx * w, gy = dy * w, gz = dz * w;
                    d1x += gx; d1y += gy; d1z += gz;
                    d2 += gx * gx + gy * gy + gz * gz;
                }
            }
    return -(d1x * d1x + d1y * d1y + d1z * d1z) - d2;
}

// ------------------------------------------------------------------ engine
void validate_params(const lsp_params& p)
{
    auto bad = [](const char* m) { throw Error(LSP_ERR_INVALID, m); };
    if (!(p.particle_radius > 0.f) || !std::isfinite(p.particle_radius)) bad("particle_radius must be > 0");
    if (!(p.kernel_radius_factor > 0.f) || !std::isfinite(p.kernel_radius_factor)) bad("kernel_radius_factor must be > 0");
    if (!(p.rest_density > 0.f) || !std::isfinite(p.rest_density)) bad("rest_density must be > 0");
    if (p.solver != LSP_SOLVER_SPH && p.solver != LSP_SOLVER_PCISPH) bad("solver must be LSP_SOLVER_SPH or LSP_SOLVER_PCISPH");
    if (p.pci_max_iterations < 0 || p.pci_max_iterations > kMaxIterationsCap) bad("pci_max_iterations out of range [0, 1024]");
    if (p.pci_min_iterations < 0) bad("pci_min_iterations must be >= 0");
    if (p.warm_start != LSP_WARM_ZERO && p.warm_start != LSP_WARM_MLP && p.warm_start != LSP_WARM_AUTO)
        bad("unknown warm_start");
    if (p.warm_auto_iterations < 0) bad("warm_auto_iterations must be >= 0");
    if (p.loop_mode != LSP_LOOP_PERSISTENT && p.loop_mode != LSP_LOOP_HOST) bad("unknown loop_mode");
}

Engine::Engine(const lsp_params& p, int device)
{
    validate_params(p);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw Error(LSP_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0) CK(cudaGetDevice(&device));
    if (device >= count) throw Error(LSP_ERR_NO_DEVICE, "device index out of range");
    dev_ = device;
    activate();
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, dev_));
    if (prop.major != 10) throw Error(LSP_ERR_NO_DEVICE, "liblsp is built for sm_100a (B200); device is sm_" +
                                                             std::to_string(prop.major) + std::to_string(prop.minor));
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    CK(cudaMallocHost((void**)&hstatus_, sizeof(DevStatus)));
    std::memset(hstatus_, 0, sizeof(DevStatus));
    status_.alloc(1);
    bounds_.alloc(6);
    loop_sync_.alloc(4);
    maxerr_.alloc(kMaxIterationsCap);
    prm_ = p;
    derive();
    mlp_.init(stream_);
}

Engine::~Engine()
{
    cudaSetDevice(dev_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (hstatus_) cudaFreeHost(hstatus_);
    for (cudaEvent_t e : evpool_) cudaEventDestroy(e);
    for (cudaEvent_t e : marks_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

void Engine::activate() const { CK(cudaSetDevice(dev_)); }

void Engine::derive()
{
    hk_.build(prm_);
    tables_dirty_ = true;
    grid_valid_ = false;   // cell size follows h
}

void Engine::set_params(const lsp_params& p)
{
    validate_params(p);
    bool geometry = p.particle_radius != prm_.particle_radius || p.kernel_radius_factor != prm_.kernel_radius_factor;
    prm_ = p;
    derive();
    auto_on_ = false;            // LSP_WARM_AUTO starts from the zero start again
    if (geometry) nbr_cap_ = 0;  // re-estimate the list capacity for the new h
}

void Engine::set_warm_start(int mode)
{
    lsp_params p = prm_;
    p.warm_start = mode;
    validate_params(p);
    prm_.warm_start = mode;
    auto_on_ = false;
}

static int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

void Engine::ensure_capacity(int64_t n)
{
    if (n <= cap_) return;
    activate();
    int64_t cap = round_up(std::max<int64_t>(n, cap_ + cap_ / 2), 256);
    DevArray<float4> np[4];
    DevArray<int32_t> nsoi;
    for (int k = 0; k < 4; k++) np[k].alloc(cap);
    nsoi.alloc(cap);
    DevArray<float4>* cur[4] = {&pos_[cur_], &vel_[cur_], &half_[cur_], &old_[cur_]};
    if (n_ > 0) {
        for (int k = 0; k < 4; k++)
            CK(cudaMemcpyAsync(np[k].p, cur[k]->p, n_ * sizeof(float4), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaMemcpyAsync(nsoi.p, slot_of_id_.p, n_ * sizeof(int32_t), cudaMemcpyDeviceToDevice, stream_));
    }
    CK(cudaStreamSynchronize(stream_));
    for (int k = 0; k < 4; k++) std::swap(cur[k]->p, np[k].p), std::swap(cur[k]->n, np[k].n);
    std::swap(slot_of_id_.p, nsoi.p), std::swap(slot_of_id_.n, nsoi.n);
    for (int k = 0; k < 4; k++) np[k].release();
    if (phist_[cur_].p) {
        DevArray<float4> nh;
        nh.alloc(cap);
        CK(cudaMemsetAsync(nh.p, 0, cap * sizeof(float4), stream_));
        if (n_ > 0) CK(cudaMemcpyAsync(nh.p, phist_[cur_].p, n_ * sizeof(float4), cudaMemcpyDeviceToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
        std::swap(phist_[cur_].p, nh.p);
        std::swap(phist_[cur_].n, nh.n);
        phist_[1 - cur_].alloc(cap);
        feat_.alloc(cap * kMlpIn);
        gradrho_.alloc(cap);
        tgt_.alloc(cap);
        features_valid_ = false;
    }
    pos_[1 - cur_].alloc(cap); vel_[1 - cur_].alloc(cap); half_[1 - cur_].alloc(cap); old_[1 - cur_].alloc(cap);
    force_.alloc(cap); ppos_.alloc(cap); ppos_alt_.alloc(cap); phalf_.alloc(cap); pforce_.alloc(cap);
    ppos_final_ = ppos_.p;
    rho_.alloc(cap); pres_.alloc(cap); prho_.alloc(cap); err_.alloc(cap); vrho_.alloc(cap);
    key_.alloc(cap); slot_.alloc(cap); sorted_key_.alloc(cap); tmp_.alloc(cap); nbr_count_.alloc(cap);
    stage_.alloc(cap * 12);
    CK(cudaMemsetAsync(force_.p, 0, cap * sizeof(float4), stream_));
    CK(cudaMemsetAsync(ppos_.p, 0, cap * sizeof(float4), stream_));
    CK(cudaMemsetAsync(ppos_alt_.p, 0, cap * sizeof(float4), stream_));
    CK(cudaMemsetAsync(phalf_.p, 0, cap * sizeof(float4), stream_));
    CK(cudaMemsetAsync(pforce_.p, 0, cap * sizeof(float4), stream_));
    for (DevArray<float>* a : {&rho_, &pres_, &prho_, &err_})
        CK(cudaMemsetAsync(a->p, 0, cap * sizeof(float), stream_));
    CK(cudaMemsetAsync(nbr_count_.p, 0, cap * sizeof(int32_t), stream_));
    cap_ = cap;
    if (nbr_cap_ > 0) ensure_neighbors(nbr_cap_);
    CK(cudaStreamSynchronize(stream_));
}

void Engine::ensure_neighbors(int cap)
{
    cap = (int)round_up(std::max(cap, 16), 8);
    if (cap > 4096) throw Error(LSP_ERR_CAPACITY, "neighbour count above 4096 per particle");
    nbr_stride_ = std::max<int64_t>(cap_, 256);
    nbr_.alloc((size_t)cap * (size_t)nbr_stride_);
    nbr_src_.alloc((size_t)cap * (size_t)nbr_stride_);
    nbr_cap_ = cap;
}

void Engine::add_particles(const float* xyz, const float* vel, int64_t m)
{
    if (m < 0 || (m > 0 && !xyz)) throw Error(LSP_ERR_INVALID, "add_particles: bad pointer or count");
    if (m == 0) return;
    if (n_ + m > (int64_t)INT32_MAX / 2) throw Error(LSP_ERR_CAPACITY, "particle count above 2^30");
    ensure_capacity(n_ + m);
    std::vector<float4> p(m), v(m), z(m, make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<int32_t> soi(m);
    for (int64_t i = 0; i < m; i++) {
        int32_t id = (int32_t)(n_ + i);
        float w;
        std::memcpy(&w, &id, 4);
        p[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], w);
        v[i] = vel ? make_float4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 1.f) : make_float4(0.f, 0.f, 0.f, 1.f);
        soi[i] = id;
    }
    activate();
    CK(cudaMemcpyAsync(pos_[cur_].p + n_, p.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(vel_[cur_].p + n_, v.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(half_[cur_].p + n_, z.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(old_[cur_].p + n_, z.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(slot_of_id_.p + n_, soi.data(), m * sizeof(int32_t), cudaMemcpyHostToDevice, stream_));
    if (phist_[cur_].p) CK(cudaMemsetAsync(phist_[cur_].p + n_, 0, m * sizeof(float4), stream_));
    CK(cudaStreamSynchronize(stream_));
    n_ += m;
    if (domain_from_particles_) grid_valid_ = false;
    stepped_ = false;   // the last step's lists, grid and features no longer cover every particle
}

void Engine::remove_particles()
{
    n_ = 0;
    if (domain_from_particles_) grid_valid_ = false;
    stepped_ = false;
}

int Engine::add_collider(const Collider& c)
{
    if ((int)cols_.size() >= kMaxColliders) throw Error(LSP_ERR_CAPACITY, "more than 64 colliders");
    cols_.push_back(c);
    cols_dirty_ = true;
    if (!domain_user_ && c.boundary) grid_valid_ = false;
    return (int)cols_.size() - 1;
}

void Engine::update_collider(int index, const Collider& c)
{
    if (index < 0 || index >= (int)cols_.size()) throw Error(LSP_ERR_INVALID, "collider index out of range");
    if (cols_[index].sphere != c.sphere) throw Error(LSP_ERR_INVALID, "collider kind mismatch");
    Collider u = c;
    u.boundary = cols_[index].boundary;
    cols_[index] = u;
    cols_dirty_ = true;
}

void Engine::remove_colliders()
{
    cols_.clear();
    cols_dirty_ = true;
    if (!domain_user_) grid_valid_ = false;
}

void Engine::set_domain(const float lo[3], const float hi[3])
{
    for (int a = 0; a < 3; a++)
        if (!(hi[a] >= lo[a]) || !std::isfinite(lo[a]) || !std::isfinite(hi[a]))
            throw Error(LSP_ERR_INVALID, "domain: need finite lo <= hi");
    std::memcpy(dom_lo_, lo, sizeof(dom_lo_));
    std::memcpy(dom_hi_, hi, sizeof(dom_hi_));
    domain_user_ = true;
    grid_valid_ = false;
}

void Engine::upload_colliders()
{
    activate();
    if (dcols_.n < (size_t)kMaxColliders) dcols_.alloc(kMaxColliders);
    if (!cols_.empty())
        CK(cudaMemcpyAsync(dcols_.p, cols_.data(), cols_.size() * sizeof(Collider), cudaMemcpyHostToDevice, stream_));
    cols_dirty_ = false;
}

// Grid box: the user domain, else the union of boundary colliders, else the particle
// bounds plus a margin. Cells are the reference CPU grid's, c = (int)(x / h).
void Engine::ensure_grid()
{
    if (grid_valid_) return;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool have = false;
    domain_from_particles_ = false;
    if (domain_user_) {
        std::memcpy(lo, dom_lo_, sizeof(lo));
        std::memcpy(hi, dom_hi_, sizeof(hi));
        have = true;
    } else {
        have = boundary_box(cols_, lo, hi);
    }
    if (!have && n_ > 0) {
        activate();
        int32_t init[6] = {INT32_MAX, INT32_MAX, INT32_MAX, INT32_MIN, INT32_MIN, INT32_MIN};
        CK(cudaMemcpyAsync(bounds_.p, init, sizeof(init), cudaMemcpyHostToDevice, stream_));
        launch_bounds(pos_[cur_].p, n_, bounds_.p, stream_);
        int32_t out[6];
        CK(cudaMemcpyAsync(out, bounds_.p, sizeof(out), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        for (int a = 0; a < 6; a++) {
            int32_t v = out[a] >= 0 ? out[a] : (out[a] ^ 0x7fffffff);
            float f;
            std::memcpy(&f, &v, 4);
            if (a < 3) lo[a] = f; else hi[a - 3] = f;
        }
        for (int a = 0; a < 3; a++) {
            if (!(lo[a] <= hi[a])) { lo[a] = 0.f; hi[a] = 0.f; }
            float margin = std::max(0.25f * (hi[a] - lo[a]), 4.f * hk_.h);
            lo[a] -= margin;
            hi[a] += margin;
        }
        domain_from_particles_ = true;
    }
    const int64_t cells = grid_from_box(lo, hi, hk_.h, org_, dim_);
    cells_ = cells;
    if (cells + 1 > cells_alloc_) {
        activate();
        // The scan reads and writes the histogram and cell table 8 entries at a time: both
        // are padded to a multiple of 8 with zeros (scan_entries).
        const int64_t alloc = scan_entries(cells + 1);
        hist_.alloc(alloc);
        cell_start_.alloc(alloc);
        tile_sums_.alloc(scan_tiles(cells + 1) + 1);
        CK(cudaMemsetAsync(hist_.p, 0, alloc * sizeof(uint32_t), stream_));
        CK(cudaMemsetAsync(cell_start_.p, 0, alloc * sizeof(uint32_t), stream_));
        cells_alloc_ = alloc;
    }
    grid_valid_ = true;
}

bool boundary_box(const std::vector<Collider>& cols, float lo[3], float hi[3])
{
    bool have = false;
    for (const Collider& c : cols) {
        if (!c.boundary) continue;
        float cc[3] = {c.cx, c.cy, c.cz};
        float e[3] = {c.hx, c.hy, c.hz};
        if (c.sphere) e[0] = e[1] = e[2] = c.radius;
        for (int a = 0; a < 3; a++) {
            float l = cc[a] - std::fabs(e[a]), u = cc[a] + std::fabs(e[a]);
            lo[a] = have ? std::min(lo[a], l) : l;
            hi[a] = have ? std::max(hi[a], u) : u;
        }
        have = true;
    }
    return have;
}

int64_t grid_from_box(const float lo[3], const float hi[3], float h, int32_t org[3], int32_t dim[3])
{
    int64_t cells = 1;
    for (int a = 0; a < 3; a++) {
        int c0 = (int)(lo[a] / h), c1 = (int)(hi[a] / h);
        org[a] = c0;
        dim[a] = std::max(1, c1 - c0 + 1);
        cells *= dim[a];
    }
    if (cells > ((int64_t)1 << 30)) throw Error(LSP_ERR_CAPACITY, "grid box holds more than 2^30 cells of size h");
    return cells;
}

DevParams physics_params(const lsp_params& p, const HostKernels& hk, float dt)
{
    DevParams P{};
    P.gx = p.gravity[0]; P.gy = p.gravity[1]; P.gz = p.gravity[2];
    P.h = hk.h;
    P.h2 = hk.h * hk.h;
    P.cut2 = hk.cut2;
    P.step = hk.step;
    P.inv_step = 1.f / hk.step;
    P.radius = p.particle_radius;
    P.mass = hk.mass;
    P.rho0 = p.rest_density;
    P.stiffness = p.stiffness;
    P.neg = p.negative_pressure_factor;
    P.viscosity = p.viscosity;
    P.sigma = p.surface_tension;
    P.sigma_thr = p.surface_tension_threshold;
    P.restitution = p.restitution;
    P.friction = p.friction;
    P.delta = p.solver == LSP_SOLVER_PCISPH ? hk.delta(p, dt) : 0.f;
    P.eta = p.pci_eta;
    P.dt = dt;
    P.keep_initial_velocity = p.keep_initial_velocity;
    P.min_it = p.pci_min_iterations;
    P.max_it = p.pci_max_iterations;
    P.exact_tables = hk.exact_tables ? 1 : 0;
    P.density_tail0 = hk.density_tail0 ? 1 : 0;
    P.force_tail0 = hk.force_tail0 ? 1 : 0;
    return P;
}

DevParams Engine::device_params(float dt) const
{
    DevParams P = physics_params(prm_, hk_, dt);
    P.n = (int)n_;
    P.ncoll = (int)cols_.size();
    P.ox = org_[0]; P.oy = org_[1]; P.oz = org_[2];
    P.nx = dim_[0]; P.ny = dim_[1]; P.nz = dim_[2];
    P.cells = (uint32_t)cells_;
    P.nbr_cap = nbr_cap_;
    P.nbr_stride = nbr_stride_;
    return P;
}

StepBuffers Engine::buffers()
{
    StepBuffers b{};
    b.pos = pos_[cur_].p; b.vel = vel_[cur_].p; b.half = half_[cur_].p; b.old = old_[cur_].p;
    b.force = force_.p; b.rho = rho_.p; b.pres = pres_.p;
    b.ppos = ppos_.p; b.phalf = phalf_.p; b.pforce = pforce_.p; b.prho = prho_.p; b.err = err_.p;
    b.nbr = nbr_.p; b.nbr_count = nbr_count_.p; b.nbr_src = nbr_src_.p; b.nbr_out = nbr_.p; b.vrho = vrho_.p;
    b.tables = tables_.p; b.colliders = dcols_.p; b.status = status_.p;
    b.hist = phist_[cur_].p;
    b.gradrho = features_on() ? gradrho_.p : nullptr;
    return b;
}

template <typename F>
void Engine::timed(int cls, F&& launch)
{
    if (!profile_) {
        launches_ += launch();
        return;
    }
    // The event pairs are summed when the profile is read (profile_read / profile), not
    // after every step, so a profiled step adds only the event records; a long profiled run
    // folds its backlog in every 1024 launches.
    if (pending_.size() >= 1024) {
        CK(cudaStreamSynchronize(stream_));
        collect_profile();
    }
    while (evpool_.size() < evnext_ + 2) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        evpool_.push_back(e);
    }
    size_t first = evnext_;
    evnext_ += 2;
    CK(cudaEventRecord(evpool_[first], stream_));
    int n = launch();
    CK(cudaEventRecord(evpool_[first + 1], stream_));
    launches_ += n;
    prof_n_[cls] += n;
    pending_.push_back({cls, first});
}

// Called after a stream synchronisation: folds the bracketed intervals into the totals.
void Engine::collect_profile()
{
    for (auto& pr : pending_) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, evpool_[pr.second], evpool_[pr.second + 1]));
        prof_ms_[pr.first] += ms;
    }
    pending_.clear();
    evnext_ = 0;
}

void Engine::profile(bool on)
{
    activate();
    CK(cudaStreamSynchronize(stream_));
    collect_profile();
    profile_ = on;
    for (int k = 0; k < LSP_PROF_COUNT; k++) { prof_ms_[k] = 0.0; prof_n_[k] = 0; }
}

void Engine::profile_read(double* ms, int64_t* launches, int capacity)
{
    activate();
    CK(cudaStreamSynchronize(stream_));
    collect_profile();
    for (int k = 0; k < LSP_PROF_COUNT && k < capacity; k++) {
        if (ms) ms[k] = prof_ms_[k];
        if (launches) launches[k] = prof_n_[k];
    }
}

void Engine::timer_mark(int slot)
{
    if (slot < 0 || slot >= 16) throw Error(LSP_ERR_INVALID, "timer slot must be in [0, 16)");
    activate();
    if (!marks_[slot]) CK(cudaEventCreate(&marks_[slot]));
    CK(cudaEventRecord(marks_[slot], stream_));
}

float Engine::timer_elapsed(int a, int b)
{
    if (a < 0 || a >= 16 || b < 0 || b >= 16 || !marks_[a] || !marks_[b])
        throw Error(LSP_ERR_INVALID, "timer slots not marked");
    activate();
    CK(cudaEventSynchronize(marks_[b]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, marks_[a], marks_[b]));
    return ms;
}

bool Engine::features_on() const
{
    return prm_.solver == LSP_SOLVER_PCISPH && (record_ || warm_on());
}

bool Engine::history_on() const
{
    // LSP_WARM_AUTO keeps the pressure history (the features' three previous pressures)
    // from the first step, so that the learned guess has it when the mode switches it on;
    // the features themselves are computed only once the guess is on.
    return prm_.solver == LSP_SOLVER_PCISPH && (record_ || prm_.warm_start != LSP_WARM_ZERO);
}

bool Engine::warm_on() const
{
    return prm_.warm_start == LSP_WARM_MLP || (prm_.warm_start == LSP_WARM_AUTO && auto_on_);
}

bool Engine::pcisph_loop(const DevParams& P, const StepBuffers& b, lsp_step_stats* st)
{
    ppos_final_ = ppos_.p;
    if (P.max_it <= 0) {
        CK(cudaMemsetAsync(pforce_.p, 0, n_ * sizeof(float4), stream_));
        if (st) { st->iterations = 0; st->converged = 0; st->max_density_error_ratio = 0.0; }
        return false;
    }
    const bool feats = features_on();
    const bool warm = warm_on();
    WarmArgs w{};
    if (feats) {
        w.feat = feat_.p;
        w.hist = phist_[cur_].p;
        w.gradrho = gradrho_.p;
        w.p_scale = P.delta * 0.01f * P.rho0;
        last_p_scale_ = w.p_scale;
        features_valid_ = true;
    }
    if (prm_.loop_mode == LSP_LOOP_PERSISTENT) {
        CK(cudaMemsetAsync(loop_sync_.p, 0, 4 * sizeof(uint32_t), stream_));
        CK(cudaMemsetAsync(maxerr_.p, 0, (size_t)(P.max_it + 4) * sizeof(uint32_t), stream_));
        if (feats) {
            w.maxerr0 = maxerr_.p;
            timed(LSP_PROF_PCI_PREDICT, [&] { launch_pci_predict(P, b, 0, stream_); return 1; });
            timed(LSP_PROF_WARM_START, [&] {
                launch_pci_density_first(P, b, w, stream_);
                if (warm) launch_warm_guess_tc(mlp_.umma(), P, b, feat_.p, stream_);
                return warm ? 2 : 1;
            });
        }
        bool ok = false;
        int grid = 0;
        timed(LSP_PROF_PCI_LOOP, [&] {
            ok = launch_pci_loop(P, b, ppos_alt_.p, loop_sync_.p, maxerr_.p, feats ? 1 : 0, warm ? 1 : 0, stream_,
                                 &grid);
            return ok ? 1 : 0;
        });
        if (ok) return true;
        cudaGetLastError();   // the device refused the cooperative launch: run the per-phase loop
        if (feats) throw Error(LSP_ERR_CUDA, "cooperative launch of the PCISPH loop was refused");
    }
    // Per-phase loop; the convergence test reads the iteration's maximum back every time.
    auto read_err = [&]() {
        float e;
        CK(cudaMemcpyAsync(&hstatus_->max_err_bits, &status_.p->max_err_bits, sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        std::memcpy(&e, &hstatus_->max_err_bits, 4);
        return e;
    };
    int k = 0, passes = 1;
    bool conv = false, rejected = false;
    timed(LSP_PROF_PCI_PREDICT, [&] { launch_pci_predict(P, b, 0, stream_); return 1; });
    if (feats) {
        w.maxerr0 = &status_.p->max_err_bits;
        timed(LSP_PROF_WARM_START, [&] {
            launch_pci_density_first(P, b, w, stream_);
            if (warm) launch_warm_guess_tc(mlp_.umma(), P, b, feat_.p, stream_);
            return warm ? 2 : 1;
        });
    } else {
        timed(LSP_PROF_PCI_DENSITY, [&] { launch_pci_density(P, b, 0, stream_); return 1; });
    }
    float e = read_err(), e0 = e;
    for (;;) {
        if (warm && !rejected && k == 1 && e > e0) {
            // The learned guess raised the error: restart from zero pressure (the plain loop).
            rejected = true;
            k = 0;
            passes++;
            timed(LSP_PROF_PCI_PREDICT, [&] { launch_pci_predict(P, b, 0, stream_); return 1; });
            timed(LSP_PROF_PCI_DENSITY, [&] { launch_pci_density(P, b, 0, stream_); return 1; });
            e = read_err();
            continue;
        }
        conv = std::fabs(e / prm_.rest_density) < prm_.pci_eta;
        // A learned guess is only checked at iteration 1, so a warm step cannot stop at 0.
        const bool unverified = warm && !rejected && k == 0;
        const bool done = (conv && k + 1 >= P.min_it && !unverified) || (k + 1 >= P.max_it);
        timed(LSP_PROF_PCI_FORCE, [&] { launch_pci_force(P, b, stream_); return 1; });
        if (done) break;
        k++;
        passes++;
        timed(LSP_PROF_PCI_PREDICT, [&] { launch_pci_predict(P, b, k, stream_); return 1; });
        timed(LSP_PROF_PCI_DENSITY, [&] { launch_pci_density(P, b, k, stream_); return 1; });
        if (k == 1) e0 = e;
        e = read_err();
    }
    if (st) {
        st->iterations = passes;
        st->converged = conv ? 1 : 0;
        st->max_density_error_ratio = (double)e / (double)prm_.rest_density;
        st->warm_start_used = (warm && !rejected) ? 1 : 0;
        st->warm_start_tried = warm ? 1 : 0;
    }
    return false;
}

int initial_neighbor_capacity(const lsp_params& p)
{
    // Lattice estimate (4/3) pi (h/s)^3 with s = 1.6 r, doubled for compression.
    double q = p.kernel_radius_factor / 1.6;
    double est = 4.18879 * q * q * q;
    return (int)std::min(4096.0, std::ceil(2.0 * est) + 16.0);
}

// At least 1.5x the count that overflowed and twice the old capacity, capped at the 4096
// limit (unless the count itself is above it, which ensure_neighbors rejects). Every
// regrowth frees and reallocates the whole list and redoes the step, and a large
// cudaFree / cudaMalloc pair has been measured to take anywhere from 15 to 600 ms, so few
// large steps beat many small ones.
int warm_auto_switch(const lsp_params& p)
{
    return p.warm_auto_iterations > 0 ? p.warm_auto_iterations : std::max(12, p.pci_max_iterations / 2);
}

int grown_neighbor_capacity(int needed, int current)
{
    const int64_t c = std::max<int64_t>((int64_t)needed + needed / 2 + 8, 2 * (int64_t)current);
    return (int)std::max<int64_t>(needed, std::min<int64_t>(c, 4096));
}

void Engine::run_step(float dt, lsp_step_stats* st)
{
    if (st) std::memset(st, 0, sizeof(*st));
    if (!(dt > 0.f) || !std::isfinite(dt)) throw Error(LSP_ERR_INVALID, "dt must be finite and > 0");
    if (n_ == 0) {
        if (st) st->converged = 1;
        return;
    }
    activate();
    ensure_grid();
    if (cols_dirty_) upload_colliders();
    if (tables_dirty_) {
        if (!tables_.p) tables_.alloc(hk_.tables.size());
        CK(cudaMemcpyAsync(tables_.p, hk_.tables.data(), hk_.tables.size() * sizeof(float), cudaMemcpyHostToDevice,
                           stream_));
        tables_dirty_ = false;
    }
    if (!dcols_.p) upload_colliders();
    if (history_on()) ensure_warm_buffers();
    if (nbr_cap_ == 0 || nbr_stride_ < cap_) ensure_neighbors(nbr_cap_ ? nbr_cap_ : initial_neighbor_capacity(prm_));
    lsp_step_stats local{};
    bool device_loop = false;
    for (int attempt = 0;; attempt++) {
        device_loop = false;
        DevParams P = device_params(dt);
        CK(cudaMemsetAsync(status_.p, 0, sizeof(DevStatus), stream_));
        GridBuildArgs g{};
        g.P = P;
        g.pos_in = pos_[cur_].p; g.vel_in = vel_[cur_].p; g.half_in = half_[cur_].p; g.old_in = old_[cur_].p;
        g.pos_out = pos_[1 - cur_].p; g.vel_out = vel_[1 - cur_].p;
        g.half_out = half_[1 - cur_].p; g.old_out = old_[1 - cur_].p;
        g.key = key_.p; g.slot = slot_.p; g.hist = hist_.p; g.tile_sums = tile_sums_.p; g.cell_start = cell_start_.p;
        g.tmp = tmp_.p; g.slot_of_id = slot_of_id_.p; g.sorted_key = sorted_key_.p;
        g.hist_in = phist_[cur_].p; g.hist_out = phist_[1 - cur_].p;
        g.nbr = nbr_src_.p; g.nbr_count = nbr_count_.p; g.status = status_.p;
        // The neighbour build also sums the start-of-step density (k_neighbors_density).
        g.tables = tables_.p; g.rho = rho_.p; g.pres = pres_.p; g.vrho = vrho_.p;
        timed(LSP_PROF_GRID_SORT, [&] { return launch_grid_keys(g, stream_); });
        timed(LSP_PROF_GRID_SCAN, [&] { return launch_grid_scan(g, stream_); });
        timed(LSP_PROF_GRID_SCATTER, [&] { return launch_grid_scatter(g, stream_); });
        timed(LSP_PROF_GRID_GATHER, [&] { return launch_grid_gather(g, stream_); });
        timed(LSP_PROF_NEIGHBORS, [&] { return launch_neighbors(g, stream_); });
        cur_ = 1 - cur_;
        StepBuffers b = buffers();
        timed(LSP_PROF_NONPRESSURE, [&] { launch_nonpressure(P, b, stream_); return 1; });
        if (prm_.solver == LSP_SOLVER_SPH) {
            timed(LSP_PROF_SPH_PRESSURE, [&] { launch_sph_pressure(P, b, stream_); return 1; });
            timed(LSP_PROF_INTEGRATE, [&] { launch_integrate_collide(P, b, false, stream_); return 1; });
            local.iterations = 0;
            local.converged = 1;
        } else {
            device_loop = pcisph_loop(P, b, &local);
            // The persistent loop integrates in its last pass; the per-phase loop does not.
            if (!device_loop)
                timed(LSP_PROF_INTEGRATE, [&] { launch_integrate_collide(P, b, true, stream_); return 1; });
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hstatus_, status_.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        if ((hstatus_->error_flags & kErrNeighborOverflow) && attempt < 3) {
            cur_ = 1 - cur_;   // the gather left the pre-step state untouched: redo the step
            ensure_neighbors(grown_neighbor_capacity((int)hstatus_->max_neighbors, nbr_cap_));
            continue;
        }
        break;
    }
    stepped_ = true;
    if (device_loop) {
        float me;
        std::memcpy(&me, &hstatus_->max_err_bits, 4);
        local.iterations = hstatus_->iterations;
        local.converged = hstatus_->converged;
        local.max_density_error_ratio = (double)me / (double)prm_.rest_density;
        local.warm_start_used = hstatus_->warm_used;
        local.warm_start_tried = warm_on() ? 1 : 0;
        ppos_final_ = (hstatus_->last_k & 1) ? ppos_alt_.p : ppos_.p;
    }
    local.max_neighbors = (int32_t)hstatus_->max_neighbors;
    local.escaped = (int32_t)hstatus_->escaped;
    if (st) *st = local;
    // LSP_WARM_AUTO: a zero-start step that needed more iterations than the switch point, or
    // missed eta, turns the learned guess on from the next step.
    if (prm_.warm_start == LSP_WARM_AUTO && !auto_on_ && prm_.solver == LSP_SOLVER_PCISPH &&
        (local.iterations > warm_auto_switch(prm_) || !local.converged))
        auto_on_ = true;
    if (hstatus_->escaped && domain_from_particles_) grid_valid_ = false;
    if (hstatus_->error_flags & kErrTimeout)
        throw Error(LSP_ERR_TIMEOUT, "a grid barrier of the persistent PCISPH loop gave up");
    if (hstatus_->error_flags & kErrNeighborOverflow)
        throw Error(LSP_ERR_CAPACITY, "neighbour list overflow persisted after resizing");
    if (hstatus_->error_flags & kErrScan)
        throw Error(LSP_ERR_CAPACITY, "a grid cell holds more than 4096 particles");
    if (hstatus_->error_flags & kErrNaN)
        throw Error(LSP_ERR_DEVICE_STATUS, "non-finite particle position at the start of the step");
    if (prm_.solver == LSP_SOLVER_PCISPH && prm_.strict_convergence && !local.converged)
        throw Error(LSP_ERR_NOT_CONVERGED, "PCISPH reached max iterations above eta");
}

void Engine::step(float dt, lsp_step_stats* st) { run_step(dt, st); }

void Engine::step_many(float dt, int steps, lsp_step_stats* st)
{
    if (steps < 0) throw Error(LSP_ERR_INVALID, "steps must be >= 0");
    for (int s = 0; s < steps; s++) run_step(dt, st);
}

void Engine::synchronize()
{
    activate();
    CK(cudaStreamSynchronize(stream_));
}

void Engine::stage(size_t floats)
{
    if (stage_.n < floats) stage_.alloc(floats);
}

void Engine::read_field(int field, float* out, int64_t n)
{
    if (!out || n != n_) throw Error(LSP_ERR_INVALID, "read_field: n must equal the particle count");
    if (n == 0) return;
    activate();
    const void* src = nullptr;
    int comps = 1, mode = 0;
    switch (field) {
    case LSP_FIELD_POSITION: src = pos_[cur_].p; comps = 3; break;
    case LSP_FIELD_VELOCITY: src = vel_[cur_].p; comps = 3; break;
    case LSP_FIELD_HALF_VELOCITY: src = half_[cur_].p; comps = 3; break;
    case LSP_FIELD_OLD_HALF_VELOCITY: src = old_[cur_].p; comps = 3; break;
    case LSP_FIELD_PRED_POSITION: src = ppos_final_ ? ppos_final_ : ppos_.p; comps = 3; break;
    case LSP_FIELD_PRED_HALF_VELOCITY: src = phalf_.p; comps = 3; break;
    case LSP_FIELD_PRED_PRESSURE_FORCE: src = pforce_.p; comps = 3; break;
    case LSP_FIELD_DENSITY: src = rho_.p; break;
    case LSP_FIELD_PRESSURE: src = pres_.p; break;
    case LSP_FIELD_PRED_DENSITY: src = prho_.p; break;
    case LSP_FIELD_DENSITY_ERROR: src = err_.p; break;
    case LSP_FIELD_FIRST_STEP: src = vel_[cur_].p; mode = 1; break;
    case LSP_FIELD_SPEED_SQUARED: src = vel_[cur_].p; mode = 2; break;
    case LSP_FIELD_NEIGHBOR_COUNT: break;
    default: throw Error(LSP_ERR_INVALID, "unknown field");
    }
    stage((size_t)n * comps);
    if (field == LSP_FIELD_NEIGHBOR_COUNT)
        launch_gather_count(nbr_count_.p, slot_of_id_.p, stage_.p, n, stream_);
    else
        launch_gather_field(src, comps, mode, slot_of_id_.p, stage_.p, n, stream_);
    CK(cudaMemcpyAsync(out, stage_.p, (size_t)n * comps * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void Engine::read_state(float* x, float* v, float* half, float* old, int32_t* first, int64_t n)
{
    if (n != n_ || !x || !v || !half || !old || !first) throw Error(LSP_ERR_INVALID, "read_state: bad arguments");
    if (n == 0) return;
    activate();
    stage((size_t)n * 13);
    float* s = stage_.p;
    launch_gather_state(pos_[cur_].p, vel_[cur_].p, half_[cur_].p, old_[cur_].p, slot_of_id_.p, s, s + 3 * n,
                        s + 6 * n, s + 9 * n, (int32_t*)(s + 12 * n), n, stream_);
    size_t b3 = (size_t)n * 3 * sizeof(float);
    CK(cudaMemcpyAsync(x, s, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(v, s + 3 * n, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(half, s + 6 * n, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(old, s + 9 * n, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(first, s + 12 * n, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void Engine::write_state(const float* x, const float* v, const float* half, const float* old, const int32_t* first,
                         int64_t n)
{
    if (n != n_ || !x || !v || !half || !old || !first) throw Error(LSP_ERR_INVALID, "write_state: bad arguments");
    if (n == 0) return;
    activate();
    stage((size_t)n * 13);
    float* s = stage_.p;
    size_t b3 = (size_t)n * 3 * sizeof(float);
    CK(cudaMemcpyAsync(s, x, b3, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(s + 3 * n, v, b3, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(s + 6 * n, half, b3, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(s + 9 * n, old, b3, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(s + 12 * n, first, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, stream_));
    launch_scatter_state(s, s + 3 * n, s + 6 * n, s + 9 * n, (const int32_t*)(s + 12 * n), slot_of_id_.p,
                         pos_[cur_].p, vel_[cur_].p, half_[cur_].p, old_[cur_].p, n, stream_);
    CK(cudaStreamSynchronize(stream_));
    if (domain_from_particles_) grid_valid_ = false;
}

bool Engine::domain(float lo[3], float hi[3]) const
{
    std::memcpy(lo, dom_lo_, sizeof(dom_lo_));
    std::memcpy(hi, dom_hi_, sizeof(dom_hi_));
    return domain_user_;
}

void Engine::read_history(float* out, int64_t n)
{
    if (!out || n != n_) throw Error(LSP_ERR_INVALID, "read_history: n must equal the particle count");
    if (n == 0) return;
    if (!phist_[cur_].p) {
        std::memset(out, 0, (size_t)n * 3 * sizeof(float));
        return;
    }
    activate();
    stage((size_t)n * 3);
    launch_gather_field(phist_[cur_].p, 3, 0, slot_of_id_.p, stage_.p, n, stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, stage_.p, (size_t)n * 3 * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void Engine::write_history(const float* in, int64_t n)
{
    if (!in || n != n_) throw Error(LSP_ERR_INVALID, "write_history: n must equal the particle count");
    if (n == 0) return;
    activate();
    ensure_warm_buffers();
    stage((size_t)n * 3);
    CK(cudaMemcpyAsync(stage_.p, in, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, stream_));
    launch_scatter_vec(stage_.p, slot_of_id_.p, phist_[cur_].p, n, stream_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
}

void Engine::read_neighbors(int64_t* offsets, int32_t* index, int64_t n, int64_t capacity)
{
    if (n != n_ || !offsets) throw Error(LSP_ERR_INVALID, "read_neighbors: bad arguments");
    if (!stepped_) throw Error(LSP_ERR_STATE, "read_neighbors: no step has run");
    std::vector<float> counts(n);
    read_field(LSP_FIELD_NEIGHBOR_COUNT, counts.data(), n);
    offsets[0] = 0;
    for (int64_t i = 0; i < n; i++) offsets[i + 1] = offsets[i] + (int64_t)counts[i];
    if (!index) return;
    if (capacity < offsets[n]) throw Error(LSP_ERR_INVALID, "read_neighbors: index capacity too small");
    activate();
    DevArray<int64_t> doff;
    DevArray<int32_t> dout;
    doff.alloc(n + 1);
    dout.alloc(std::max<int64_t>(offsets[n], 1));
    CK(cudaMemcpyAsync(doff.p, offsets, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    launch_neighbor_export(nbr_.p, nbr_count_.p, nbr_stride_, pos_[cur_].p, slot_of_id_.p, doff.p, dout.p, n, stream_);
    CK(cudaMemcpyAsync(index, dout.p, offsets[n] * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void Engine::grid_info(int32_t dims[3], int32_t origin[3], int64_t* cells) const
{
    for (int a = 0; a < 3; a++) {
        if (dims) dims[a] = dim_[a];
        if (origin) origin[a] = org_[a];
    }
    if (cells) *cells = cells_;
}

void Engine::read_grid(uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start, int64_t cells_plus_one)
{
    if (n != n_) throw Error(LSP_ERR_INVALID, "read_grid: n must equal the particle count");
    if (!stepped_) throw Error(LSP_ERR_STATE, "read_grid: no step has run");
    activate();
    if (keys) CK(cudaMemcpyAsync(keys, sorted_key_.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    if (ids) {
        std::vector<float4> p(n);
        CK(cudaMemcpyAsync(p.data(), pos_[cur_].p, n * sizeof(float4), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        for (int64_t i = 0; i < n; i++) std::memcpy(&ids[i], &p[i].w, 4);
    }
    if (cell_start) {
        if (cells_plus_one != cells_ + 1) throw Error(LSP_ERR_INVALID, "read_grid: cell table size mismatch");
        CK(cudaMemcpyAsync(cell_start, cell_start_.p, cells_plus_one * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           stream_));
    }
    CK(cudaStreamSynchronize(stream_));
}

// ------------------------------------------------------------------ learned warm start

void Engine::ensure_warm_buffers()
{
    if (phist_[cur_].p || cap_ == 0) return;
    activate();
    for (int k = 0; k < 2; k++) {
        phist_[k].alloc(cap_);
        CK(cudaMemsetAsync(phist_[k].p, 0, cap_ * sizeof(float4), stream_));
    }
    feat_.alloc(cap_ * kMlpIn);
    gradrho_.alloc(cap_);
    tgt_.alloc(cap_);
    CK(cudaMemsetAsync(feat_.p, 0, cap_ * kMlpIn * sizeof(float), stream_));
    CK(cudaMemsetAsync(gradrho_.p, 0, cap_ * sizeof(float), stream_));
}

void Engine::mlp_reset(uint64_t seed)
{
    activate();
    mlp_.reset(seed);
}

void Engine::mlp_set(const float* w, int n)
{
    activate();
    mlp_.set(w, n);
}

void Engine::mlp_get(float* w, int n)
{
    activate();
    mlp_.get(w, n);
}

void Engine::mlp_set_loss_asymmetry(float w) { mlp_.set_over_weight(w); }

void Engine::mlp_record(bool on)
{
    record_ = on;
    if (on) ensure_warm_buffers();
}

// Adam steps on the features and final pressures of the last step (targets p / p_scale).
float Engine::mlp_train(int iterations, int batch, float lr, uint64_t seed)
{
    if (!features_valid_ || !stepped_ || n_ == 0)
        throw Error(LSP_ERR_STATE, "mlp_train needs a PCISPH step that recorded features (lsp_mlp_record)");
    if (iterations <= 0 || batch <= 0) throw Error(LSP_ERR_INVALID, "iterations and batch must be > 0");
    activate();
    launch_scale(pres_.p, tgt_.p, n_, 1.f / last_p_scale_, stream_);
    return mlp_.train(feat_.p, tgt_.p, n_, iterations, batch, lr, seed);
}

void Engine::mlp_forward(const float* feat, int64_t n, float* out)
{
    activate();
    mlp_.forward(feat, n, out);
}

float Engine::mlp_gradient(const float* feat, const float* target, int64_t n, float* grad)
{
    activate();
    return mlp_.gradient(feat, target, n, grad);
}

void Engine::read_features(float* out, int64_t n)
{
    if (!out || n != n_) throw Error(LSP_ERR_INVALID, "read_features: n must equal the particle count");
    if (!features_valid_) throw Error(LSP_ERR_STATE, "no step has recorded features");
    activate();
    stage((size_t)n * kMlpIn);
    launch_gather_rows(feat_.p, kMlpIn, slot_of_id_.p, stage_.p, n, stream_);
    CK(cudaMemcpyAsync(out, stage_.p, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

}  // namespace lsp
