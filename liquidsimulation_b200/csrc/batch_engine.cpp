// Batch of independent scenes: layout, step sequencing, CUDA graph, autotuner.
// See batch_engine.h and batch_kernels.h.
#include "batch_engine.h"
#include "mlp.cuh"
#include "mlp_tc.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace lsp {

#define CK(call) LSP_CK(call)

static int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

BatchEngine::BatchEngine(int device)
{
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
    mlp_.init(stream_);
}

BatchEngine::~BatchEngine()
{
    cudaSetDevice(dev_);
    if (stream_) cudaStreamSynchronize(stream_);
    drop_graphs();
    if (hparams_) cudaFreeHost(hparams_);
    if (hstatus_) cudaFreeHost(hstatus_);
    for (cudaEvent_t e : marks_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

void BatchEngine::activate() const { CK(cudaSetDevice(dev_)); }

const BatchEngine::Scene& BatchEngine::at(int scene) const
{
    if (scene < 0 || scene >= (int)sc_.size()) throw Error(LSP_ERR_INVALID, "scene index out of range");
    return sc_[scene];
}
BatchEngine::Scene& BatchEngine::at(int scene)
{
    if (scene < 0 || scene >= (int)sc_.size()) throw Error(LSP_ERR_INVALID, "scene index out of range");
    return sc_[scene];
}

int BatchEngine::add_scene(const lsp_params& p, const float* xyz, const float* vel, int64_t n, const float* lo,
                           const float* hi)
{
    if (built_) throw Error(LSP_ERR_STATE, "scenes are added before the batch's first step");
    validate_params(p);
    if (n < 1 || !xyz) throw Error(LSP_ERR_INVALID, "a scene needs n >= 1 particles and positions");
    if ((lo == nullptr) != (hi == nullptr)) throw Error(LSP_ERR_INVALID, "domain: give both lo and hi or neither");
    if ((int)sc_.size() >= kMaxBatchScenes) throw Error(LSP_ERR_CAPACITY, "more than 4096 scenes in a batch");
    if (n_ + n > (int64_t)INT32_MAX / 2) throw Error(LSP_ERR_CAPACITY, "batch particle count above 2^30");
    const bool pci = p.solver == LSP_SOLVER_PCISPH;
    if (!sc_.empty() && pci != pcisph_) throw Error(LSP_ERR_INVALID, "all scenes of a batch use the same solver");
    if (pci && p.pci_max_iterations < 1) throw Error(LSP_ERR_INVALID, "batched PCISPH needs pci_max_iterations >= 1");
    if (p.warm_start != LSP_WARM_ZERO)
        throw Error(LSP_ERR_INVALID, "a batch's warm start is set for all scenes (lsp_batch_set_warm_start)");
    Scene s;
    s.prm = p;
    s.hk.build(p);
    if (s.hk.tables.size() != (size_t)kSceneTableFloats) throw Error(LSP_ERR_INVALID, "unexpected kernel table size");
    if (lo) {
        for (int a = 0; a < 3; a++)
            if (!(hi[a] >= lo[a]) || !std::isfinite(lo[a]) || !std::isfinite(hi[a]))
                throw Error(LSP_ERR_INVALID, "domain: need finite lo <= hi");
        std::memcpy(s.lo, lo, sizeof(s.lo));
        std::memcpy(s.hi, hi, sizeof(s.hi));
        s.user_domain = true;
    }
    s.n = n;
    s.base = n_;
    for (int64_t i = 0; i < n; i++) {
        const int32_t id = (int32_t)(n_ + i);   // caller id across the batch: base + index in the scene
        float w;
        std::memcpy(&w, &id, 4);
        init_pos_.push_back(make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], w));
        init_vel_.push_back(vel ? make_float4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 1.f)
                                : make_float4(0.f, 0.f, 0.f, 1.f));
    }
    pcisph_ = pci;
    n_ += n;
    sc_.push_back(std::move(s));
    return (int)sc_.size() - 1;
}

int BatchEngine::add_collider(int scene, const Collider& c)
{
    if (built_) throw Error(LSP_ERR_STATE, "colliders are added before the batch's first step");
    Scene& s = at(scene);
    if ((int)s.cols.size() >= kMaxColliders) throw Error(LSP_ERR_CAPACITY, "more than 64 colliders in a scene");
    s.cols.push_back(c);
    return (int)s.cols.size() - 1;
}

void BatchEngine::update_collider(int scene, int index, const Collider& c)
{
    Scene& s = at(scene);
    if (index < 0 || index >= (int)s.cols.size()) throw Error(LSP_ERR_INVALID, "collider index out of range");
    if (s.cols[index].sphere != c.sphere) throw Error(LSP_ERR_INVALID, "collider kind mismatch");
    Collider u = c;
    u.boundary = s.cols[index].boundary;
    s.cols[index] = u;
    cols_dirty_ = true;
}

void BatchEngine::grid_info(int scene, int32_t dims[3], int32_t origin[3], int64_t* cells) const
{
    const Scene& s = at(scene);
    if (!built_) throw Error(LSP_ERR_STATE, "the grid is laid out at the batch's first step");
    for (int a = 0; a < 3; a++) {
        if (dims) dims[a] = s.dim[a];
        if (origin) origin[a] = s.org[a];
    }
    if (cells) *cells = s.cells;
}

// Grid boxes, cell and collider ranges, device arrays. The grid box of each scene follows
// the single-scene rule (Engine::ensure_grid): the user domain, else the union of the
// boundary colliders, else the particle bounds plus max(25 %, 4 h) on each side.
void BatchEngine::build()
{
    if (sc_.empty()) throw Error(LSP_ERR_STATE, "the batch has no scenes");
    activate();
    int64_t cell_base = 0;
    int coll_off = 0, max_it = 1;
    for (Scene& s : sc_) {
        float lo[3], hi[3];
        bool have = false;
        if (s.user_domain) {
            std::memcpy(lo, s.lo, sizeof(lo));
            std::memcpy(hi, s.hi, sizeof(hi));
            have = true;
        } else {
            have = boundary_box(s.cols, lo, hi);
        }
        if (!have) {
            for (int a = 0; a < 3; a++) {
                lo[a] = std::numeric_limits<float>::infinity();
                hi[a] = -std::numeric_limits<float>::infinity();
            }
            for (int64_t i = 0; i < s.n; i++) {
                const float4 p = init_pos_[s.base + i];
                const float c[3] = {p.x, p.y, p.z};
                for (int a = 0; a < 3; a++) {
                    lo[a] = std::min(lo[a], c[a]);
                    hi[a] = std::max(hi[a], c[a]);
                }
            }
            for (int a = 0; a < 3; a++) {
                if (!(lo[a] <= hi[a])) { lo[a] = 0.f; hi[a] = 0.f; }
                float margin = std::max(0.25f * (hi[a] - lo[a]), 4.f * s.hk.h);
                lo[a] -= margin;
                hi[a] += margin;
            }
        }
        s.cells = grid_from_box(lo, hi, s.hk.h, s.org, s.dim);
        s.cell_base = cell_base;
        cell_base += s.cells;
        s.coll_off = coll_off;
        coll_off += (int)s.cols.size();
        max_it = std::max(max_it, s.prm.pci_max_iterations);
    }
    if (cell_base + 1 > ((int64_t)1 << 31)) throw Error(LSP_ERR_CAPACITY, "batch grid boxes hold more than 2^31 cells");
    cells_ = cell_base;
    mstride_ = max_it + 4;
    const int S = (int)sc_.size();
    const int64_t cap = round_up(n_, 256);

    for (int k = 0; k < 2; k++) {
        pos_[k].alloc(cap); vel_[k].alloc(cap); half_[k].alloc(cap); old_[k].alloc(cap);
    }
    force_.alloc(cap); ppos_.alloc(cap); ppos_alt_.alloc(cap); phalf_.alloc(cap); pforce_.alloc(cap);
    rho_.alloc(cap); pres_.alloc(cap); prho_.alloc(cap); err_.alloc(cap); vrho_.alloc(cap);
    key_.alloc(cap); slot_.alloc(cap); sorted_key_.alloc(cap); tmp_.alloc(cap);
    slot_of_id_.alloc(cap); nbr_count_.alloc(cap);
    // The scan reads and writes the histogram and cell table 8 entries at a time: both are
    // padded to a multiple of 8 with zeros (scan_entries).
    hist_.alloc(scan_entries(cells_ + 1));
    cell_start_.alloc(scan_entries(cells_ + 1));
    tile_sums_.alloc(scan_tiles(cells_ + 1) + 1);
    loop_sync_.alloc(4);
    maxerr_.alloc((size_t)S * mstride_);
    status_.alloc(S + 1);
    dparams_.alloc(S);
    tables_.alloc((size_t)S * kSceneTableStride);
    dcols_.alloc(std::max(coll_off, 1));
    CK(cudaMallocHost((void**)&hparams_, S * sizeof(DevParams)));
    CK(cudaMallocHost((void**)&hstatus_, (S + 1) * sizeof(DevStatus)));
    std::memset(hstatus_, 0, (S + 1) * sizeof(DevStatus));

    CK(cudaMemsetAsync(hist_.p, 0, scan_entries(cells_ + 1) * sizeof(uint32_t), stream_));
    CK(cudaMemsetAsync(cell_start_.p, 0, scan_entries(cells_ + 1) * sizeof(uint32_t), stream_));
    for (DevArray<float4>* a : {&force_, &ppos_, &ppos_alt_, &phalf_, &pforce_})
        CK(cudaMemsetAsync(a->p, 0, cap * sizeof(float4), stream_));
    for (DevArray<float>* a : {&rho_, &pres_, &prho_, &err_}) CK(cudaMemsetAsync(a->p, 0, cap * sizeof(float), stream_));
    CK(cudaMemsetAsync(nbr_count_.p, 0, cap * sizeof(int32_t), stream_));

    std::vector<float4> zero(n_, make_float4(0.f, 0.f, 0.f, 0.f));
    std::vector<int32_t> soi(n_);
    for (int64_t i = 0; i < n_; i++) soi[i] = (int32_t)i;
    CK(cudaMemcpyAsync(pos_[0].p, init_pos_.data(), n_ * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(vel_[0].p, init_vel_.data(), n_ * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(half_[0].p, zero.data(), n_ * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(old_[0].p, zero.data(), n_ * sizeof(float4), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(slot_of_id_.p, soi.data(), n_ * sizeof(int32_t), cudaMemcpyHostToDevice, stream_));

    std::vector<float> tab((size_t)S * kSceneTableStride, 0.f);
    for (int s = 0; s < S; s++)
        std::copy(sc_[s].hk.tables.begin(), sc_[s].hk.tables.end(), tab.begin() + (size_t)s * kSceneTableStride);
    CK(cudaMemcpyAsync(tables_.p, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    cur_ = 0;
    init_pos_.clear();
    init_pos_.shrink_to_fit();
    init_vel_.clear();
    init_vel_.shrink_to_fit();

    nbr_stride_ = std::max<int64_t>(cap, 256);
    int cap0 = 16;
    for (const Scene& s : sc_) cap0 = std::max(cap0, initial_neighbor_capacity(s.prm));
    built_ = true;
    auto_on_.assign(sc_.size(), 0);
    auto_any_ = false;
    warm_scene_.alloc(sc_.size());
    upload_auto();
    if (history_on()) ensure_warm_buffers();
    ensure_neighbors(cap0);
    upload_colliders();
    build_items();
}

void BatchEngine::ensure_neighbors(int cap)
{
    cap = (int)round_up(std::max(cap, 16), 8);
    if (cap > 4096) throw Error(LSP_ERR_CAPACITY, "neighbour count above 4096 per particle");
    activate();
    nbr_.alloc((size_t)cap * (size_t)nbr_stride_);
    nbr_src_.alloc((size_t)cap * (size_t)nbr_stride_);
    nbr_cap_ = cap;
    params_dirty_ = true;
    drop_graphs();
}

void BatchEngine::upload_params(float dt)
{
    const int S = (int)sc_.size();
    for (int i = 0; i < S; i++) {
        const Scene& s = sc_[i];
        DevParams P = physics_params(s.prm, s.hk, dt);
        P.n = (int)s.n;
        P.ncoll = (int)s.cols.size();
        P.ox = s.org[0]; P.oy = s.org[1]; P.oz = s.org[2];
        P.nx = s.dim[0]; P.ny = s.dim[1]; P.nz = s.dim[2];
        P.cells = (uint32_t)s.cells;
        P.nbr_cap = nbr_cap_;
        P.nbr_stride = nbr_stride_;
        P.base = (int)s.base;
        P.cell_base = (uint32_t)s.cell_base;
        P.coll_off = s.coll_off;
        P.scene = i;
        hparams_[i] = P;
    }
    CK(cudaMemcpyAsync(dparams_.p, hparams_, S * sizeof(DevParams), cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    dt_ = dt;
    params_dirty_ = false;
}

void BatchEngine::upload_colliders()
{
    std::vector<Collider> all;
    for (const Scene& s : sc_) all.insert(all.end(), s.cols.begin(), s.cols.end());
    if (!all.empty()) {
        CK(cudaMemcpyAsync(dcols_.p, all.data(), all.size() * sizeof(Collider), cudaMemcpyHostToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
    }
    cols_dirty_ = false;
}

void BatchEngine::build_items()
{
    std::vector<BatchItem> items;
    const int T = threads_;
    for (int i = 0; i < (int)sc_.size(); i++) {
        const Scene& s = sc_[i];
        for (int64_t b = 0; b < s.n; b += T) {
            BatchItem it;
            it.scene = i;
            it.begin = (int)(s.base + b);
            it.end = (int)(s.base + std::min<int64_t>(s.n, b + T));
            it.pad = 0;
            items.push_back(it);
        }
    }
    items_.alloc(items.size());
    CK(cudaMemcpyAsync(items_.p, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, stream_));
    CK(cudaStreamSynchronize(stream_));
    items_count_ = (int)items.size();
    drop_graphs();
}

void BatchEngine::drop_graphs()
{
    for (int c = 0; c < 2; c++) {
        if (graph_[c]) cudaGraphExecDestroy(graph_[c]);
        graph_[c] = nullptr;
        graph_launches_[c] = 0;
    }
}

int BatchEngine::loop_grid() const
{
    const int most = batch_loop_max_blocks(threads_, (int)sc_.size());
    if (most <= 0) throw Error(LSP_ERR_CUDA, "the device cannot run the batch's cooperative PCISPH kernel");
    int g = loop_blocks_ > 0 ? std::min(loop_blocks_, most) : most;
    return std::max(1, std::min(g, items_count_));
}

BatchArgs BatchEngine::args()
{
    BatchArgs a{};
    a.sp = dparams_.p;
    a.tables = tables_.p;
    a.items = items_.p;
    a.items_count = items_count_;
    a.scenes = (int)sc_.size();
    a.threads = threads_;
    a.st = status_.p;
    return a;
}

StepBuffers BatchEngine::buffers(int c)
{
    StepBuffers b{};
    b.pos = pos_[c].p; b.vel = vel_[c].p; b.half = half_[c].p; b.old = old_[c].p;
    b.force = force_.p; b.rho = rho_.p; b.pres = pres_.p;
    b.ppos = ppos_.p; b.phalf = phalf_.p; b.pforce = pforce_.p; b.prho = prho_.p; b.err = err_.p;
    b.nbr = nbr_.p; b.nbr_count = nbr_count_.p; b.nbr_src = nbr_src_.p; b.nbr_out = nbr_.p; b.vrho = vrho_.p;
    b.tables = tables_.p; b.colliders = dcols_.p; b.status = status_.p + sc_.size();
    b.hist = history_on() ? phist_[c].p : nullptr;
    b.gradrho = features_on() ? gradrho_.p : nullptr;
    return b;
}

// The step of every scene from buffer parity c into 1 - c (the grid build gathers the
// persistent state into the other buffer; every later pass works there), ending with the
// status copy to pinned host memory. Only asynchronous calls: it is also what the graph
// capture records.
int BatchEngine::enqueue_step(int c, int grid)
{
    const int S = (int)sc_.size();
    int launches = 0;
    CK(cudaMemsetAsync(status_.p, 0, (S + 1) * sizeof(DevStatus), stream_));
    BatchArgs a = args();
    launches += launch_batch_keys(a, pos_[c].p, key_.p, slot_.p, hist_.p, stream_);
    GridBuildArgs g{};
    g.P.n = (int)n_;
    g.P.cells = (uint32_t)cells_;
    g.pos_in = pos_[c].p; g.vel_in = vel_[c].p; g.half_in = half_[c].p; g.old_in = old_[c].p;
    g.pos_out = pos_[1 - c].p; g.vel_out = vel_[1 - c].p; g.half_out = half_[1 - c].p; g.old_out = old_[1 - c].p;
    g.key = key_.p; g.slot = slot_.p; g.hist = hist_.p; g.tile_sums = tile_sums_.p; g.cell_start = cell_start_.p;
    g.tmp = tmp_.p; g.slot_of_id = slot_of_id_.p; g.sorted_key = sorted_key_.p;
    const bool feats = features_on();
    g.hist_in = history_on() ? phist_[c].p : nullptr;
    g.hist_out = history_on() ? phist_[1 - c].p : nullptr;
    g.status = status_.p + S;
    launches += launch_grid_order(g, stream_);
    StepBuffers b = buffers(1 - c);
    launches += launch_batch_neighbors_density(a, pos_[1 - c].p, cell_start_.p, nbr_src_.p, nbr_count_.p, rho_.p,
                                               pres_.p, vel_[1 - c].p, vrho_.p, stream_);
    launches += launch_batch_nonpressure(a, b, stream_);
    if (pcisph_) {
        CK(cudaMemsetAsync(loop_sync_.p, 0, 4 * sizeof(uint32_t), stream_));
        CK(cudaMemsetAsync(maxerr_.p, 0, (size_t)S * mstride_ * sizeof(uint32_t), stream_));
        if (feats) {
            // Iteration 0 outside the persistent kernel: predict, then density with the
            // features and (warm start) the network's guess.
            BatchWarmArgs w{};
            w.feat = feat_.p;
            w.maxerr = maxerr_.p;
            w.mstride = mstride_;
            launches += launch_batch_pci_predict0(a, b, stream_);
            launches += launch_batch_density_first(a, b, w, stream_);
            if (guess_on()) {
                // The network's guess on the tensor cores, one block per item (in
                // LSP_WARM_AUTO only for the scenes switched on).
                launch_batch_warm_guess_tc(mlp_.umma(), dparams_.p, items_.p, items_count_, b, feat_.p,
                                           warm_ == LSP_WARM_AUTO ? warm_scene_.p : nullptr, status_.p + S,
                                           stream_);
                launches++;
            }
        }
        BatchLoopArgs l{};
        l.ppos_alt = ppos_alt_.p;
        l.sync = loop_sync_.p;
        l.maxerr = maxerr_.p;
        l.mstride = mstride_;
        l.first_done = feats ? 1 : 0;
        l.warm = guess_on() ? 1 : 0;
        l.warm_scene = warm_ == LSP_WARM_AUTO ? warm_scene_.p : nullptr;
        if (!launch_batch_pci_loop(a, b, l, grid, stream_))
            throw Error(LSP_ERR_CUDA, "the cooperative launch of the batch's PCISPH loop was refused");
        launches++;   // the loop integrates each scene in its last pass
    } else {
        launches += launch_batch_sph_pressure(a, b, stream_);
        launches += launch_batch_integrate(a, b, false, stream_);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hstatus_, status_.p, (S + 1) * sizeof(DevStatus), cudaMemcpyDeviceToHost, stream_));
    return launches;
}

void BatchEngine::run_once(int c)
{
    activate();
    // Occupancy queries stay outside the stream capture.
    const int grid = pcisph_ ? loop_grid() : 0;
    if (use_graph_ && graph_ok_ && !graph_[c]) {
        cudaGraph_t g = nullptr;
        int l = 0;
        bool ok = true;
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            l = enqueue_step(c, grid);
        } catch (const Error&) {
            ok = false;
        }
        cudaError_t e = cudaStreamEndCapture(stream_, &g);
        cudaGraphExec_t ex = nullptr;
        if (ok && e == cudaSuccess && g) e = cudaGraphInstantiate(&ex, g, 0);
        if (g) cudaGraphDestroy(g);
        if (!ok || e != cudaSuccess || !ex) {
            cudaGetLastError();   // capture refused: the step runs as direct launches
            graph_ok_ = false;
        } else {
            graph_[c] = ex;
            graph_launches_[c] = l;
        }
    }
    if (use_graph_ && graph_ok_ && graph_[c]) {
        CK(cudaGraphLaunch(graph_[c], stream_));
        launches_ += graph_launches_[c];
    } else {
        launches_ += enqueue_step(c, grid);
    }
    CK(cudaStreamSynchronize(stream_));
}

bool BatchEngine::run_checked()
{
    const int S = (int)sc_.size();
    for (int attempt = 0;; attempt++) {
        run_once(cur_);
        uint32_t need = 0;
        bool overflow = false;
        for (int s = 0; s < S; s++) {
            if (hstatus_[s].error_flags & kErrNeighborOverflow) {
                overflow = true;
                need = std::max(need, hstatus_[s].max_neighbors);
            }
        }
        if (!overflow) return true;
        if (attempt >= 3) return false;
        // The grid build left the pre-step buffers untouched: grow the lists and redo.
        ensure_neighbors(grown_neighbor_capacity((int)need, nbr_cap_));
        upload_params(dt_);
    }
}

void BatchEngine::finish_step(lsp_step_stats* stats)
{
    const int S = (int)sc_.size();
    cur_ = 1 - cur_;
    features_valid_ = features_on();
    uint32_t errors = hstatus_[S].error_flags;
    bool not_converged = false;
    for (int s = 0; s < S; s++) {
        const DevStatus& st = hstatus_[s];
        lsp_step_stats local{};
        if (pcisph_) {
            float me;
            std::memcpy(&me, &st.max_err_bits, 4);
            local.iterations = st.iterations;
            local.converged = st.converged;
            local.max_density_error_ratio = (double)me / (double)sc_[s].prm.rest_density;
            local.warm_start_used = st.warm_used;
            local.warm_start_tried = (warm_ == LSP_WARM_MLP || (warm_ == LSP_WARM_AUTO && auto_on_[s])) ? 1 : 0;
            sc_[s].last_k = st.last_k;
            if (sc_[s].prm.strict_convergence && !st.converged) not_converged = true;
        } else {
            local.converged = 1;
        }
        local.max_neighbors = (int32_t)st.max_neighbors;
        local.escaped = (int32_t)st.escaped;
        if (stats) stats[s] = local;
        errors |= st.error_flags;
    }
    if (warm_ == LSP_WARM_AUTO && pcisph_) {
        // A zero-start scene that needed more iterations than its switch point, or missed
        // eta, uses the guess from the next step on (the single-scene rule, per scene). The
        // first switch adds the feature pass to the step, so its graph is captured again.
        bool changed = false;
        for (int s = 0; s < S; s++) {
            const int thr = warm_auto_switch(sc_[s].prm);
            if (!auto_on_[s] && ((int)hstatus_[s].iterations > thr || !hstatus_[s].converged)) {
                auto_on_[s] = 1;
                changed = true;
            }
        }
        if (changed) {
            if (!auto_any_) drop_graphs();
            auto_any_ = true;
            upload_auto();
        }
    }
    if (errors & kErrTimeout) throw Error(LSP_ERR_TIMEOUT, "a grid barrier of the batch's PCISPH loop gave up");
    if (errors & kErrNeighborOverflow) throw Error(LSP_ERR_CAPACITY, "neighbour list overflow persisted after resizing");
    if (errors & kErrScan) throw Error(LSP_ERR_CAPACITY, "a grid cell holds more than 4096 particles");
    if (errors & kErrNaN) throw Error(LSP_ERR_DEVICE_STATUS, "non-finite particle position at the start of the step");
    if (not_converged) throw Error(LSP_ERR_NOT_CONVERGED, "PCISPH reached max iterations above eta");
}

void BatchEngine::step(float dt, lsp_step_stats* stats)
{
    if (!(dt > 0.f) || !std::isfinite(dt)) throw Error(LSP_ERR_INVALID, "dt must be finite and > 0");
    if (!built_) build();
    activate();
    if (params_dirty_ || dt != dt_) upload_params(dt);
    if (cols_dirty_) upload_colliders();
    run_checked();
    finish_step(stats);
}

void BatchEngine::set_launch(int use_graph, int threads, int loop_blocks)
{
    if (!batch_threads_supported(threads)) throw Error(LSP_ERR_INVALID, "threads must be 128, 256, 512 or 1024");
    if (loop_blocks < 0) throw Error(LSP_ERR_INVALID, "loop_blocks must be >= 0");
    use_graph_ = use_graph != 0;
    loop_blocks_ = loop_blocks;
    if (threads != threads_) {
        threads_ = threads;
        if (built_) build_items();
    }
    drop_graphs();
}

void BatchEngine::get_launch(int* use_graph, int* threads, int* loop_blocks, int* graph_active) const
{
    if (use_graph) *use_graph = use_graph_ ? 1 : 0;
    if (threads) *threads = threads_;
    if (loop_blocks) *loop_blocks = loop_blocks_;
    if (graph_active) *graph_active = (use_graph_ && graph_ok_ && (graph_[0] || graph_[1])) ? 1 : 0;
}

// Candidates: every supported block size, with the persistent kernel at full residency and
// at half of it. Each candidate runs the same step (from the same pre-step buffers) once to
// capture its graph, then `repeats` timed times; the state only advances at the end.
void BatchEngine::autotune(float dt, int repeats, lsp_batch_tuning* out, lsp_step_stats* stats)
{
    if (!(dt > 0.f) || !std::isfinite(dt)) throw Error(LSP_ERR_INVALID, "dt must be finite and > 0");
    if (repeats < 1 || repeats > 100) throw Error(LSP_ERR_INVALID, "repeats must be in [1, 100]");
    if (!built_) build();
    activate();
    if (params_dirty_ || dt != dt_) upload_params(dt);
    if (cols_dirty_) upload_colliders();
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_));
    struct Cand {
        int threads, blocks;
        float ms;
    };
    std::vector<Cand> cands;
    for (int T : {128, 256, 512, 1024}) {
        if (!pcisph_) {
            cands.push_back({T, 0, 0.f});
            continue;
        }
        const int most = batch_loop_max_blocks(T, (int)sc_.size());
        if (most <= 0) continue;
        cands.push_back({T, most, 0.f});
        const int per_sm = most / std::max(sms, 1);
        if (per_sm >= 2) cands.push_back({T, (per_sm / 2) * sms, 0.f});
    }
    if (cands.empty()) throw Error(LSP_ERR_CUDA, "no launch shape can run the batch's persistent kernel");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const bool graph = use_graph_;
    size_t best = 0;
    try {
        for (size_t k = 0; k < cands.size(); k++) {
            set_launch(graph ? 1 : 0, cands[k].threads, cands[k].blocks);
            run_checked();   // capture (and list growth, if the step needs it)
            float bestms = std::numeric_limits<float>::infinity();
            for (int r = 0; r < repeats; r++) {
                CK(cudaEventRecord(e0, stream_));
                run_once(cur_);
                CK(cudaEventRecord(e1, stream_));
                CK(cudaEventSynchronize(e1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                bestms = std::min(bestms, ms);
            }
            cands[k].ms = bestms;
            if (bestms < cands[best].ms) best = k;
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    set_launch(graph ? 1 : 0, cands[best].threads, cands[best].blocks);
    // The chosen shape runs the step once more; that run's results become the step.
    if (!run_checked()) {
        finish_step(stats);   // reports the persisting overflow
        return;
    }
    finish_step(stats);
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->threads = cands[best].threads;
        out->loop_blocks = cands[best].blocks;
        out->candidates = (int32_t)std::min<size_t>(cands.size(), 16);
        for (int k = 0; k < out->candidates; k++) {
            out->cand_threads[k] = cands[k].threads;
            out->cand_loop_blocks[k] = cands[k].blocks;
            out->cand_ms[k] = cands[k].ms;
        }
    }
}

// ------------------------------------------------------------------ read-back

void BatchEngine::stage(size_t floats)
{
    if (stage_.n < floats) stage_.alloc(floats);
}

void BatchEngine::check_scene(int scene) const
{
    at(scene);
    if (!built_) throw Error(LSP_ERR_STATE, "no step has run");
}

void BatchEngine::read_particles(int scene, float* x, float* v, int64_t n)
{
    check_scene(scene);
    const Scene& s = sc_[scene];
    if (n != s.n || !x) throw Error(LSP_ERR_INVALID, "read_particles: n must equal the scene's particle count");
    read_field(scene, LSP_FIELD_POSITION, x, n);
    if (v) read_field(scene, LSP_FIELD_VELOCITY, v, n);
}

void BatchEngine::read_field(int scene, int field, float* out, int64_t n)
{
    check_scene(scene);
    const Scene& s = sc_[scene];
    if (!out || n != s.n) throw Error(LSP_ERR_INVALID, "read_field: n must equal the scene's particle count");
    activate();
    const void* src = nullptr;
    int comps = 1, mode = 0;
    switch (field) {
    case LSP_FIELD_POSITION: src = pos_[cur_].p; comps = 3; break;
    case LSP_FIELD_VELOCITY: src = vel_[cur_].p; comps = 3; break;
    case LSP_FIELD_HALF_VELOCITY: src = half_[cur_].p; comps = 3; break;
    case LSP_FIELD_OLD_HALF_VELOCITY: src = old_[cur_].p; comps = 3; break;
    case LSP_FIELD_PRED_POSITION: src = (pcisph_ && (s.last_k & 1)) ? ppos_alt_.p : ppos_.p; comps = 3; break;
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
    const int32_t* soi = slot_of_id_.p + s.base;
    if (field == LSP_FIELD_NEIGHBOR_COUNT)
        launch_gather_count(nbr_count_.p, soi, stage_.p, n, stream_);
    else
        launch_gather_field(src, comps, mode, soi, stage_.p, n, stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, stage_.p, (size_t)n * comps * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void BatchEngine::read_neighbors(int scene, int64_t* offsets, int32_t* index, int64_t n, int64_t capacity)
{
    check_scene(scene);
    const Scene& s = sc_[scene];
    if (n != s.n || !offsets) throw Error(LSP_ERR_INVALID, "read_neighbors: bad arguments");
    std::vector<float> counts(n);
    read_field(scene, LSP_FIELD_NEIGHBOR_COUNT, counts.data(), n);
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
    launch_neighbor_export(nbr_.p, nbr_count_.p, nbr_stride_, pos_[cur_].p, slot_of_id_.p + s.base, doff.p, dout.p,
                           n, stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(index, dout.p, offsets[n] * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    for (int64_t e = 0; e < offsets[n]; e++) index[e] -= (int32_t)s.base;   // batch ids -> scene caller ids
}

void BatchEngine::read_grid(int scene, uint32_t* keys, int32_t* ids, int64_t n, uint32_t* cell_start,
                            int64_t cells_plus_one)
{
    check_scene(scene);
    const Scene& s = sc_[scene];
    if (n != s.n) throw Error(LSP_ERR_INVALID, "read_grid: n must equal the scene's particle count");
    activate();
    if (keys) {
        CK(cudaMemcpyAsync(keys, sorted_key_.p + s.base, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        for (int64_t i = 0; i < n; i++) keys[i] -= (uint32_t)s.cell_base;
    }
    if (ids) {
        std::vector<float4> p(n);
        CK(cudaMemcpyAsync(p.data(), pos_[cur_].p + s.base, n * sizeof(float4), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        for (int64_t i = 0; i < n; i++) {
            std::memcpy(&ids[i], &p[i].w, 4);
            ids[i] -= (int32_t)s.base;
        }
    }
    if (cell_start) {
        if (cells_plus_one != s.cells + 1) throw Error(LSP_ERR_INVALID, "read_grid: cell table size mismatch");
        CK(cudaMemcpyAsync(cell_start, cell_start_.p + s.cell_base, cells_plus_one * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        for (int64_t i = 0; i < cells_plus_one; i++) cell_start[i] -= (uint32_t)s.base;
    }
}

void BatchEngine::read_state(float* x, float* v, float* half, float* old, int32_t* first, int64_t n)
{
    if (n != n_ || !x || !v || !half || !old || !first) throw Error(LSP_ERR_INVALID, "read_state: bad arguments");
    if (!built_) throw Error(LSP_ERR_STATE, "no step has run");
    activate();
    stage((size_t)n * 13);
    float* s = stage_.p;
    launch_gather_state(pos_[cur_].p, vel_[cur_].p, half_[cur_].p, old_[cur_].p, slot_of_id_.p, s, s + 3 * n,
                        s + 6 * n, s + 9 * n, (int32_t*)(s + 12 * n), n, stream_);
    CK(cudaGetLastError());
    size_t b3 = (size_t)n * 3 * sizeof(float);
    CK(cudaMemcpyAsync(x, s, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(v, s + 3 * n, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(half, s + 6 * n, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(old, s + 9 * n, b3, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(first, s + 12 * n, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void BatchEngine::write_state(const float* x, const float* v, const float* half, const float* old,
                              const int32_t* first, int64_t n)
{
    if (n != n_ || !x || !v || !half || !old || !first) throw Error(LSP_ERR_INVALID, "write_state: bad arguments");
    if (!built_) throw Error(LSP_ERR_STATE, "no step has run");
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
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream_));
}

// ------------------------------------------------------------------ learned warm start

void BatchEngine::ensure_warm_buffers()
{
    if (!built_ || phist_[0].p) return;
    activate();
    const int64_t cap = (int64_t)pos_[0].n;
    for (int k = 0; k < 2; k++) {
        phist_[k].alloc(cap);
        CK(cudaMemsetAsync(phist_[k].p, 0, cap * sizeof(float4), stream_));
    }
    feat_.alloc(cap * kMlpIn);
    gradrho_.alloc(cap);
    tgt_.alloc(cap);
    CK(cudaMemsetAsync(feat_.p, 0, cap * kMlpIn * sizeof(float), stream_));
    CK(cudaMemsetAsync(gradrho_.p, 0, cap * sizeof(float), stream_));
    CK(cudaStreamSynchronize(stream_));
}

void BatchEngine::set_warm_start(int mode)
{
    if (mode != LSP_WARM_ZERO && mode != LSP_WARM_MLP && mode != LSP_WARM_AUTO) throw Error(LSP_ERR_INVALID, "unknown warm_start");
    if (mode != LSP_WARM_ZERO && !sc_.empty() && !pcisph_)
        throw Error(LSP_ERR_INVALID, "the learned warm start needs PCISPH scenes");
    warm_ = mode;
    std::fill(auto_on_.begin(), auto_on_.end(), 0);
    auto_any_ = false;
    if (built_) upload_auto();
    drop_graphs();
    if (history_on()) ensure_warm_buffers();
}

void BatchEngine::upload_auto()
{
    if (auto_on_.empty()) return;
    activate();
    CK(cudaMemcpyAsync(warm_scene_.p, auto_on_.data(), auto_on_.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                       stream_));
    CK(cudaStreamSynchronize(stream_));
}

void BatchEngine::mlp_record(bool on)
{
    record_ = on;
    drop_graphs();
    if (history_on()) ensure_warm_buffers();
}

void BatchEngine::mlp_reset(uint64_t seed)
{
    activate();
    mlp_.reset(seed);
}

void BatchEngine::mlp_set(const float* w, int n)
{
    activate();
    mlp_.set(w, n);
}

void BatchEngine::mlp_get(float* w, int n)
{
    activate();
    mlp_.get(w, n);
}

void BatchEngine::mlp_set_loss_asymmetry(float w) { mlp_.set_over_weight(w); }

float BatchEngine::mlp_train(int iterations, int batch, float lr, uint64_t seed)
{
    if (!built_ || !features_valid_)
        throw Error(LSP_ERR_STATE, "mlp_train needs a PCISPH step that recorded features (lsp_batch_mlp_record)");
    if (iterations <= 0 || batch <= 0) throw Error(LSP_ERR_INVALID, "iterations and batch must be > 0");
    activate();
    launch_batch_targets(args(), pres_.p, tgt_.p, stream_);
    CK(cudaGetLastError());
    return mlp_.train(feat_.p, tgt_.p, n_, iterations, batch, lr, seed);
}

void BatchEngine::read_features(int scene, float* out, int64_t n)
{
    check_scene(scene);
    const Scene& s = sc_[scene];
    if (!out || n != s.n) throw Error(LSP_ERR_INVALID, "read_features: n must equal the scene's particle count");
    if (!features_valid_) throw Error(LSP_ERR_STATE, "no step has recorded features");
    activate();
    stage((size_t)n * kMlpIn);
    launch_gather_rows(feat_.p, kMlpIn, slot_of_id_.p + s.base, stage_.p, n, stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, stage_.p, (size_t)n * kMlpIn * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
}

void BatchEngine::timer_mark(int slot)
{
    if (slot < 0 || slot >= 16) throw Error(LSP_ERR_INVALID, "timer slot must be in [0, 16)");
    activate();
    if (!marks_[slot]) CK(cudaEventCreate(&marks_[slot]));
    CK(cudaEventRecord(marks_[slot], stream_));
}

float BatchEngine::timer_elapsed(int a, int b)
{
    if (a < 0 || a >= 16 || b < 0 || b >= 16 || !marks_[a] || !marks_[b])
        throw Error(LSP_ERR_INVALID, "timer slots not marked");
    activate();
    CK(cudaEventSynchronize(marks_[b]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, marks_[a], marks_[b]));
    return ms;
}

}  // namespace lsp
