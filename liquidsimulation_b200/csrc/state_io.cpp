// State files: lsp_save_state / lsp_load_state / lsp_state_file_info (include/lsp.h).
//
// Layout (little-endian, no padding):
//   char     magic[8] = "LSPSTAT1"
//   uint32   version = 1
//   uint32   flags: 1 = warm-start pressure history present, 2 = MLP weights present,
//                   4 = user grid box present
//   uint64   seed (caller's label of the scene, stored as given)
//   int64    n particles
//   int32    colliders
//   uint32   sizeof(lsp_params)
//   lsp_params
//   float    domain_lo[3], domain_hi[3]
//   colliders x { int32 sphere, int32 boundary, float center[3], float half_extent[3], float radius }
//   float    x[3n], v[3n], v_half[3n], v_half_old[3n]; int32 first_step[n]      (caller order)
//   [float   pressure_history[3n]]                                              (flag 1)
//   [float   mlp_weights[1377]]                                                 (flag 2)
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lsp.h"
#include "engine.h"
#include "lsp_handle.h"
#include "mlp.cuh"

namespace {

constexpr char kMagic[8] = {'L', 'S', 'P', 'S', 'T', 'A', 'T', '1'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kHasHistory = 1, kHasMlp = 2, kHasDomain = 4;

struct FileCloser {
    void operator()(FILE* f) const
    {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<FILE, FileCloser>;

struct Header {
    uint32_t flags = 0;
    uint64_t seed = 0;
    int64_t n = 0;
    int32_t colliders = 0;
    lsp_params params{};
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

template <typename T>
void put(FILE* f, const T* p, size_t count)
{
    if (count && std::fwrite(p, sizeof(T), count, f) != count)
        throw lsp::Error(LSP_ERR_INVALID, "state file: write failed");
}
template <typename T>
void get(FILE* f, T* p, size_t count)
{
    if (count && std::fread(p, sizeof(T), count, f) != count)
        throw lsp::Error(LSP_ERR_INVALID, "state file: truncated");
}

File open_file(const char* path, const char* mode)
{
    if (!path) throw lsp::Error(LSP_ERR_INVALID, "null pointer: path");
    File f(std::fopen(path, mode));
    if (!f) throw lsp::Error(LSP_ERR_INVALID, std::string("state file: cannot open ") + path);
    return f;
}

Header read_header(FILE* f)
{
    char magic[8];
    uint32_t version = 0, psize = 0;
    Header h;
    get(f, magic, 8);
    if (std::memcmp(magic, kMagic, 8) != 0) throw lsp::Error(LSP_ERR_INVALID, "state file: bad magic");
    get(f, &version, 1);
    if (version != kVersion) throw lsp::Error(LSP_ERR_INVALID, "state file: unsupported version");
    get(f, &h.flags, 1);
    get(f, &h.seed, 1);
    get(f, &h.n, 1);
    get(f, &h.colliders, 1);
    get(f, &psize, 1);
    if (psize != sizeof(lsp_params)) throw lsp::Error(LSP_ERR_INVALID, "state file: parameter block size mismatch");
    get(f, &h.params, 1);
    get(f, h.lo, 3);
    get(f, h.hi, 3);
    if (h.n < 0 || h.n > (int64_t)1 << 30 || h.colliders < 0 || h.colliders > lsp::kMaxColliders)
        throw lsp::Error(LSP_ERR_INVALID, "state file: counts out of range");
    return h;
}

lsp::Engine& E(lsp_solver* s)
{
    if (!s || !s->e) throw lsp::Error(LSP_ERR_INVALID, "null solver handle");
    return *s->e;
}

}  // namespace

extern "C" {

int lsp_save_state(lsp_solver* s, const char* path, uint64_t seed)
{
    return lsp::guard([&] {
        lsp::Engine& e = E(s);
        const int64_t n = e.count();
        std::vector<float> x(3 * n), v(3 * n), hv(3 * n), ov(3 * n), hist;
        std::vector<int32_t> first(n);
        if (n) e.read_state(x.data(), v.data(), hv.data(), ov.data(), first.data(), n);
        Header h;
        h.seed = seed;
        h.n = n;
        h.params = e.params();
        h.colliders = (int32_t)e.colliders().size();
        if (e.domain(h.lo, h.hi)) h.flags |= kHasDomain;
        if (e.has_history() && n) {
            hist.resize(3 * n);
            e.read_history(hist.data(), n);
            h.flags |= kHasHistory;
        }
        std::vector<float> w(lsp::kMlpParams);
        e.mlp_get(w.data(), lsp::kMlpParams);
        h.flags |= kHasMlp;
        File f = open_file(path, "wb");
        const uint32_t psize = sizeof(lsp_params);
        put(f.get(), kMagic, 8);
        put(f.get(), &kVersion, 1);
        put(f.get(), &h.flags, 1);
        put(f.get(), &h.seed, 1);
        put(f.get(), &h.n, 1);
        put(f.get(), &h.colliders, 1);
        put(f.get(), &psize, 1);
        put(f.get(), &h.params, 1);
        put(f.get(), h.lo, 3);
        put(f.get(), h.hi, 3);
        for (const lsp::Collider& c : e.colliders()) {
            const int32_t kinds[2] = {c.sphere, c.boundary};
            const float g[7] = {c.cx, c.cy, c.cz, c.hx, c.hy, c.hz, c.radius};
            put(f.get(), kinds, 2);
            put(f.get(), g, 7);
        }
        put(f.get(), x.data(), x.size());
        put(f.get(), v.data(), v.size());
        put(f.get(), hv.data(), hv.size());
        put(f.get(), ov.data(), ov.size());
        put(f.get(), first.data(), first.size());
        if (h.flags & kHasHistory) put(f.get(), hist.data(), hist.size());
        put(f.get(), w.data(), w.size());
        if (std::fflush(f.get()) != 0) throw lsp::Error(LSP_ERR_INVALID, "state file: write failed");
    });
}

int lsp_load_state(lsp_solver* s, const char* path)
{
    return lsp::guard([&] {
        lsp::Engine& e = E(s);
        File f = open_file(path, "rb");
        Header h = read_header(f.get());
        std::vector<lsp::Collider> cols(h.colliders);
        for (lsp::Collider& c : cols) {
            int32_t kinds[2];
            float g[7];
            get(f.get(), kinds, 2);
            get(f.get(), g, 7);
            c = lsp::Collider{};
            c.sphere = kinds[0];
            c.boundary = kinds[1];
            c.cx = g[0]; c.cy = g[1]; c.cz = g[2];
            c.hx = g[3]; c.hy = g[4]; c.hz = g[5];
            c.radius = g[6];
        }
        const int64_t n = h.n;
        std::vector<float> x(3 * n), v(3 * n), hv(3 * n), ov(3 * n), hist;
        std::vector<int32_t> first(n);
        get(f.get(), x.data(), x.size());
        get(f.get(), v.data(), v.size());
        get(f.get(), hv.data(), hv.size());
        get(f.get(), ov.data(), ov.size());
        get(f.get(), first.data(), first.size());
        if (h.flags & kHasHistory) {
            hist.resize(3 * n);
            get(f.get(), hist.data(), hist.size());
        }
        std::vector<float> w;
        if (h.flags & kHasMlp) {
            w.resize(lsp::kMlpParams);
            get(f.get(), w.data(), w.size());
        }
        // Everything read and checked: now replace the solver's scene.
        e.set_params(h.params);
        e.remove_particles();
        e.remove_colliders();
        for (const lsp::Collider& c : cols) e.add_collider(c);
        if (h.flags & kHasDomain)
            e.set_domain(h.lo, h.hi);
        else
            e.clear_domain();
        if (n) {
            e.add_particles(x.data(), v.data(), n);
            e.write_state(x.data(), v.data(), hv.data(), ov.data(), first.data(), n);
            if (h.flags & kHasHistory) e.write_history(hist.data(), n);
        }
        if (!w.empty()) e.mlp_set(w.data(), lsp::kMlpParams);
    });
}

int lsp_state_file_info(const char* path, lsp_params* params, int64_t* n, int32_t* colliders, uint64_t* seed)
{
    return lsp::guard([&] {
        File f = open_file(path, "rb");
        Header h = read_header(f.get());
        if (params) *params = h.params;
        if (n) *n = h.n;
        if (colliders) *colliders = h.colliders;
        if (seed) *seed = h.seed;
    });
}

}  // extern "C"
