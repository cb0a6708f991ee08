// lsp_solver.hpp -- header-only C++ mirror of LiquidPhysics' solver classes over the
// C ABI in lsp.h. A C++ application that used LiPhEn::SPHSolver / LiPhEn::PCISPHSolver
// (LiquidPhysics/include/SPHSolver.h:25-168, PCISPHSolver.h:7-44) keeps the same calls:
// addParticle, addStaticCollisionObject (box / sphere), the parameter setters and
// getters, update(dt) (PhysicSolver.h:10), plus bulk read-back in place of reading the
// particle objects. Errors throw lsp::SolverError (the reference has no error channel).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "lsp.h"

namespace lsp {

struct SolverError : std::runtime_error {
    int code;
    SolverError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int code)
{
    if (code != LSP_OK) throw SolverError(code, std::string("liblsp: ") + lsp_last_error());
}

struct Vec3 {
    float x, y, z;
};

enum class CollisionType { OBSTACLE = LSP_OBSTACLE, BOUNDARY = LSP_BOUNDARY };

class SPHSolver {
public:
    explicit SPHSolver(int device = -1) : SPHSolver(LSP_SOLVER_SPH, device) {}
    virtual ~SPHSolver()
    {
        if (h_) lsp_destroy(h_);
    }
    SPHSolver(const SPHSolver&) = delete;
    SPHSolver& operator=(const SPHSolver&) = delete;

    // PhysicSolver::update (PhysicSolver.cpp:12-21).
    lsp_step_stats update(float deltaTime)
    {
        lsp_step_stats st{};
        check(lsp_step(h_, deltaTime, &st));
        return st;
    }

    // SPHSolver::addParticle (SPHSolver.cpp:129-135): a particle at rest or with a velocity.
    void addParticle(Vec3 position, Vec3 velocity = {0.f, 0.f, 0.f})
    {
        float p[3] = {position.x, position.y, position.z};
        float v[3] = {velocity.x, velocity.y, velocity.z};
        check(lsp_add_particles(h_, p, v, 1));
    }
    void addParticles(const float* xyz, const float* vel, int64_t n) { check(lsp_add_particles(h_, xyz, vel, n)); }
    void removeParticles() { check(lsp_remove_particles(h_)); }

    // SPHSolver::addStaticCollisionObject with a StaticCollisionBox / StaticCollisionSphere.
    void addStaticCollisionBox(Vec3 center, Vec3 halfDimensions, CollisionType type = CollisionType::OBSTACLE)
    {
        float c[3] = {center.x, center.y, center.z}, h[3] = {halfDimensions.x, halfDimensions.y, halfDimensions.z};
        check(lsp_add_box(h_, c, h, (int)type));
    }
    void addStaticCollisionSphere(Vec3 center, float radius, CollisionType type = CollisionType::OBSTACLE)
    {
        float c[3] = {center.x, center.y, center.z};
        check(lsp_add_sphere(h_, c, radius, (int)type));
    }
    void removeStaticCollisionObjects() { check(lsp_remove_colliders(h_)); }
    void cleanUp()
    {
        removeParticles();
        removeStaticCollisionObjects();
    }

    // Getters (SPHSolver.h:79-95).
    Vec3 getGravity() const { lsp_params p = params(); return {p.gravity[0], p.gravity[1], p.gravity[2]}; }
    int getParticleCount() const { int64_t n = 0; check(lsp_particle_count(h_, &n)); return (int)n; }
    float getParticleRadius() const { return params().particle_radius; }
    float getParticleMass() const { float m = 0; check(lsp_particle_mass(h_, &m)); return m; }
    float getKernelRadius() const { float k = 0; check(lsp_kernel_radius(h_, &k)); return k; }
    float getKernelRadiusFactor() const { return params().kernel_radius_factor; }
    float getRestDensity() const { return params().rest_density; }
    float getViscosityCoefficient() const { return params().viscosity; }
    float getPressureStiffnessCoefficient() const { return params().stiffness; }
    float getNegativePressureFactor() const { return params().negative_pressure_factor; }
    float getSurfaceTensionCoefficient() const { return params().surface_tension; }
    float getSurfaceTensionThreshold() const { return params().surface_tension_threshold; }
    float getResitutionCoefficient() const { return params().restitution; }
    float getFrictionCoefficient() const { return params().friction; }

    // Setters (SPHSolver.h:97-109).
    void setHasCollisionObjectDataChanged(bool) {}
    void setGravity(Vec3 g) { edit([&](lsp_params& p) { p.gravity[0] = g.x; p.gravity[1] = g.y; p.gravity[2] = g.z; }); }
    void setParticleRadius(float v) { edit([&](lsp_params& p) { p.particle_radius = v; }); }
    void setKernelRadiusFactor(float v) { edit([&](lsp_params& p) { p.kernel_radius_factor = v; }); }
    void setRestDensity(float v) { edit([&](lsp_params& p) { p.rest_density = v; }); }
    void setViscosityCoefficient(float v) { edit([&](lsp_params& p) { p.viscosity = v; }); }
    void setPressureStiffnessCoefficient(float v) { edit([&](lsp_params& p) { p.stiffness = v; }); }
    void setNegativePressureFactor(float v) { edit([&](lsp_params& p) { p.negative_pressure_factor = v; }); }
    void setSurfaceTensionCoefficient(float v) { edit([&](lsp_params& p) { p.surface_tension = v; }); }
    void setSurfaceTensionThreshold(float v) { edit([&](lsp_params& p) { p.surface_tension_threshold = v; }); }
    void setRestitutionCoefficient(float v) { edit([&](lsp_params& p) { p.restitution = v; }); }
    void setFrictionCoefficient(float v) { edit([&](lsp_params& p) { p.friction = v; }); }

    // Read-back in caller order (replaces reading the particle objects after update).
    std::vector<float> positions() { return field(LSP_FIELD_POSITION, 3); }
    std::vector<float> velocities() { return field(LSP_FIELD_VELOCITY, 3); }
    std::vector<float> densities() { return field(LSP_FIELD_DENSITY, 1); }
    std::vector<float> pressures() { return field(LSP_FIELD_PRESSURE, 1); }
    std::vector<float> field(int id, int comps)
    {
        int64_t n = getParticleCount();
        std::vector<float> out((size_t)n * comps);
        check(lsp_read_field(h_, id, out.data(), n));
        return out;
    }

    lsp_solver* handle() { return h_; }

protected:
    SPHSolver(int kind, int device)
    {
        lsp_params p;
        lsp_params_default(&p);
        p.solver = kind;
        check(lsp_create(&p, device, &h_));
    }
    lsp_params params() const
    {
        lsp_params p;
        check(lsp_get_params(h_, &p));
        return p;
    }
    template <typename F>
    void edit(F&& f)
    {
        lsp_params p = params();
        f(p);
        check(lsp_set_params(h_, &p));
    }
    lsp_solver* h_ = nullptr;
};

class PCISPHSolver : public SPHSolver {
public:
    explicit PCISPHSolver(int device = -1) : SPHSolver(LSP_SOLVER_PCISPH, device) {}
    // PCISPHSolver.h:16-20. The reference's loop runs at most getMinIterations() times.
    int getMinIterations() const { return params().pci_max_iterations; }
    float getMaxDensityErrorRatio() const { return params().pci_eta; }
    void setMinIterations(int v) { edit([&](lsp_params& p) { p.pci_max_iterations = v; }); }
    void setMaxDensityErrorRatio(float v) { edit([&](lsp_params& p) { p.pci_eta = v; }); }
    // Extension (no counterpart in the reference): the initial pressure of the loop,
    // LSP_WARM_ZERO (the reference), LSP_WARM_MLP (the learned guess, lsp_mlp_* in lsp.h) or
    // LSP_WARM_AUTO (zero start until a step needs more than `autoIterations` iterations or
    // misses eta, the learned guess after that; 0 = max(12, max iterations / 2)).
    void setWarmStart(int mode, int autoIterations = 0)
    {
        edit([&](lsp_params& p) {
            p.warm_start = mode;
            p.warm_auto_iterations = autoIterations;
        });
    }
    int getWarmStart() const { return params().warm_start; }
};

// Many independent scenes stepped together (lsp_batch_* in lsp.h): what an application
// would otherwise do with one solver object per scene, each updated in turn. Scenes and
// their colliders are added before the first update; each scene's results equal those of
// its own solver object.
class SceneBatch {
public:
    explicit SceneBatch(int device = -1) { check(lsp_batch_create(device, &b_)); }
    ~SceneBatch()
    {
        if (b_) lsp_batch_destroy(b_);
    }
    SceneBatch(const SceneBatch&) = delete;
    SceneBatch& operator=(const SceneBatch&) = delete;

    // A scene from parameters (lsp_params_default + edits) and particles in caller order.
    // domain_lo / domain_hi may both be null (grid box from the boundary colliders).
    int addScene(const lsp_params& params, const float* xyz, const float* vel, int64_t n,
                 const float* domain_lo = nullptr, const float* domain_hi = nullptr)
    {
        int32_t k = -1;
        check(lsp_batch_add_scene(b_, &params, xyz, vel, n, domain_lo, domain_hi, &k));
        counts_.push_back(n);
        return k;
    }
    void addStaticCollisionBox(int scene, Vec3 center, Vec3 halfExtent, CollisionType type)
    {
        float c[3] = {center.x, center.y, center.z}, h[3] = {halfExtent.x, halfExtent.y, halfExtent.z};
        check(lsp_batch_add_box(b_, scene, c, h, (int)type));
    }
    void addStaticCollisionSphere(int scene, Vec3 center, float radius, CollisionType type)
    {
        float c[3] = {center.x, center.y, center.z};
        check(lsp_batch_add_sphere(b_, scene, c, radius, (int)type));
    }
    // One step of every scene; per-scene statistics.
    std::vector<lsp_step_stats> update(float deltaTime)
    {
        std::vector<lsp_step_stats> st(counts_.size());
        check(lsp_batch_step(b_, deltaTime, st.data()));
        return st;
    }
    // Chooses the launch shape on the next step and performs that step.
    lsp_batch_tuning autotune(float deltaTime, int repeats = 3)
    {
        lsp_batch_tuning t{};
        std::vector<lsp_step_stats> st(counts_.size());
        check(lsp_batch_autotune(b_, deltaTime, repeats, &t, st.data()));
        return t;
    }
    int sceneCount() const { return (int)counts_.size(); }
    int64_t particleCount(int scene) const { return counts_.at(scene); }
    std::vector<float> positions(int scene) { return field(scene, LSP_FIELD_POSITION, 3); }
    std::vector<float> velocities(int scene) { return field(scene, LSP_FIELD_VELOCITY, 3); }
    std::vector<float> densities(int scene) { return field(scene, LSP_FIELD_DENSITY, 1); }
    std::vector<float> field(int scene, int id, int comps)
    {
        int64_t n = particleCount(scene);
        std::vector<float> out((size_t)n * comps);
        check(lsp_batch_read_field(b_, scene, id, out.data(), n));
        return out;
    }
    lsp_batch* handle() { return b_; }

private:
    lsp_batch* b_ = nullptr;
    std::vector<int64_t> counts_;
};

}  // namespace lsp
