// Drives the C++ solver API (include/lsp_solver.hpp) the way an application of the
// reference drives LiPhEn::PCISPHSolver: set parameters, add particles and colliders,
// call update(dt), read positions back. Reads a scene from argv[1], writes the final
// positions and densities (caller order, float32) to argv[2].
//
// scene file: int32 n, int32 steps, float dt, float radius, float factor, float rho0,
// float viscosity, float eta, int32 max_iterations, float box[6] (center, half),
// then n * 3 float positions.
#include <cstdio>
#include <vector>

#include "lsp_solver.hpp"

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    int n = 0, steps = 0, maxIt = 0;
    float dt, radius, factor, rho0, visc, eta, box[6];
    bool ok = std::fread(&n, 4, 1, f) && std::fread(&steps, 4, 1, f) && std::fread(&dt, 4, 1, f) &&
              std::fread(&radius, 4, 1, f) && std::fread(&factor, 4, 1, f) && std::fread(&rho0, 4, 1, f) &&
              std::fread(&visc, 4, 1, f) && std::fread(&eta, 4, 1, f) && std::fread(&maxIt, 4, 1, f) &&
              std::fread(box, 4, 6, f) == 6;
    std::vector<float> pos((size_t)n * 3);
    ok = ok && std::fread(pos.data(), 4, pos.size(), f) == pos.size();
    std::fclose(f);
    if (!ok) return 4;
    try {
        lsp::PCISPHSolver solver;
        solver.setParticleRadius(radius);
        solver.setKernelRadiusFactor(factor);
        solver.setRestDensity(rho0);
        solver.setViscosityCoefficient(visc);
        solver.setMaxDensityErrorRatio(eta);
        solver.setMinIterations(maxIt);
        for (int i = 0; i < n; i++) solver.addParticle({pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]});
        solver.addStaticCollisionBox({box[0], box[1], box[2]}, {box[3], box[4], box[5]}, lsp::CollisionType::BOUNDARY);
        for (int s = 0; s < steps; s++) solver.update(dt);
        std::vector<float> x = solver.positions(), rho = solver.densities();
        FILE* o = std::fopen(argv[2], "wb");
        if (!o) return 5;
        std::fwrite(x.data(), 4, x.size(), o);
        std::fwrite(rho.data(), 4, rho.size(), o);
        std::fclose(o);
        std::printf("%d particles, %d steps, mass %.9g\n", solver.getParticleCount(), steps, solver.getParticleMass());
    } catch (const lsp::SolverError& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
