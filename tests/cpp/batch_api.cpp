// Drives the C++ batch API (lsp::SceneBatch in include/lsp_solver.hpp): several scenes
// with their own parameters, particles and boundary boxes, stepped together; the first
// step goes through the autotuner. Reads the scenes from argv[1], writes each scene's final
// positions and densities (caller order, float32), scene after scene, to argv[2].
//
// file: int32 scenes, int32 steps, float dt, then per scene: lsp_params (raw bytes),
// int32 n, float box[6] (center, half extent), n * 3 float positions.
#include <cstdio>
#include <vector>

#include "lsp_solver.hpp"

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    int scenes = 0, steps = 0;
    float dt = 0.f;
    bool ok = std::fread(&scenes, 4, 1, f) && std::fread(&steps, 4, 1, f) && std::fread(&dt, 4, 1, f);
    try {
        lsp::SceneBatch batch;
        for (int k = 0; ok && k < scenes; k++) {
            lsp_params p;
            int n = 0;
            float box[6];
            ok = std::fread(&p, sizeof(p), 1, f) && std::fread(&n, 4, 1, f) && std::fread(box, 4, 6, f) == 6;
            std::vector<float> pos((size_t)n * 3);
            ok = ok && std::fread(pos.data(), 4, pos.size(), f) == pos.size();
            if (!ok) break;
            int s = batch.addScene(p, pos.data(), nullptr, n);
            batch.addStaticCollisionBox(s, {box[0], box[1], box[2]}, {box[3], box[4], box[5]},
                                        lsp::CollisionType::BOUNDARY);
        }
        std::fclose(f);
        if (!ok) return 4;
        lsp_batch_tuning t = batch.autotune(dt);
        for (int s = 1; s < steps; s++) batch.update(dt);
        FILE* o = std::fopen(argv[2], "wb");
        if (!o) return 5;
        for (int k = 0; k < batch.sceneCount(); k++) {
            std::vector<float> x = batch.positions(k), rho = batch.densities(k);
            std::fwrite(x.data(), 4, x.size(), o);
            std::fwrite(rho.data(), 4, rho.size(), o);
        }
        std::fclose(o);
        std::printf("%d scenes, %d steps, tuned %d threads x %d blocks\n", batch.sceneCount(), steps, t.threads,
                    t.loop_blocks);
    } catch (const lsp::SolverError& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
