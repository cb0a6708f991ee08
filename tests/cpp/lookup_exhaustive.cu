// Exhaustive host check of the device lookup's slot computation (table_slot in
// liquidsimulation_b200/csrc/lsp_device.cuh): for every float d in [0, h) it must equal
// (int)(d / step), the index of the reference's SPHKernel::get*Weight (SPHKernel.cpp:19).
// The thresholds are built by the same bisection as HostKernels::build. Host and device
// share IEEE single rounding (-ffp-contract=off here, -fmad=false in the library), so the
// host result is the device result.
//   usage: lookup_exhaustive <particle radius> <kernel radius factor>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <limits>
#include "lsp_device.cuh"

int main(int argc, char** argv)
{
    float radius = argc > 1 ? std::strtof(argv[1], nullptr) : 0.0125f;
    float factor = argc > 2 ? std::strtof(argv[2], nullptr) : 3.2f;
    const float h = factor * radius;                 // SPHSolver::recalcKernelRadius
    const float step = h / 1000;                     // SPHKernel::recalcDivisionStep
    float thr[lsp::kTableSize + 1];
    thr[0] = 0.f;
    const float hi_d = 2.f * h;
    uint32_t hi_bits;
    std::memcpy(&hi_bits, &hi_d, 4);
    for (int k = 1; k < lsp::kTableSize; k++) {
        uint32_t lo = 0, hi = hi_bits;
        while (lo < hi) {
            uint32_t mid = lo + (hi - lo) / 2;
            float d;
            std::memcpy(&d, &mid, 4);
            if ((int)(d / step) >= k) hi = mid; else lo = mid + 1;
        }
        std::memcpy(&thr[k], &lo, 4);
    }
    thr[lsp::kTableSize] = std::numeric_limits<float>::infinity();
    const float inv_step = 1.f / step;
    uint32_t h_bits;
    std::memcpy(&h_bits, &h, 4);
    unsigned long long bad = 0, total = 0;
    for (uint32_t b = 0; b < h_bits; b++) {
        float d;
        std::memcpy(&d, &b, 4);
        int want = (int)(d / step);
        int got = lsp::table_slot(d, inv_step, thr);
        total++;
        if (want != got) {
            if (bad < 5) std::printf("mismatch d=%.9g want %d got %d\n", d, want, got);
            bad++;
        }
    }
    std::printf("checked %llu floats in [0, h=%.9g): %llu mismatches\n", total, h, bad);
    return bad ? 1 : 0;
}
