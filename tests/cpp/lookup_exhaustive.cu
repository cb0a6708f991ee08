// Exhaustive host check of the device lookup's slot computation (table_slot in
// liquidsimulation_b200/csrc/lsp_device.cuh): for every float d in [0, h) it must equal
// (int)(d / step), the index of the reference's SPHKernel::get*Weight (SPHKernel.cpp:19).
// The thresholds are built by the same bisection as HostKernels::build. Host and device
// share IEEE single rounding (-ffp-contract=off here, -fmad=false in the library), so the
// host result is the device result.
//
// Second part, the squared-distance form (table_slot_sq_from): for every float s below the
// cutoff bound cut2 the slot must equal (int)(sqrt(s) / step) when the first guess of the
// distance is the exact square root or is off by a relative 2^-20 either way (eight times
// the error of the device's approximate square root), and s >= cut2 must hold exactly when
// sqrt(s) >= h.
//   usage: lookup_exhaustive <particle radius> <kernel radius factor>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <cmath>
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
    float thr2[lsp::kTableSize + 1];
    thr2[0] = 0.f;
    for (int k = 1; k < lsp::kTableSize; k++) thr2[k] = sq_bound(thr[k]);
    thr2[lsp::kTableSize] = std::numeric_limits<float>::infinity();
    const float cut2 = sq_bound(h);
    uint32_t c_bits;
    std::memcpy(&c_bits, &cut2, 4);
    unsigned long long bad2 = 0, total2 = 0;
    const double eps = 1.0 / (1 << 20);
    for (uint32_t b = 0; b < c_bits + 4096u; b++) {
        float s;
        std::memcpy(&s, &b, 4);
        const float d = std::sqrt(s);
        if ((d >= h) != (s >= cut2)) {
            if (bad2 < 5) std::printf("cutoff mismatch s=%.9g\n", s);
            bad2++;
        }
        if (b >= c_bits) continue;
        const int want = (int)(d / step);
        const float guesses[3] = {d, (float)(d * (1.0 - eps)), (float)(d * (1.0 + eps))};
        for (float g : guesses) {
            const int got = lsp::table_slot_sq_from(s, g, inv_step, thr2);
            total2++;
            if (want != got) {
                if (bad2 < 5) std::printf("mismatch s=%.9g guess %.9g want %d got %d\n", s, g, want, got);
                bad2++;
            }
        }
    }
    std::printf("checked %llu squared-distance lookups below cut2=%.9g: %llu mismatches\n", total2, cut2, bad2);
    return (bad || bad2) ? 1 : 0;
}
