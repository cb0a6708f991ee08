// Per-particle operations of the step, shared by the single-scene kernels (sph.cu,
// pcisph.cu) and the batched kernels (batch.cu): each function computes one particle's
// result exactly as the reference CPU solver does (citations at each function), so both
// kernel families produce the same bits.
#pragma once

#include "lsp_device.cuh"
#include "lsp_kernels.h"

namespace lsp {

// T_THRESH: slot thresholds on the distance; T_THRESH2: on the squared distance.
enum { T_W = 0, T_DW = 1, T_D2W = 2, T_SPIKY_DW = 3, T_VISC_D2W = 4, T_THRESH = 5, T_THRESH2 = 6 };

// Copies table t (the threshold tables have one entry more) into shared memory.
__device__ __forceinline__ void stage_table(float* sm, const float* g, int t)
{
    const int len = t >= T_THRESH ? kTableSize + 1 : kTableSize;
    const int off = t == T_THRESH2 ? kThresh2Offset : t * kTableSize;
    for (int i = threadIdx.x; i < len; i += blockDim.x) sm[i] = g[off + i];
}
// The non-pressure pass's slot records (NonpressureWeights), built in shared memory from
// the table block g.
__device__ __forceinline__ void stage_nonpressure_slots(float4* ra, float4* rb, const float* g)
{
    const float* th = g + kThresh2Offset;
    const float* dw = g + T_DW * kTableSize;
    const float* d2w = g + T_D2W * kTableSize;
    const float* vd2w = g + T_VISC_D2W * kTableSize;
    for (int k = threadIdx.x; k < kTableSize; k += blockDim.x) {
        const int km = k ? k - 1 : 0;
        ra[k] = make_float4(th[k], dw[km], dw[k], d2w[km]);
        rb[k] = make_float4(d2w[k], vd2w[km], vd2w[k], 0.f);
    }
}

// Cell key of a position inside the scene's grid box: the CPU grid's cell (int)(x / h)
// per axis (SPHSpatialGrid.cpp:80-82), clamped into the box, ordered x slowest and z
// fastest, plus the scene's first cell in a batch.
__device__ __forceinline__ uint32_t cell_key(const DevParams& P, const float4& p, bool& escaped, bool& bad)
{
    bad = !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z));
    int c[3] = {cell_coord(p.x, P.h), cell_coord(p.y, P.h), cell_coord(p.z, P.h)};
    const int o[3] = {P.ox, P.oy, P.oz};
    const int d[3] = {P.nx, P.ny, P.nz};
    escaped = false;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        int v = c[a];
        if (v < o[a]) { v = o[a]; escaped = true; }
        if (v > o[a] + d[a] - 1) { v = o[a] + d[a] - 1; escaped = true; }
        c[a] = v - o[a];
    }
    return P.cell_base + (uint32_t)(((uint32_t)c[0] * (uint32_t)P.ny + (uint32_t)c[1]) * (uint32_t)P.nz + (uint32_t)c[2]);
}

// Start-of-step neighbour list of particle i: every j with |x_i - x_j|^2 <= h^2,
// including i, in the reference's order (SPHSpatialGrid::findNeighborParticles,
// SPHSpatialGrid.cpp:39-76): cell ranges from (x -+ h) / h per axis, x then y rows,
// each row a contiguous z-run of the sorted array. Stores at most nbr_cap entries and
// returns the true count. With kDensity it also sums W over the accepted pairs in list
// order from their squared distances, the sum density_one forms over the stored list
// (|x_i - x_j|^2 equals |x_j - x_i|^2 bit for bit; W and TH2 as in density_one).
template <bool kDensity = false, bool kTail0 = false>
__device__ __forceinline__ int neighbors_one(const DevParams& P, const float4* __restrict__ pos,
                                             const uint32_t* __restrict__ cell_start, int32_t* __restrict__ nbr,
                                             int i, const float* W = nullptr, const float* TH2 = nullptr,
                                             float* wsum = nullptr)
{
    float sum = 0.f;
    const float4 pi = pos[i];
    const V3 xi = v3(pi);
    const float h = P.h;
    int lo[3] = {(int)((xi.x - h) / h), (int)((xi.y - h) / h), (int)((xi.z - h) / h)};
    int hi[3] = {(int)((xi.x + h) / h), (int)((xi.y + h) / h), (int)((xi.z + h) / h)};
    const int o[3] = {P.ox, P.oy, P.oz};
    const int d[3] = {P.nx, P.ny, P.nz};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        // Both ends clamped into the box: a particle outside it searches the edge cell
        // that holds every clamped particle.
        lo[a] = min(max(lo[a], o[a]), o[a] + d[a] - 1) - o[a];
        hi[a] = min(max(hi[a], o[a]), o[a] + d[a] - 1) - o[a];
    }
    const int cap = P.nbr_cap;
    const int64_t stride = P.nbr_stride;
    // Plain column-major (entry c at nbr[c * stride + i]); the non-pressure pass regroups the
    // lists into list_entry's layout for the walks after it.
    int32_t* out = nbr + i;
    int c = 0;
    if (lo[2] <= hi[2]) {
        for (int cx = lo[0]; cx <= hi[0]; cx++) {
            for (int cy = lo[1]; cy <= hi[1]; cy++) {
                uint32_t row = P.cell_base + ((uint32_t)cx * (uint32_t)P.ny + (uint32_t)cy) * (uint32_t)P.nz;
                const uint32_t beg = cell_start[row + lo[2]];
                const uint32_t end = cell_start[row + hi[2] + 1];
                const float4* pe = pos + end;
                int32_t q = (int32_t)beg;
                for (const float4* pq = pos + beg; pq < pe; pq++, q++) {
                    const V3 dq = xi - v3(*pq);
                    const float s = sqmag(dq);
                    if (s <= P.h2) {
                        if (kDensity) sum += lookup_sq<kTail0>(W, TH2, s, P);
                        if (c < cap) {
                            *out = q;
                            out += stride;
                        }
                        c++;
                    }
                }
            }
        }
    }
    if (kDensity) *wsum = sum;
    return c;
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated histogram of cell keys: one atomic per distinct key in the warp; lanes
// with the same key take consecutive slots in lane order. All 32 lanes must call it.
__device__ __forceinline__ uint32_t hist_slot(uint32_t k, bool valid, uint32_t* hist)
{
    const int lane = threadIdx.x & 31;
    uint32_t peers = __match_any_sync(0xffffffffu, k);
    uint32_t leader = __ffs(peers) - 1;
    uint32_t rank = __popc(peers & lanemask_lt());
    uint32_t base = 0;
    if (valid && lane == (int)leader) base = atomicAdd(&hist[k], (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + rank;
}

// Escaped and non-finite positions of the warp, one atomic each. All 32 lanes call it.
__device__ __forceinline__ void record_key_flags(bool valid, bool escaped, bool bad, DevStatus* st)
{
    uint32_t esc = __ballot_sync(0xffffffffu, valid && escaped);
    uint32_t nan = __ballot_sync(0xffffffffu, valid && bad);
    if ((threadIdx.x & 31) == 0) {
        if (esc) atomicAdd(&st->escaped, (uint32_t)__popc(esc));
        if (nan) atomicOr(&st->error_flags, kErrNaN);
    }
}

// The stored neighbour count never exceeds the list capacity, so later passes stay inside
// the list even in an overflowed step; the true count only feeds the step's maximum and the
// overflow flag (one atomic per warp). All 32 lanes call it.
__device__ __forceinline__ void record_neighbor_count(const DevParams& P, int c, bool valid, DevStatus* st)
{
    uint32_t m = valid ? (uint32_t)c : 0u;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0 && m > 0) {
        atomicMax(&st->max_neighbors, m);
        if (m > (uint32_t)P.nbr_cap) atomicOr(&st->error_flags, kErrNeighborOverflow);
    }
}

// SPHSolver::calcParticleDensityPressure, CPU branch (SPHSolver.cpp:442-463).
// The distance serves only the table, so the lookup takes the squared distance (TH2: the
// thresholds on d^2; the same slot and value as the reference's sqrt-then-divide).
__device__ __forceinline__ void density_one(const DevParams& P, const StepBuffers& b, const float* W,
                                            const float* TH2, int i)
{
    const V3 xi = v3(b.pos[i]);
    float sum = 0.f;
    for_each_neighbor<4>(b.nbr, i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return b.pos[j]; },
                         [&](int, float4 pj) { sum += lookup_sq(W, TH2, sqmag(v3(pj) - xi), P); });
    float rho = P.mass * sum;
    float pr = P.stiffness * (rho - P.rho0);
    if (pr < 0.f) pr *= P.neg;
    b.rho[i] = rho;
    b.pres[i] = pr;
}

// SPHSolver::accumulateNonPressureForces, CPU branch (SPHSolver.cpp:201-248). The
// reference walks the list up to three times (normal, colour Laplacian when the normal
// exceeds the threshold, viscosity); each sum is independent, so one walk computes all
// three with the same per-sum rounding. kGrad adds |grad rho|, a warm-start feature. The
// distance serves only the tables (the normal sums the unnormalised difference), so the
// slot comes from the squared distance (slot records NA / NB on d^2).
//
// With kExactDiv its seven quotients by the neighbour density per pair come from one
// reciprocal of rho_j (recip_rn, div_by): the same bits while the step's positions,
// velocities and densities are in range (DevStatus::np_unsafe clear) and the tables' entries
// are (DevParams::exact_tables), since every numerator is then 0 or at least 2^-80 in
// magnitude (nonpressure_one chooses).
template <bool kGrad, bool kExactDiv>
__device__ __forceinline__ void nonpressure_walk(const DevParams& P, const StepBuffers& b, const float4* NA,
                                                 const float4* NB, int i)
{
    const V3 xi = v3(b.pos[i]);
    const V3 vi = v3(b.vel[i]);
    const float rhoi = b.rho[i];
    V3 F = v3(0.f, 0.f, 0.f);
    F += v3(P.gx, P.gy, P.gz) * rhoi;
    V3 normal = v3(0.f, 0.f, 0.f);
    V3 visc = v3(0.f, 0.f, 0.f);
    float lap = 0.f;
    V3 grad = v3(0.f, 0.f, 0.f);   // sum (rho_j - rho_i) / rho_j grad W_ij: a warm-start feature only
    struct Rec {
        float4 x, vr;   // position; velocity and density ({v, rho}, StepBuffers::vrho)
    };
    for_each_neighbor_regroup(b.nbr_src, b.nbr_out, i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return Rec{b.pos[j], b.vrho[j]}; },
                         [&](int j, const Rec& r) {
                             const V3 xj = v3(r.x);
                             V3 dir = xi - xj;
                             // |x_i - x_j|^2 equals |x_j - x_i|^2 bit for bit
                             const NonpressureWeights at(NA, NB, sqmag(dir), P);
                             const float w_dw = at.dw;
                             if (kExactDiv) {
                                 const float y = recip_rn(r.vr.w);
                                 auto q = [&](float a) { return div_by(a, r.vr.w, y); };
                                 const V3 n = dir * w_dw;
                                 normal += v3(q(n.x), q(n.y), q(n.z));
                                 lap += q(at.d2w);
                                 if (j != i) {
                                     const V3 dv = v3(r.vr) - vi;
                                     visc += v3(q(dv.x), q(dv.y), q(dv.z)) * at.vd2w;
                                 }
                                 if (kGrad) grad += dir * (w_dw * q(r.vr.w - rhoi));
                             } else {
                                 normal += dir * w_dw / r.vr.w;
                                 lap += at.d2w / r.vr.w;
                                 if (j != i) visc += ((v3(r.vr) - vi) / r.vr.w) * at.vd2w;
                                 if (kGrad) grad += dir * (w_dw * ((r.vr.w - rhoi) / r.vr.w));
                             }
                         });
    if (kGrad) b.gradrho[i] = P.mass * mag(grad);
    normal *= P.mass;
    float len = mag(normal);
    if (len > P.sigma_thr) F += (normal / len) * (-P.sigma * lap * P.mass);
    visc *= P.viscosity * P.mass;
    F += visc;
    b.force[i] = f4(F, 0.f);
}
template <bool kGrad>
__device__ __forceinline__ void nonpressure_one(const DevParams& P, const StepBuffers& b, const float4* NA,
                                                const float4* NB, int i)
{
    if (P.exact_tables && *(const volatile uint32_t*)&b.status->np_unsafe == 0u)
        nonpressure_walk<kGrad, true>(P, b, NA, NB, i);
    else
        nonpressure_walk<kGrad, false>(P, b, NA, NB, i);
}

// SPHSolver::accumulatePressureForces, CPU branch (SPHSolver.cpp:268-290).
__device__ __forceinline__ void sph_pressure_one(const DevParams& P, const StepBuffers& b, const float* SDW,
                                                 const float* TH, int i)
{
    const V3 xi = v3(b.pos[i]);
    const float rhoi = b.rho[i];
    const float tf = b.pres[i] / (rhoi * rhoi);
    V3 pf = v3(0.f, 0.f, 0.f);
    struct Rec {
        float4 x;
        float rho, p;
    };
    for_each_neighbor<4>(b.nbr, i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return Rec{b.pos[j], b.rho[j], b.pres[j]}; },
                         [&](int j, const Rec& r) {
                             if (j == i) return;
                             const V3 xj = v3(r.x);
                             float d = mag(xi - xj);
                             V3 dir = (xi - xj) / d;
                             pf += dir * lookup(SDW, TH, d, P) * (tf + r.p / (r.rho * r.rho));
                         });
    pf *= -(P.mass * rhoi);
    V3 F = v3(b.force[i]);
    F += pf;
    b.force[i] = f4(F, 0.f);
}

// SPHParticle::integrate (SPHParticle.cpp:30-44) then SPHSolver::handleCollisions
// (SPHSolver.cpp:337-355) for one particle. With add_pforce the PCISPH pressure force is
// added first (PCISPHSolver.cpp:166-169).
__device__ __forceinline__ void integrate_one(const DevParams& P, const StepBuffers& b, int i, int add_pforce)
{
    float4 p4 = b.pos[i], v4 = b.vel[i], h4 = b.half[i], o4 = b.old[i];
    V3 F = v3(b.force[i]);
    if (add_pforce) F += v3(b.pforce[i]);
    const float rho = b.rho[i];
    V3 acc = F / rho;
    V3 half = v3(h4);
    float first = v4.w;
    if (first != 0.f) {
        half = v3(v4) - acc * P.dt / 2.f;
        first = 0.f;
    }
    V3 old = half;
    half = v3(half.x + acc.x * P.dt, half.y + acc.y * P.dt, half.z + acc.z * P.dt);
    V3 x = v3(p4);
    x = v3(x.x + half.x * P.dt, x.y + half.y * P.dt, x.z + half.z * P.dt);
    collide_all(b.colliders + P.coll_off, P.ncoll, x, half, P);
    V3 v = (old + half) / 2.f;
    b.pos[i] = f4(x, p4.w);
    b.vel[i] = f4(v, first);
    b.half[i] = f4(half, h4.w);
    b.old[i] = f4(old, o4.w);
    if (b.hist) {
        // Warm-start pressure history: (p_n, p_{n-1}, p_{n-2}) for the next step's features.
        float4 hs = b.hist[i];
        b.hist[i] = make_float4(b.pres[i], hs.x, hs.y, 0.f);
    }
}

// PCISPHSolver.cpp:67-97 for one particle. Iteration 0 starts from p = 0, F_p = 0
// (:58-62). aproximateVelocity (:96, SPHParticle.cpp:46-49) sets v = (v_half_old + v_half)/2;
// within a step it is idempotent, so it is applied in iteration 0 only, after the
// prediction has read v.
__device__ __forceinline__ void pci_predict_one(const DevParams& P, const StepBuffers& b, int i, int iteration,
                                                float4* ppos)
{
    float4 v4 = b.vel[i];
    V3 F = v3(b.force[i]);
    V3 Fp = iteration == 0 ? v3(0.f, 0.f, 0.f) : v3(b.pforce[i]);
    const float rho = b.rho[i];
    V3 hv = v3(b.half[i]);
    V3 acc = (F + Fp) / rho;
    if (v4.w != 0.f) hv = v3(v4) - acc * P.dt / 2.f;
    V3 ph = hv + acc * P.dt;
    V3 px = v3(b.pos[i]) + ph * P.dt;
    collide_all(b.colliders + P.coll_off, P.ncoll, px, ph, P);
    // The force pass divides by pair distances with div_by while every prediction of the
    // step stays in its exact range; one position outside switches it to IEEE division.
    if (!(exact_div_safe(px.x) && exact_div_safe(px.y) && exact_div_safe(px.z))) atomicOr(&b.status->div_unsafe, 1u);
    ppos[i] = f4(px, 0.f);
    b.phalf[i] = f4(ph, 0.f);
    if (iteration == 0 && !P.keep_initial_velocity) {
        V3 v = (v3(b.old[i]) + v3(b.half[i])) / 2.f;
        b.vel[i] = f4(v, v4.w);
    }
}

// PCISPHSolver.cpp:100-126 for one particle; returns |error| (0 for NaN, which the
// reference's std::max ignores). Table lookups on the squared distance (TH2), as in
// density_one (kTail0: DevParams::density_tail0 holds).
template <bool kTail0 = false>
__device__ __forceinline__ float pci_density_one(const DevParams& P, const StepBuffers& b, const float* W,
                                                 const float* TH2, int i, int iteration, float4* ppos)
{
    const V3 xi = v3(ppos[i]);
    float sum = 0.f;
    for_each_neighbor<4>(b.nbr, i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return ppos[j]; },
                         [&](int, float4 pj) { sum += lookup_sq<kTail0>(W, TH2, sqmag(v3(pj) - xi), P); });
    float pd = P.mass * sum;
    float er = pd - P.rho0;
    float pp = P.delta * er;
    if (pp < 0.f) {
        er *= P.neg;
        pp *= P.neg;
    }
    float p = (iteration == 0 ? 0.f : b.pres[i]) + pp;
    b.prho[i] = pd;
    b.err[i] = er;
    b.pres[i] = p;
    // p / rho*^2, the per-particle factor of the pressure force, rides in x*.w so the force
    // pass fetches a neighbour's position and factor in one 16-byte load. Other threads
    // read only x*.xyz of this element during this pass.
    reinterpret_cast<float*>(ppos + i)[3] = p / (pd * pd);
    float a = fabsf(er);
    return a == a ? a : 0.f;
}

// PCISPHSolver.cpp:129-150 for one particle. s = p / rho*^2 is the per-particle factor the
// reference recomputes per pair; the prefactor uses the current density rho_i. The pair
// distance is an IEEE square root and the direction (x_i - x_j) / d three IEEE quotients;
// with kExactDiv they come from sqrt_rn and one reciprocal of d (recip_rn, div_by), the same
// bits for the predicted positions the step's predict passes found safe
// (DevStatus::div_unsafe clear).
template <bool kExactDiv, bool kTail0 = false>
__device__ __forceinline__ void pci_force_walk(const DevParams& P, const StepBuffers& b, const float* SDW,
                                               const float* TH, int i, const float4* ppos)
{
    const float4 pi4 = ppos[i];
    const V3 xi = v3(pi4);
    const float tf = pi4.w;
    V3 pf = v3(0.f, 0.f, 0.f);
    for_each_neighbor<2>(b.nbr, i, P.nbr_stride, __ldg(b.nbr_count + i),
                         [&](int j) { return ppos[j]; },
                         [&](int j, float4 pj4) {
                             if (j == i) return;
                             // |x_i - x_j| rounds exactly like the reference's |x_j - x_i|
                             // (the squares are equal), so one difference serves both.
                             const V3 dq = xi - v3(pj4);
                             const float d = kExactDiv ? sqrt_rn(sqmag(dq)) : mag(dq);
                             V3 dir;
                             if (kExactDiv) {
                                 const float y = recip_rn(d);
                                 dir = v3(div_by(dq.x, d, y), div_by(dq.y, d, y), div_by(dq.z, d, y));
                             } else {
                                 dir = dq / d;
                             }
                             pf += dir * lookup<kTail0>(SDW, TH, d, P) * (tf + pj4.w);
                         });
    pf *= -(P.mass * b.rho[i]);
    if (isnan(pf.x)) pf = v3(0.f, 0.f, 0.f);
    b.pforce[i] = f4(pf, 0.f);
}
template <bool kTail0 = false>
__device__ __forceinline__ void pci_force_one(const DevParams& P, const StepBuffers& b, const float* SDW,
                                              const float* TH, int i, const float4* ppos)
{
    if (*(const volatile uint32_t*)&b.status->div_unsafe == 0u) pci_force_walk<true, kTail0>(P, b, SDW, TH, i, ppos);
    else pci_force_walk<false, kTail0>(P, b, SDW, TH, i, ppos);
}

}  // namespace lsp
