// Device-side types and per-particle arithmetic shared by all kernels.
//
// All translation units of liblsp are compiled with -fmad=false -prec-div=true
// -prec-sqrt=true -ftz=false: every +, -, *, / and sqrtf below rounds once, IEEE
// round-to-nearest, in source order. The per-particle expressions restate the
// reference's CPU solver operation by operation (citations at each function), so
// each particle's result matches the reference's bits when the neighbour sums are
// taken in the same order, which the grid build guarantees.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace lsp {

constexpr int kTableSize = 1001;        // SPHKernel m_subdivision = 1000 (SPHKernel.cpp:4-7)
// Kernel table block: 5 tables of kTableSize, the kTableSize + 1 slot thresholds on the
// distance, then the kTableSize + 1 thresholds on the squared distance.
constexpr int kThreshOffset = 5 * kTableSize;
constexpr int kThresh2Offset = kThreshOffset + kTableSize + 1;
constexpr int kTableFloats = kThresh2Offset + kTableSize + 1;
constexpr int kMaxColliders = 64;
constexpr int kMaxIterationsCap = 1024;

// Error bits of DevStatus::error_flags.
constexpr uint32_t kErrNaN = 1u;             // non-finite position or density
constexpr uint32_t kErrNeighborOverflow = 2u; // a neighbour list exceeded its capacity
constexpr uint32_t kErrTimeout = 4u;         // a bounded grid barrier gave up
constexpr uint32_t kErrScan = 8u;            // the cell scan saw inconsistent counts

struct Collider {
    int sphere;     // 0 box, 1 sphere
    int boundary;   // 0 obstacle (keep out), 1 boundary (keep in)
    float cx, cy, cz;
    float hx, hy, hz;   // box half extents
    float radius;       // sphere radius
    float pad;
};

struct DevStatus {
    uint32_t error_flags;
    uint32_t escaped;
    uint32_t max_neighbors;
    uint32_t max_err_bits;      // float bits of the current iteration's max |density error|
    int32_t iterations;
    int32_t converged;
    int32_t warm_used;
    uint32_t barrier_count;     // grid barrier arrivals (persistent loop)
    uint32_t barrier_gen;
    uint32_t timeout_site;
    float last_ratio;
    int32_t last_k;             // logical index of the loop's last iteration (persistent loop)
    uint32_t div_unsafe;        // a predicted position left exact_div_safe's range this step
    uint32_t np_unsafe;         // a start-of-step position, velocity or density left the range
                                // where the non-pressure pass divides with div_by
    uint32_t pad[2];
};

struct DevParams {
    float gx, gy, gz;
    float h;            // kernel radius = grid spacing
    float h2;           // h * h, the neighbour-test bound (SPHSpatialGrid.cpp:69)
    float cut2;         // smallest float s with sqrt(s) >= h: the table cutoff on d^2
    float step;         // table division step h / 1000 (SPHKernel.cpp:134-137)
    float inv_step;     // 1 / step, rounded (only a first guess of the table slot)
    float radius;       // particle radius (collisions)
    float mass;
    float rho0;
    float stiffness;
    float neg;          // negative pressure factor
    float viscosity;
    float sigma;
    float sigma_thr;
    float restitution;
    float friction;
    float delta;        // PCISPH pressure scaling of this step
    float eta;
    float dt;
    int n;
    int keep_initial_velocity;
    int ncoll;
    int ox, oy, oz;     // grid origin in cell coordinates
    int nx, ny, nz;     // grid dimensions
    uint32_t cells;
    int nbr_cap;        // neighbour list capacity per particle
    int64_t nbr_stride; // column stride of the neighbour list (>= n)
    int min_it, max_it;
    // Batches of scenes (all zero for a single scene): the scene's first particle slot,
    // its first cell in the batch's cell table and its first collider.
    int base;
    uint32_t cell_base;
    int coll_off;
    int scene;
    int exact_tables;   // HostKernels::exact_tables
    int density_tail0;  // HostKernels::density_tail0
    int force_tail0;    // HostKernels::force_tail0
};

// ----------------------------------------------------------------- vector ops
// Vector3D semantics (LiquidPhysics/src/Math/Vector3D.cpp): component-wise, in order.
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3(const float4& a) { return V3{a.x, a.y, a.z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ void operator+=(V3& a, V3 b) { a.x = a.x + b.x; a.y = a.y + b.y; a.z = a.z + b.z; }
__device__ __forceinline__ void operator*=(V3& a, float s) { a.x = a.x * s; a.y = a.y * s; a.z = a.z * s; }
// Vector3D::operator*(Vector3D) is a dot product (Vector3D.cpp:133-136).
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// Vector3D::squareMagnitude / magnitude (Vector3D.cpp:55-63).
__device__ __forceinline__ float sqmag(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__device__ __forceinline__ float mag(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
// Vector3D::normalize (Vector3D.cpp:66-71): scale by the rounded reciprocal.
__device__ __forceinline__ void normalize(V3& a)
{
    float m = mag(a);
    if (m > 0.f) a *= (1.f / m);
}
__device__ __forceinline__ float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// Correctly rounded quotients a / d from one reciprocal per denominator, after Markstein's
// method (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Develop. 34(1), 1990; "IA-64 and Elementary Functions", 2000,
// ch. 8): one Newton-Raphson step with fused multiply-adds turns the hardware's approximate
// reciprocal (within one ulp) into RN(1 / d), and with y = RN(1 / d) and q0 = RN(a * y),
// within one ulp of a / d, the residual r = a - d * q0 is exact and RN(q0 + r * y) is
// RN(a / d). recip_rn is checked against the IEEE reciprocal for every positive normal
// float and div_by against IEEE division on billions of pairs
// (tests/cpp/exact_div_check.cu). The theorem needs every value normal: callers use them
// only where 2^-51 <= d <= 2^28 and a is 0 or 2^-51 <= |a| <= d (exact_div_safe). A zero
// numerator gives a zero of either sign, which adds to a sum started at +0 like the IEEE
// quotient's zero does.
__device__ __forceinline__ float recip_rn(float d)
{
    float y0;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(d));
    const float e = __fmaf_rn(-d, y0, 1.f);
    return __fmaf_rn(e, y0, y0);
}
__device__ __forceinline__ float div_by(float a, float d, float y)
{
    const float q0 = __fmul_rn(a, y);
    const float r = __fmaf_rn(-d, q0, a);
    return __fmaf_rn(r, y, q0);
}
// The IEEE square root of s in the same style: the approximate reciprocal square root, then
// one correction with the exact residual s - g^2 (Markstein's square-root step). Equal to
// the IEEE square root for every float s >= 2^-102 (checked for every one on the GPU,
// tests/cpp/exact_div_check.cu); below that the residual underflows and it is not exact.
// s = 0 gives NaN where IEEE gives 0: the force pass only takes it for pairs j != i, whose
// direction is 0 / 0 = NaN either way at zero distance.
__device__ __forceinline__ float sqrt_rn(float s)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(s));
    const float g = __fmul_rn(s, y);
    const float h = __fmul_rn(0.5f, y);
    const float r = __fmaf_rn(-g, g, s);
    return __fmaf_rn(r, h, g);
}
// A density the non-pressure pass may divide by with div_by: 2^-20 <= rho <= 2^20 (so that
// with numerators 0 or at least 2^-80 in magnitude every quotient and residual stays normal).
__device__ __forceinline__ bool exact_div_density(float r) { return r >= 0x1p-20f && r <= 0x1p20f; }
// A coordinate with which every pair difference, its squared length and its quotient by the
// pair distance stay where sqrt_rn and div_by are exact: 0, or 2^-28 <= |c| <= 2^26 (nonzero
// differences of such floats are at least 2^-51, squared lengths at least 2^-102 and at most
// 3 * 2^54, distances at most 2^28).
__device__ __forceinline__ bool exact_div_safe(float c)
{
    const float a = fabsf(c);
    return a == 0.f || (a >= 0x1p-28f && a <= 0x1p26f);
}

// SPHKernel::get*Weight (SPHKernel.cpp:13-44): zero at or beyond h, else the table
// entry at trunc(d / step), with d / step rounded as IEEE division rounds it.
//
// The slot is found without a division. thr[k] (kTableSize + 1 entries, built on the
// host by bisection over floats) is the smallest distance whose IEEE quotient d / step
// truncates to at least k, so the exact slot is the largest k with thr[k] <= d. An
// approximate quotient d * (1 / step), rounded to the nearest integer by the magic-number
// addition (1.5 * 2^23), lands on that slot or the one above it (its relative error is a
// few ulp and d / step < 1001), and one comparison with thr picks the right one. The
// clamp keeps any input inside the table (slots 0..1000; NaN takes slot 1000, +inf too,
// and the cutoff zeroes the latter).
__host__ __device__ __forceinline__ int slot_guess(float d, float inv_step)
{
    float r = d * inv_step + 12582912.f;
    int32_t bits;
    memcpy(&bits, &r, 4);
    int k = bits - 0x4B400000;
    return k < 1 ? 1 : (k > kTableSize - 1 ? kTableSize - 1 : k);
}
__host__ __device__ __forceinline__ int table_slot(float d, float inv_step, const float* thr)
{
    const int k = slot_guess(d, inv_step);
    return !(d < thr[k]) ? k : k - 1;
}

// The same slot from the squared distance s = |dx|^2 for passes that need the distance only
// for the table: the IEEE square root is monotone, so sqrt(s) >= thr[k] exactly when
// s >= thr2[k] (thr2[k]: the smallest float whose rounded square root reaches thr[k], built
// on the host by bisection). The first guess uses the approximate square root (relative
// error near 2^-23, far inside the half-slot margin of the rounding guess); the comparison
// is exact, so the slot is the one sqrt(s) would give, without the IEEE square root.
__host__ __device__ __forceinline__ int table_slot_sq_from(float s, float d_guess, float inv_step, const float* thr2)
{
    const int k = slot_guess(d_guess, inv_step);
    return !(s < thr2[k]) ? k : k - 1;
}
__device__ __forceinline__ int table_slot_sq(float s, float inv_step, const float* thr2)
{
    float d;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(d) : "f"(s));
    return table_slot_sq_from(s, d, inv_step, thr2);
}

// The table read is unconditional (the slot is always inside the table) and the cutoff a
// select: measured faster than branching around the read.
// kTail0 (DevParams::force_tail0, for the spiky table): every d >= h takes slot 1000, whose
// entry is a zero, so the cutoff's select is left out. (Its sign may be negative; a force sum
// starts at +0 and a sum of roundings to nearest never reaches -0 from there, so adding either
// zero leaves it unchanged.)
template <bool kTail0 = false>
__device__ __forceinline__ float lookup(const float* tab, const float* thr, float d, const DevParams& P)
{
    const float w = tab[table_slot(d, P.inv_step, thr)];
    return (kTail0 || !(d >= P.h)) ? w : 0.f;
}
// lookup(tab, thr, sqrt(s), P) bit for bit, from the squared distance (d >= h exactly when
// s >= cut2).
// kTail0 (DevParams::density_tail0, for the W table): every s >= cut2 takes slot 1000,
// whose entry is +0, so the cutoff's select is redundant and left out.
template <bool kTail0 = false>
__device__ __forceinline__ float lookup_sq(const float* tab, const float* thr2, float s, const DevParams& P)
{
    const float w = tab[table_slot_sq(s, P.inv_step, thr2)];
    return (kTail0 || !(s >= P.cut2)) ? w : 0.f;
}

// The non-pressure pass reads three tables at one squared distance s. Its slot records
// a[k] = {thr2[k], DW[k-1], DW[k], D2W[k-1]} and b[k] = {D2W[k], VD2W[k-1], VD2W[k], -} give
// all three values with two 16-byte shared-memory reads once the first guess k is known,
// instead of a threshold read followed by three dependent table reads (measured 6.6 %
// faster; for one table the split threshold and table reads are faster). The slot is the
// one table_slot_sq_from picks, so the values are the same entries.
struct NonpressureWeights {
    float dw, d2w, vd2w;
    __device__ __forceinline__ NonpressureWeights(const float4* ra, const float4* rb, float s, const DevParams& P)
    {
        float g;
        asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(g) : "f"(s));
        const int k = slot_guess(g, P.inv_step);
        const float4 a = ra[k], b = rb[k];
        const bool hi = !(s < a.x);
        const bool inside = !(s >= P.cut2);
        dw = inside ? (hi ? a.z : a.y) : 0.f;
        d2w = inside ? (hi ? b.x : a.w) : 0.f;
        vd2w = inside ? (hi ? b.z : b.y) : 0.f;
    }
};

// ----------------------------------------------------------------- collisions
// StaticCollisionObject::resolveCollisionWithParticle (StaticCollisionObject.cpp:21-38).
__device__ __forceinline__ void resolve(V3& pos, V3& vel, V3 n, V3 point, const DevParams& P)
{
    float sep = dot(vel, n);
    if (sep < 0.f) {
        V3 vn = n * sep;
        V3 vt = vel - vn;
        vn *= -P.restitution;
        vt *= P.friction;
        vel = vn + vt;
    }
    pos = point;
}

// StaticCollisionBox (StaticCollisionBox.cpp:10-118) and StaticCollisionSphere
// (StaticCollisionSphere.cpp:10-56) detection, then resolve on contact.
__device__ __forceinline__ void collide(const Collider& o, V3& pos, V3& vel, const DevParams& P)
{
    const float r = P.radius;
    V3 c = v3(o.cx, o.cy, o.cz);
    V3 n = v3(0.f, 0.f, 0.f);
    V3 point = pos;
    bool found = false;
    if (!o.sphere) {
        V3 half = v3(o.hx, o.hy, o.hz);
        V3 dv = c - pos;
        V3 dist = v3(fabsf(dv.x), fabsf(dv.y), fabsf(dv.z));
        if (!o.boundary) {
            V3 pen = half - dist;
            pen = v3(pen.x + r, pen.y + r, pen.z + r);
            if (pen.x > 0.f && pen.y > 0.f && pen.z > 0.f) {
                found = true;
                if (pen.x <= pen.y && pen.x <= pen.z) {
                    n.x = (pos.x - c.x >= 0.f) ? 1.f : -1.f;
                    point.x = c.x + n.x * (half.x + r);
                } else if (pen.y <= pen.x && pen.y <= pen.z) {
                    n.y = (pos.y - c.y >= 0.f) ? 1.f : -1.f;
                    point.y = c.y + n.y * (half.y + r);
                } else if (pen.z <= pen.y && pen.z <= pen.x) {
                    n.z = (pos.z - c.z >= 0.f) ? 1.f : -1.f;
                    point.z = c.z + n.z * (half.z + r);
                }
            }
        } else {
            V3 pen = dist - half;
            pen = v3(pen.x + r, pen.y + r, pen.z + r);
            if (pen.x > 0.f || pen.y > 0.f || pen.z > 0.f) {
                found = true;
                if (pen.x > 0.f) {
                    n.x = (pos.x - c.x <= 0.f) ? 1.f : -1.f;
                    point.x = c.x - n.x * (half.x - r);
                }
                if (pen.y > 0.f) {
                    n.y = (pos.y - c.y <= 0.f) ? 1.f : -1.f;
                    point.y = c.y - n.y * (half.y - r);
                }
                if (pen.z > 0.f) {
                    n.z = (pos.z - c.z <= 0.f) ? 1.f : -1.f;
                    point.z = c.z - n.z * (half.z - r);
                }
                normalize(n);
            }
        }
    } else {
        float R = o.radius;
        float dist = mag(c - pos);
        float pen = o.boundary ? dist - (R - r) : (R + r) - dist;
        if (pen > 0.f) {
            found = true;
            // Contact point from the un-normalised normal (StaticCollisionSphere.cpp:44-50).
            if (!o.boundary) {
                n = pos - c;
                point = c + n * (R + r);
            } else {
                n = c - pos;
                point = c - n * (R - r);
            }
            normalize(n);
        }
    }
    if (found) resolve(pos, vel, n, point, P);
}

__device__ __forceinline__ void collide_all(const Collider* cols, int ncoll, V3& pos, V3& vel, const DevParams& P)
{
    for (int c = 0; c < ncoll; c++) collide(cols[c], pos, vel, P);
}

// Neighbour-list layout: entry k of particle i is component k & 3 of the int4 at group k >> 2,
// and each group is column-major over the particles (group g of particle i at
// ((int4*)nbr)[g * stride + i]). A reader fetches four indices with one coalesced 16-byte
// load. The neighbour build writes plain column-major lists (one 4-byte store per accepted
// entry, the cheapest for its accept branch) and the non-pressure pass, which walks every
// list first, stores them in this layout (for_each_neighbor_regroup).
__device__ __forceinline__ int list_entry(const int32_t* __restrict__ nbr, int64_t stride, int64_t i, int k)
{
    return nbr[(((int64_t)(k >> 2) * stride + i) << 2) + (k & 3)];
}

// for_each_neighbor (B = 2) over particle i's plain column-major list `src` (entry k at
// src[k * stride + i]) that also stores the list in list_entry's grouped layout at `dst`: every
// second pair of entries completes a group, which goes out as one 16-byte store (all lanes store
// in step, so the stores coalesce), and the next pair's indices are in flight while the current
// pair's records are fetched and its pairs computed, as in for_each_neighbor.
template <typename Load, typename F>
__device__ __forceinline__ void for_each_neighbor_regroup(const int32_t* __restrict__ src, int32_t* __restrict__ dst,
                                                          int i, int64_t stride, int cnt, Load load, F f)
{
    const int32_t* l = src + i;
    int32_t* g = dst + 4 * (int64_t)i;   // the current group of particle i
    const int full = cnt >> 1;
    int j0 = 0, j1 = 0;
    if (full > 0) {
        j0 = __ldg(l);
        j1 = __ldg(l + stride);
        l += 2 * stride;
    }
    int p0 = 0, p1 = 0;   // the first pair of the current group
    for (int b = 0; b < full; b++) {
        const auto r0 = load(j0);
        const auto r1 = load(j1);
        int n0 = 0, n1 = 0;
        if (b + 1 < full) {
            n0 = __ldg(l);
            n1 = __ldg(l + stride);
            l += 2 * stride;
        }
        if (b & 1) {
            *reinterpret_cast<int4*>(g) = make_int4(p0, p1, j0, j1);
            g += 4 * stride;
        } else {
            p0 = j0;
            p1 = j1;
        }
        f(j0, r0);
        f(j1, r1);
        j0 = n0;
        j1 = n1;
    }
    // The last, partial group: a pending pair and / or the odd last entry (its unused
    // components are never read).
    if (cnt & 1) {
        const int jj = __ldg(l);
        *reinterpret_cast<int4*>(g) = (full & 1) ? make_int4(p0, p1, jj, 0) : make_int4(jj, 0, 0, 0);
        f(jj, load(jj));
    } else if (full & 1) {
        *reinterpret_cast<int4*>(g) = make_int4(p0, p1, 0, 0);
    }
}

// Walks particle i's neighbour list in list order, software pipelined: while a group's
// records are fetched and its pairs computed (B records at a time, B = 1, 2 or 4), the next
// group's four indices are already in flight, so the list's DRAM latency overlaps the
// arithmetic. f(j, record) runs strictly in list order, so every sum accumulates in the
// reference's order.
template <int B, typename Load, typename F>
__device__ __forceinline__ void for_each_neighbor(const int32_t* __restrict__ nbr, int i, int64_t stride, int cnt,
                                                  Load load, F f)
{
    static_assert(B == 1 || B == 2 || B == 4, "a walk batch divides the 4-entry group");
    const int4* g = reinterpret_cast<const int4*>(nbr) + i;
    const int full = cnt >> 2;
    const int rest = cnt & 3;
    int4 cur = make_int4(0, 0, 0, 0);
    if (cnt > 0) cur = __ldg(g);
    for (int q = 0; q < full; q++) {
        g += stride;
        int4 nxt = make_int4(0, 0, 0, 0);
        if (q + 1 < full || rest) nxt = __ldg(g);
        const int j[4] = {cur.x, cur.y, cur.z, cur.w};
#pragma unroll
        for (int s0 = 0; s0 < 4; s0 += B) {
            decltype(load(0)) r[B];
#pragma unroll
            for (int u = 0; u < B; u++) r[u] = load(j[s0 + u]);
#pragma unroll
            for (int u = 0; u < B; u++) f(j[s0 + u], r[u]);
        }
        cur = nxt;
    }
    // The last, partial group: its first `rest` components.
    if (rest > 0) f(cur.x, load(cur.x));
    if (rest > 1) f(cur.y, load(cur.y));
    if (rest > 2) f(cur.z, load(cur.z));
}

// Cell coordinate of the reference's CPU grid (SPHSpatialGrid.cpp:80-82).
__device__ __forceinline__ int cell_coord(float x, float h) { return (int)(x / h); }

__device__ __forceinline__ int id_of(const float4& p) { return __float_as_int(p.w); }

}  // namespace lsp
