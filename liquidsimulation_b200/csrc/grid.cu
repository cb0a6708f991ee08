// Uniform-grid build: cell keys, counting sort by (cell, caller id), particle reorder,
// dense cell table, and the start-of-step neighbour lists.
//
// Replaces the reference's per-step grid build, both its CPU hash grid
// (SPHSpatialGrid.cpp:19-90, via SPHSolver.cpp:431-440) and its OpenCL grid
// (calcGridIndices / countDigitsInBuckets / permuteParticles / buildCellList,
// SPHKernels.cl:66-186 with the host scan at SPHSolver.cpp:1052-1119).
//
// Cells are the CPU grid's cells, c = (int)(x / h) per axis, inside a fixed grid box;
// the key orders them x slowest, z fastest, which is the order in which the CPU's
// neighbour search visits cells. Sorting by (key, caller id) therefore lays out every
// 3-cell z-run of the 3x3 row neighbourhood as one contiguous range, in exactly the
// CPU's visiting order, so neighbour lists come out in the reference's order.
//
// The sort is a counting sort (a radix sort whose single digit is the whole cell key):
//   k_keys_hist   key per particle; warp-aggregated histogram (__match_any_sync) with slots
//   k_scan_*      exclusive scan of the histogram = dense cell table (lower bounds)
//   k_scatter     particle -> (cell start + slot)
//   k_rank_gather deterministic rank by caller id inside each cell, then one gather of
//                 the 64-byte persistent state into the new order
//   k_neighbors_density  the start-of-step neighbour lists (plain column-major; the
//                 non-pressure pass regroups them), reference order, with the density and
//                 pressure summed over the accepted pairs
#include "lsp_kernels.h"
#include "particle_ops.cuh"

namespace lsp {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr int kMaxCellOccupancy = 4096;

__global__ void k_keys_hist(DevParams P, const float4* __restrict__ pos, uint32_t* __restrict__ key,
                            uint32_t* __restrict__ slot, uint32_t* __restrict__ hist, DevStatus* st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < P.n;
    uint32_t k = 0xffffffffu;
    bool escaped = false, bad = false;
    if (valid) k = cell_key(P, pos[i], escaped, bad);
    const uint32_t sl = hist_slot(k, valid, hist);
    if (valid) {
        key[i] = k;
        slot[i] = sl;
    }
    record_key_flags(valid, escaped, bad, st);
}

// Block-wide exclusive scan of kScanItems consecutive items per thread, warp shuffles
// inside each warp, then the warp totals.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums, uint32_t* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t warp_prefix = warp ? warp_sums[warp - 1] : 0u;
    if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// The histogram and the cell table are padded with zeros to a multiple of 8 entries
// (scan_entries): each thread moves its 8 consecutive entries as two 16-byte vectors. n8 is
// the padded count.
__device__ __forceinline__ void load8(const uint32_t* p, uint32_t (&v)[kScanItems])
{
    const uint4 a = *reinterpret_cast<const uint4*>(p);
    const uint4 b = *reinterpret_cast<const uint4*>(p + 4);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* __restrict__ in, int64_t n8,
                                                             uint32_t* __restrict__ tile_sums)
{
    __shared__ uint32_t ws[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t s = 0;
    if (base < n8) {
        uint32_t v[kScanItems];
        load8(in + base, v);
#pragma unroll
        for (int j = 0; j < kScanItems; j++) s += v[j];
    }
    uint32_t total;
    block_exclusive_scan(s, ws, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block scans the tile sums in place (exclusive), chunk by chunk with a carry; only
// launched when there are more than kFoldTiles tiles.
__global__ void __launch_bounds__(1024) k_scan_top(uint32_t* tile_sums, int tiles)
{
    __shared__ uint32_t ws[32];
    uint32_t carry = 0;
    for (int b = 0; b < tiles; b += blockDim.x) {
        int i = b + threadIdx.x;
        uint32_t v = i < tiles ? tile_sums[i] : 0u;
        uint32_t total;
        uint32_t ex = block_exclusive_scan(v, ws, &total);
        if (i < tiles) tile_sums[i] = carry + ex;
        carry += total;
        __syncthreads();
    }
}

// Exclusive scan of the histogram into the dense cell table; clears the histogram for the
// next step. With fold, the block sums the tile totals before its own tile (up to kFoldTiles
// of them) itself; otherwise k_scan_top has turned tile_sums into those prefixes.
constexpr int kFoldTiles = 4096;
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(uint32_t* __restrict__ hist, int64_t n8,
                                                             const uint32_t* __restrict__ tile_sums, int fold,
                                                             uint32_t* __restrict__ out)
{
    __shared__ uint32_t ws[32];
    uint32_t prefix;
    if (fold) {
        uint32_t s = 0;
        for (int k = threadIdx.x; k < (int)blockIdx.x; k += blockDim.x) s += tile_sums[k];
        block_exclusive_scan(s, ws, &prefix);
    } else {
        prefix = tile_sums[blockIdx.x];
    }
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (base < n8) load8(hist + base, v);
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) s += v[j];
    uint32_t ex = block_exclusive_scan(s, ws, nullptr) + prefix;
    if (base < n8) {
        uint32_t o[kScanItems];
#pragma unroll
        for (int j = 0; j < kScanItems; j++) {
            o[j] = ex;
            ex += v[j];
        }
        *reinterpret_cast<uint4*>(out + base) = make_uint4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<uint4*>(out + base + 4) = make_uint4(o[4], o[5], o[6], o[7]);
        *reinterpret_cast<uint4*>(hist + base) = make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(hist + base + 4) = make_uint4(0u, 0u, 0u, 0u);
    }
}

__global__ void k_scatter(DevParams P, const float4* __restrict__ pos, const uint32_t* __restrict__ key,
                          const uint32_t* __restrict__ slot, const uint32_t* __restrict__ cell_start,
                          int2* __restrict__ tmp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    uint32_t k = key[i];
    tmp[cell_start[k] + slot[i]] = make_int2(i, id_of(pos[i]));
}

// Final slot = cell start + number of particles of the same cell with a smaller caller id.
// Then moves the particle's persistent state (x|id, v|first, v_half|p1, v_half_old|p2).
__global__ void k_rank_gather(DevParams P, const int2* __restrict__ tmp, const uint32_t* __restrict__ key,
                              const uint32_t* __restrict__ cell_start,
                              const float4* __restrict__ ipos, const float4* __restrict__ ivel,
                              const float4* __restrict__ ihalf, const float4* __restrict__ iold,
                              float4* __restrict__ opos, float4* __restrict__ ovel,
                              float4* __restrict__ ohalf, float4* __restrict__ oold,
                              int32_t* __restrict__ slot_of_id, uint32_t* __restrict__ sorted_key, DevStatus* st,
                              const float4* __restrict__ ihist, float4* __restrict__ ohist)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.n) return;
    int2 e = tmp[p];
    uint32_t k = key[e.x];
    uint32_t beg = cell_start[k], end = cell_start[k + 1];
    uint32_t rank = 0;
    if (end - beg <= (uint32_t)kMaxCellOccupancy) {
        for (uint32_t q = beg; q < end; q++) rank += tmp[q].y < e.y ? 1u : 0u;
    } else {
        rank = (uint32_t)p - beg;   // order inside an overfull cell is not the reference's
        atomicOr(&st->error_flags, kErrScan);
    }
    uint32_t dest = beg + rank;
    const float4 x = ipos[e.x], v = ivel[e.x];
    opos[dest] = x;
    ovel[dest] = v;
    // The non-pressure pass divides pair terms by densities with div_by while every position
    // and velocity of the step is in exact_div_safe's range.
    if (!(exact_div_safe(x.x) && exact_div_safe(x.y) && exact_div_safe(x.z) && exact_div_safe(v.x) &&
          exact_div_safe(v.y) && exact_div_safe(v.z)))
        atomicOr(&st->np_unsafe, 1u);
    ohalf[dest] = ihalf[e.x];
    oold[dest] = iold[e.x];
    if (ohist) ohist[dest] = ihist[e.x];
    slot_of_id[e.y] = (int32_t)dest;
    sorted_key[dest] = k;
}

// Start-of-step neighbour lists (neighbors_one, plain column-major) plus the start-of-step density
// and pressure of density_one (SPHSolver::calcParticleDensityPressure,
// SPHSolver.cpp:442-463), summed while the list is built: a pass over the stored list and
// its position gathers would cost more. (A list that
// overflows its capacity raises the overflow flag and the step is redone, so the sum over
// every accepted pair never differs from the stored list's.)
template <bool kTail0>
__global__ void k_neighbors_density(DevParams P, const float4* __restrict__ pos,
                                    const uint32_t* __restrict__ cell_start, int32_t* __restrict__ nbr,
                                    int32_t* __restrict__ count, DevStatus* st, const float* __restrict__ tables,
                                    float* __restrict__ rho, float* __restrict__ pres,
                                    const float4* __restrict__ vel, float4* __restrict__ vrho)
{
    __shared__ float W[kTableSize], TH2[kTableSize + 1];
    stage_table(W, tables, T_W);
    stage_table(TH2, tables, T_THRESH2);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < P.n;
    int c = 0;
    if (valid) {
        float sum;
        c = neighbors_one<true, kTail0>(P, pos, cell_start, nbr, i, W, TH2, &sum);
        count[i] = min(c, P.nbr_cap);
        const float r = P.mass * sum;
        float pr = P.stiffness * (r - P.rho0);
        if (pr < 0.f) pr *= P.neg;
        rho[i] = r;
        pres[i] = pr;
        const float4 v = vel[i];
        vrho[i] = make_float4(v.x, v.y, v.z, r);
        if (!exact_div_density(r)) atomicOr(&st->np_unsafe, 1u);
    }
    record_neighbor_count(P, c, valid, st);
}

// ------------------------------------------------------------------ launchers

static inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int launch_grid_keys(const GridBuildArgs& a, cudaStream_t s)
{
    if (a.P.n <= 0) return 0;
    k_keys_hist<<<blocks_for(a.P.n, 256), 256, 0, s>>>(a.P, a.pos_in, a.key, a.slot, a.hist, a.status);
    return 1;
}

int launch_grid_scan(const GridBuildArgs& a, cudaStream_t s)
{
    const int64_t n8 = scan_entries((int64_t)a.P.cells + 1);
    const int tiles = (int)scan_tiles((int64_t)a.P.cells + 1);
    k_scan_tiles<<<tiles, kScanThreads, 0, s>>>(a.hist, n8, a.tile_sums);
    const int fold = tiles <= kFoldTiles ? 1 : 0;
    if (!fold) k_scan_top<<<1, 1024, 0, s>>>(a.tile_sums, tiles);
    k_scan_apply<<<tiles, kScanThreads, 0, s>>>(a.hist, n8, a.tile_sums, fold, a.cell_start);
    return fold ? 2 : 3;
}

int launch_grid_scatter(const GridBuildArgs& a, cudaStream_t s)
{
    if (a.P.n <= 0) return 0;
    k_scatter<<<blocks_for(a.P.n, 256), 256, 0, s>>>(a.P, a.pos_in, a.key, a.slot, a.cell_start, a.tmp);
    return 1;
}

int launch_grid_gather(const GridBuildArgs& a, cudaStream_t s)
{
    if (a.P.n <= 0) return 0;
    k_rank_gather<<<blocks_for(a.P.n, 256), 256, 0, s>>>(a.P, a.tmp, a.key, a.cell_start, a.pos_in, a.vel_in,
                                                         a.half_in, a.old_in, a.pos_out, a.vel_out, a.half_out,
                                                         a.old_out, a.slot_of_id, a.sorted_key, a.status,
                                                         a.hist_in, a.hist_out);
    return 1;
}

int launch_grid_order(const GridBuildArgs& a, cudaStream_t s)
{
    const int T = 256;
    const DevParams& P = a.P;
    int launches = launch_grid_scan(a, s);
    if (P.n > 0) {
        k_scatter<<<blocks_for(P.n, T), T, 0, s>>>(P, a.pos_in, a.key, a.slot, a.cell_start, a.tmp);
        k_rank_gather<<<blocks_for(P.n, T), T, 0, s>>>(P, a.tmp, a.key, a.cell_start, a.pos_in, a.vel_in,
                                                       a.half_in, a.old_in, a.pos_out, a.vel_out, a.half_out,
                                                       a.old_out, a.slot_of_id, a.sorted_key, a.status, a.hist_in,
                                                       a.hist_out);
        launches += 2;
    }
    return launches;
}

int launch_grid_sort(const GridBuildArgs& a, cudaStream_t s)
{
    const int T = 256;
    const DevParams& P = a.P;
    int launches = 0;
    if (P.n > 0) {
        k_keys_hist<<<blocks_for(P.n, T), T, 0, s>>>(P, a.pos_in, a.key, a.slot, a.hist, a.status);
        launches++;
    }
    return launches + launch_grid_order(a, s);
}

int launch_neighbors(const GridBuildArgs& a, cudaStream_t s)
{
    const int T = 256;
    if (a.P.n <= 0) return 0;
    if (a.P.density_tail0)
        k_neighbors_density<true><<<blocks_for(a.P.n, T), T, 0, s>>>(a.P, a.pos_out, a.cell_start, a.nbr, a.nbr_count,
                                                                     a.status, a.tables, a.rho, a.pres, a.vel_out,
                                                                     a.vrho);
    else
        k_neighbors_density<false><<<blocks_for(a.P.n, T), T, 0, s>>>(a.P, a.pos_out, a.cell_start, a.nbr,
                                                                      a.nbr_count, a.status, a.tables, a.rho, a.pres,
                                                                      a.vel_out, a.vrho);
    return 1;
}

}  // namespace lsp
