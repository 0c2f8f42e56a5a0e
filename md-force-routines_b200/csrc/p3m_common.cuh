// Shared device-side definitions of the p3m_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "p3m_b200.h"
#include "p3m_list_layout.h"  // PP_LIST_PAD and the neighbour-list layout

namespace p3m {

// Mesh bricks of the deterministic charge assignment: a brick is BRICK^3 base
// cells; the order-6 stencil of a particle with base index i reaches nodes
// i..i+5 (yukawa_pm_ord6.py:52-93), so a brick's tile spans BRICK+5 nodes.
constexpr int BRICK = 16;
constexpr int HALO = 5;
constexpr int TILE = BRICK + HALO;
constexpr int TILE3 = TILE * TILE * TILE;

// Lines per pencil tile in the FFT passes (consecutive y rows or z lines).
constexpr int PENCIL = 16;
constexpr int LOG_PENCIL = 4;
static_assert(PENCIL == 1 << LOG_PENCIL, "PENCIL is 2^LOG_PENCIL");
// Complex lines per item of the x passes (two real rows each): 32, or M/2 for
// M = 32, so each radix pass has a group for every one of 256 threads; 16 at
// M = 256, where the shorter items balance the last wave (FFT 0.576 against
// 0.587 ms at 256^3; at 64^3 16 lines measured 0.144 against 0.130).
constexpr int XL_MAX = 32;
// PP cells are at least (rc + skin) / D wide (D, the cell divisor of a
// context: 1 or 2), so the neighbours of a particle lie in the (2 D + 1)^3
// cells around its own.
constexpr int CELL_DIV_MAX = 2;
__host__ __device__ constexpr int cell_stencil(int d) { return (2 * d + 1) * (2 * d + 1) * (2 * d + 1); }
__host__ __device__ constexpr int x_lines_log(int logM)
{
    return logM >= 8 ? 4 : (logM - 1 < 5 ? logM - 1 : 5);
}
constexpr int MAX_LOGM = 8;  // M <= 256
constexpr int PBLK = 256;      // particles per block in replica-aligned particle kernels

// Device status bits (first error wins in the host's reading order).
enum : int {
    ST_BOX = 1,        // particle outside [-L, 2L) or position not finite
    ST_NONFINITE = 2,  // NaN/Inf in velocities, forces or energies (read first)
    ST_NBOVF = 4,      // a particle has more list neighbours than the list holds
};

// Intervals of the tabulated FP32 pair functions on [0, rc].
#ifndef P3M_PP_TABLE_N
#define P3M_PP_TABLE_N 512
#endif
constexpr int PP_TABLE_N = P3M_PP_TABLE_N;  // FP32 pair table: cubic intervals on [0, rc]

// Per-replica constants. Offsets index the concatenated device arrays.
struct RepDev {
    int n, p_off;          // particles, offset into particle arrays
    int M, logM;           // mesh side and log2
    int nc, cell_off;      // PP cells per side, offset into cell arrays
    int nb, brick_off;     // bricks per side, offset into brick arrays
    long long mesh_off;    // offset into real meshes (M^3 per replica)
    long long spec_off;    // offset into half spectra ((M/2+1) M^2)
    long long tile_off;    // offset into assignment tiles (nb^3 TILE^3)
    // work-item offsets of the mesh passes (prefix sums over replicas)
    int wa_off;            // x-R2C / x-C2R items: M * M/(2 x_lines)
    int wb_off;            // y-line items: (M/2+1) * M/PENCIL (multi-pass replicas)
    int wc_off;            // z-line items: (M/2+1) * M/PENCIL (multi-pass replicas)
    int wp_off;            // plane items: M/2+1 (replicas with M <= PLANE_MAX)
    int blk_off;           // offset of this replica's particle blocks (PBLK each)
    int pp_blk_off;        // offset of this replica's blocks in the PP force kernel
    int nq_blk_off;        // offset of this replica's blocks in the n(q,t) kernel
    int sc_off;            // first brick-sort chunk (DevState::sort_ch particles) of this replica
    long long sh_off;      // offset into the brick-sort count table (chunks x nb^3)
    double L, kappa, alpha, rc, cellw, h, dt, t_desired, af, uf, kf;
    double skin, rcl;      // Verlet skin and list cutoff rc + skin
    double pbuf;           // inner-list buffer: the pair kernel reads the outer-list entries
                           // closer than rc + pbuf (0: it reads the outer list itself)
    double qmax;           // largest |charge| of the replica
    double inv_cellw, inv_h, inv_L, inv_V;
};

template <typename T> struct V4;
template <> struct V4<float> { using t = float4; };
template <> struct V4<double> { using t = double4; };
template <typename T> struct C2;
template <> struct C2<float> { using t = float2; };
template <> struct C2<double> { using t = double2; };

template <typename T>
__device__ __forceinline__ typename C2<T>::t make_c(T x, T y)
{
    typename C2<T>::t r;
    r.x = x;
    r.y = y;
    return r;
}

template <typename T>
__device__ __forceinline__ typename C2<T>::t cmul(typename C2<T>::t a, typename C2<T>::t b)
{
    typename C2<T>::t r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// Replica owning a global index: largest r with off(r) <= idx.
template <typename F>
__device__ __forceinline__ int find_rep(int idx, int nrep, F off)
{
    int lo = 0, hi = nrep - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (off(mid) <= idx) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (fixed tree). All threads must call it; the result
// is valid in thread 0. `scratch` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *scratch)
{
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x < 32) {
        int nw = (blockDim.x + 31) >> 5;
        t = (lane < nw) ? scratch[lane] : 0.0;
        t = warp_sum(t);
    }
    return t;
}

__device__ __forceinline__ void raise_status(int *status, int bit)
{
    atomicOr(status, bit);
}

// Asynchronous global -> shared copies (cp.async, 4 or 8 bytes per thread),
// so a block can have all of a tile's loads in flight at once.
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem_dst, const void *gmem_src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(gmem_src), "n"(BYTES));
}
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src));
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// One periodic fold by a box length (positions are kept in [-L, 2L)).
__device__ __forceinline__ double fold_box(double x, double L)
{
    if (x < 0.0) return x + L;
    if (x >= L) return x - L;
    return x;
}

__device__ __forceinline__ int fold_index(int i, int M)
{
    if (i < 0) return i + M;
    if (i >= M) return i - M;
    return i;
}

// 4-bit sub-cell coordinates interleaved into a 12-bit Morton code (z-order
// of the 16^3 sub-cells of a PP cell).
__device__ __forceinline__ int morton12(int x, int y, int z)
{
    auto spread = [](int b) { return (b & 1) | ((b & 2) << 2) | ((b & 4) << 4) | ((b & 8) << 6); };
    return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}

// PP cell and mesh brick of a particle (see p3m_sort.cu). Raises ST_BOX and
// files the particle under cell 0 when it is outside [-L, 2L) or not finite.
// cell == nullptr skips the cell key; sub (may be NULL) receives the Morton
// code of the particle's sub-cell within its cell.
__device__ __forceinline__ void particle_keys(const RepDev &R, double x, double y, double z,
                                              int has_mesh, int *cell, int *brick, int *status,
                                              int *sub = nullptr)
{
    const double L = R.L;
    const bool ok = (x >= -L && x < 2.0 * L) && (y >= -L && y < 2.0 * L) && (z >= -L && z < 2.0 * L);
    if (!ok) {
        raise_status(status, ST_BOX);
        x = y = z = 0.0;
    }
    if (cell) {
        const double xw = fold_box(x, L), yw = fold_box(y, L), zw = fold_box(z, L);
        const int cx = min((int)floor(xw / R.cellw), R.nc - 1);
        const int cy = min((int)floor(yw / R.cellw), R.nc - 1);
        const int cz = min((int)floor(zw / R.cellw), R.nc - 1);
        *cell = R.cell_off + cx + R.nc * (cy + R.nc * cz);
        if (sub) {
            auto q4 = [](double t, int c) { return max(0, min(15, (int)((t - c) * 16.0))); };
            *sub = morton12(q4(xw / R.cellw, cx), q4(yw / R.cellw, cy), q4(zw / R.cellw, cz));
        }
    }
    *brick = -1;
    if (has_mesh && R.M > 0) {
        const int ix = fold_index((int)floor(x / R.h), R.M);
        const int iy = fold_index((int)floor(y / R.h), R.M);
        const int iz = fold_index((int)floor(z / R.h), R.M);
        *brick = R.brick_off + ix / BRICK + R.nb * (iy / BRICK + R.nb * (iz / BRICK));
    }
}

}  // namespace p3m
