// Particle keys and counting sorts (PP cells and mesh bricks).
//
// The PP cell of a particle is floor(x / (L/floor(L/rc))) per axis, the same
// cell grid as yukawa_pp.py:17-28 and :44-52; positions are first folded by
// one box length into [0, L) (a particle at exactly x = L lands in cell 0,
// where the reference would index past its grid). The mesh brick is the
// BRICK^3 block of base indices floor(x/h) (yukawa_pm_ord6.py:17-27), folded
// into [0, M).
//
// The cell sort is deterministic: counts and offsets come from integer
// atomics and a scan; the order inside a cell is then fixed by sorting each
// cell's particle indices ascending (rank sort), so every rerun stages
// neighbours in the same order and sums forces in the same order. The brick
// sort keeps the atomic order because the assignment accumulates in integer
// fixed point (order-independent) and the gather has no cross-particle sums.
#include "p3m_kernels.h"

namespace p3m {

template <typename T>
__global__ void k_keys(const RepDev *__restrict__ reps, const int *__restrict__ prep,
                       const double *__restrict__ pos, int ntot, int *__restrict__ cell_key,
                       int *__restrict__ cell_count, int *__restrict__ brick_key,
                       int *__restrict__ brick_count, int has_mesh, int *status)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        const RepDev &R = reps[prep[i]];
        int c, b;
        particle_keys(R, pos[3 * i + 0], pos[3 * i + 1], pos[3 * i + 2], has_mesh, &c, &b, status);
        cell_key[i] = c;
        atomicAdd(&cell_count[c], 1);
        if (b >= 0) {
            brick_key[i] = b;
            atomicAdd(&brick_count[b], 1);
        }
    }
}

// Exclusive scan of one count array into start[0..n] (single block), zeroing
// the counts and the scatter cursors for the next use.
__device__ void block_scan_array(int *count, int *start, int *cursor, int n, int *sm)
{
    int carry = 0;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + tid;
        int v = (i < n) ? count[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane == 31) sm[w] = x;
        __syncthreads();
        if (w == 0) {
            int s = (lane < nw) ? sm[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += t;
            }
            sm[32 + lane] = s;  // inclusive warp totals
        }
        __syncthreads();
        int excl = carry + x - v + (w > 0 ? sm[32 + w - 1] : 0);
        if (i < n) {
            start[i] = excl;
            count[i] = 0;
            cursor[i] = 0;
        }
        carry += sm[32 + nw - 1];
        __syncthreads();
    }
    if (tid == 0) start[n] = carry;
}

__global__ void k_scan(int *cell_count, int *cell_start, int *cell_cursor, int ncell,
                       int *brick_count, int *brick_start, int *brick_cursor, int nbrick)
{
    __shared__ int sm[64];
    if (blockIdx.x == 0)
        block_scan_array(cell_count, cell_start, cell_cursor, ncell, sm);
    else if (nbrick > 0)
        block_scan_array(brick_count, brick_start, brick_cursor, nbrick, sm);
}

__global__ void k_scatter(const int *__restrict__ cell_key, const int *__restrict__ cell_start,
                          int *cell_cursor, int *__restrict__ cell_tmp,
                          const int *__restrict__ brick_key, const int *__restrict__ brick_start,
                          int *brick_cursor, int *__restrict__ brick_perm,
                          int *__restrict__ brick_slot, int ntot, int has_mesh)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        int c = cell_key[i];
        cell_tmp[cell_start[c] + atomicAdd(&cell_cursor[c], 1)] = i;
        if (has_mesh) {
            int b = brick_key[i];
            int s = brick_start[b] + atomicAdd(&brick_cursor[b], 1);
            brick_perm[s] = i;
            brick_slot[i] = s;
        }
    }
}

// One warp per cell: order the cell's particles by index and write their
// positions relative to the cell origin (FP64) in that order.
__global__ void k_fix_cells(const RepDev *__restrict__ reps, int nrep,
                            const int *__restrict__ cell_start, const int *__restrict__ cell_tmp,
                            const double *__restrict__ pos, int *__restrict__ cell_perm,
                            int *__restrict__ cell_slot, double4 *__restrict__ xs, int ncell)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int c = blockIdx.x * wpb + (threadIdx.x >> 5); c < ncell; c += gridDim.x * wpb) {
        const int r = find_rep(c, nrep, [&](int k) { return reps[k].cell_off; });
        const RepDev &R = reps[r];
        const int start = cell_start[c], n = cell_start[c + 1] - start;
        const int local = c - R.cell_off;
        const int cx = local % R.nc, cy = (local / R.nc) % R.nc, cz = local / (R.nc * R.nc);
        for (int e0 = 0; e0 < n; e0 += 32) {
            int e = e0 + lane;
            int v = (e < n) ? cell_tmp[start + e] : 0x7fffffff;
            int rank = 0;
            for (int f = 0; f < n; ++f) rank += (cell_tmp[start + f] < v) ? 1 : 0;
            if (e < n) {
                int s = start + rank;
                cell_perm[s] = v;
                cell_slot[v] = s;
                double x = fold_box(pos[3 * v + 0], R.L);
                double y = fold_box(pos[3 * v + 1], R.L);
                double z = fold_box(pos[3 * v + 2], R.L);
                xs[s] = make_double4(x - cx * R.cellw, y - cy * R.cellw, z - cz * R.cellw, 0.0);
            }
        }
    }
}

static int grid_for(int n, int threads, int cap = 148 * 16)
{
    int g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    return g < cap ? g : cap;
}

template <typename T> void launch_keys(const DevState &s, cudaStream_t st)
{
    k_keys<T><<<grid_for(s.ntot, 256), 256, 0, st>>>(s.reps, s.prep, s.pos, s.ntot, s.cell_key,
                                                      s.cell_count, s.brick_key, s.brick_count,
                                                      s.has_mesh, s.status);
}

void launch_scan(const DevState &s, cudaStream_t st)
{
    k_scan<<<2, 1024, 0, st>>>(s.cell_count, s.cell_start, s.cell_cursor, s.ncell,
                               s.brick_count, s.brick_start, s.brick_cursor,
                               s.has_mesh ? s.nbrick : 0);
}

void launch_scatter(const DevState &s, cudaStream_t st)
{
    k_scatter<<<grid_for(s.ntot, 256), 256, 0, st>>>(s.cell_key, s.cell_start, s.cell_cursor,
                                                      s.cell_tmp, s.brick_key, s.brick_start,
                                                      s.brick_cursor, s.brick_perm,
                                                      s.brick_slot, s.ntot, s.has_mesh);
}

template <typename T> void launch_fix_cells(const DevState &s, cudaStream_t st)
{
    const int wpb = 8;
    int blocks = (s.ncell + wpb - 1) / wpb;
    k_fix_cells<<<blocks, wpb * 32, 0, st>>>(s.reps, s.nrep, s.cell_start, s.cell_tmp, s.pos,
                                             s.cell_perm, s.cell_slot, (double4 *)s.xs_cell,
                                             s.ncell);
}

template void launch_keys<float>(const DevState &, cudaStream_t);
template void launch_keys<double>(const DevState &, cudaStream_t);
template void launch_fix_cells<float>(const DevState &, cudaStream_t);
template void launch_fix_cells<double>(const DevState &, cudaStream_t);

}  // namespace p3m
