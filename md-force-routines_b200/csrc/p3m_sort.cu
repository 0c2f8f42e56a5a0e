// Particle keys and counting sorts (PP cells and mesh bricks).
//
// The PP cell of a particle is floor(x / (L/floor(L/rc))) per axis, the same
// cell grid as yukawa_pp.py:17-28 and :44-52; positions are first folded by
// one box length into [0, L) (a particle at exactly x = L lands in cell 0,
// where the reference would index past its grid). The mesh brick is the
// BRICK^3 block of base indices floor(x/h) (yukawa_pm_ord6.py:17-27), folded
// into [0, M).
//
// The cell sort (the grid of the neighbour-list build, cells >= rc + skin)
// runs only on rebuild steps, per replica: each replica has its own rebuild
// flag, its cells are scanned within its own particle range, and the cell
// kernels skip the work of replicas whose flag is clear -- so a replica's
// lists, and its rounding, do not depend on the other replicas of a batch. It is deterministic: counts and offsets
// come from integer atomics and a scan; the order inside a cell is then
// fixed by sorting each cell's particle indices ascending (rank sort), so
// every rerun builds the same lists. The brick sort runs every step; each
// brick's particles are then put in ascending index order the same way, so
// the assignment adds them in a fixed order.
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

// Cell keys of a rebuild step (the drift kernel computed the brick keys).
__global__ void k_cell_keys(const RepDev *__restrict__ reps, const int *__restrict__ prep,
                            const double *__restrict__ pos, int ntot, int *__restrict__ cell_key,
                            int *__restrict__ cell_count, const int *__restrict__ rebuild,
                            int *status)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        const int r = prep[i];
        if (!rebuild[r]) continue;
        const RepDev &R = reps[r];
        int c, b;
        particle_keys(R, pos[3 * i + 0], pos[3 * i + 1], pos[3 * i + 2], 0, &c, &b, status);
        cell_key[i] = c;
        atomicAdd(&cell_count[c], 1);
    }
}

// Exclusive scan of count[0..n) into start[0..n], offset by `base` (single
// block), zeroing the counts and the scatter cursors for the next use.
__device__ void block_scan_array(int *count, int *start, int *cursor, int n, int base, int *sm)
{
    int carry = base;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
    for (int b0 = 0; b0 < n; b0 += blockDim.x) {
        int i = b0 + tid;
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

// Block 0: the cells of every replica whose rebuild flag is set, each within
// its own particle range [p_off, p_off + n). Block 1: all bricks.
__global__ void k_scan(const RepDev *__restrict__ reps, int nrep, int *cell_count,
                       int *cell_start, int *cell_cursor, int *brick_count, int *brick_start,
                       int *brick_cursor, int nbrick, const int *__restrict__ rebuild)
{
    __shared__ int sm[64];
    if (blockIdx.x == 0) {
        for (int r = 0; r < nrep; ++r) {
            if (!rebuild[r]) continue;
            const RepDev &R = reps[r];
            const int c0 = R.cell_off, nc = R.nc * R.nc * R.nc;
            block_scan_array(cell_count + c0, cell_start + c0, cell_cursor + c0, nc, R.p_off, sm);
            __syncthreads();
        }
    } else if (nbrick > 0) {
        block_scan_array(brick_count, brick_start, brick_cursor, nbrick, 0, sm);
    }
}

__global__ void k_scatter(const int *__restrict__ cell_key, const int *__restrict__ cell_start,
                          int *cell_cursor, int *__restrict__ cell_tmp,
                          const int *__restrict__ brick_key, const int *__restrict__ brick_start,
                          int *brick_cursor, int *__restrict__ brick_tmp,
                          int ntot, int has_mesh,
                          const int *__restrict__ prep, const int *__restrict__ rebuild)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        if (rebuild[prep[i]]) {
            int c = cell_key[i];
            cell_tmp[cell_start[c] + atomicAdd(&cell_cursor[c], 1)] = i;
        }
        if (has_mesh) {
            int b = brick_key[i];
            brick_tmp[brick_start[b] + atomicAdd(&brick_cursor[b], 1)] = i;
        }
    }
}

// One warp per cell: order the cell's particles by index, and remember every
// particle's position at this rebuild (the reference point of the skin check).
__global__ void k_fix_cells(const RepDev *__restrict__ reps, int nrep,
                            const int *__restrict__ cell_start, const int *__restrict__ cell_tmp,
                            const double *__restrict__ pos, int *__restrict__ cell_perm,
                            int *__restrict__ cell_slot, double *__restrict__ pos_ref, int ncell,
                            const int *__restrict__ rebuild)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int c = blockIdx.x * wpb + (threadIdx.x >> 5); c < ncell; c += gridDim.x * wpb) {
        if (!rebuild[find_rep(c, nrep, [&](int k) { return reps[k].cell_off; })]) continue;
        const int start = cell_start[c], n = cell_start[c + 1] - start;
        for (int e0 = 0; e0 < n; e0 += 32) {
            int e = e0 + lane;
            int v = (e < n) ? cell_tmp[start + e] : 0x7fffffff;
            int rank = 0;
            for (int f = 0; f < n; ++f) rank += (cell_tmp[start + f] < v) ? 1 : 0;
            if (e < n) {
                int s = start + rank;
                cell_perm[s] = v;
                cell_slot[v] = s;
                pos_ref[3 * v + 0] = pos[3 * v + 0];
                pos_ref[3 * v + 1] = pos[3 * v + 1];
                pos_ref[3 * v + 2] = pos[3 * v + 2];
            }
        }
    }
}

// One warp per brick: order the brick's particles by index.
__global__ void k_fix_bricks(const int *__restrict__ brick_start, const int *__restrict__ brick_tmp,
                             int *__restrict__ brick_perm, int *__restrict__ brick_slot, int nbrick)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int b = blockIdx.x * wpb + (threadIdx.x >> 5); b < nbrick; b += gridDim.x * wpb) {
        const int start = brick_start[b], n = brick_start[b + 1] - start;
        for (int e0 = 0; e0 < n; e0 += 32) {
            const int e = e0 + lane;
            const int v = (e < n) ? brick_tmp[start + e] : 0x7fffffff;
            int rank = 0;
            for (int f = 0; f < n; ++f) rank += (brick_tmp[start + f] < v) ? 1 : 0;
            if (e < n) {
                brick_perm[start + rank] = v;
                brick_slot[v] = start + rank;
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

void launch_cell_keys(const DevState &s, cudaStream_t st)
{
    k_cell_keys<<<grid_for(s.ntot, 256), 256, 0, st>>>(s.reps, s.prep, s.pos, s.ntot, s.cell_key,
                                                       s.cell_count, s.rebuild, s.status);
}

void launch_scan(const DevState &s, cudaStream_t st)
{
    k_scan<<<2, 1024, 0, st>>>(s.reps, s.nrep, s.cell_count, s.cell_start, s.cell_cursor,
                               s.brick_count, s.brick_start, s.brick_cursor,
                               s.has_mesh ? s.nbrick : 0, s.rebuild);
}

void launch_scatter(const DevState &s, cudaStream_t st)
{
    k_scatter<<<grid_for(s.ntot, 256), 256, 0, st>>>(s.cell_key, s.cell_start, s.cell_cursor,
                                                      s.cell_tmp, s.brick_key, s.brick_start,
                                                      s.brick_cursor, s.brick_tmp, s.ntot,
                                                      s.has_mesh, s.prep, s.rebuild);
}

void launch_fix_bricks(const DevState &s, cudaStream_t st)
{
    const int wpb = 8;
    k_fix_bricks<<<(s.nbrick + wpb - 1) / wpb, wpb * 32, 0, st>>>(s.brick_start, s.brick_tmp,
                                                                 s.brick_perm, s.brick_slot,
                                                                 s.nbrick);
}

template <typename T> void launch_fix_cells(const DevState &s, cudaStream_t st)
{
    const int wpb = 8;
    int blocks = (s.ncell + wpb - 1) / wpb;
    k_fix_cells<<<blocks, wpb * 32, 0, st>>>(s.reps, s.nrep, s.cell_start, s.cell_tmp, s.pos,
                                             s.cell_perm, s.cell_slot, s.pos_ref, s.ncell,
                                             s.rebuild);
}

template void launch_keys<float>(const DevState &, cudaStream_t);
template void launch_keys<double>(const DevState &, cudaStream_t);
template void launch_fix_cells<float>(const DevState &, cudaStream_t);
template void launch_fix_cells<double>(const DevState &, cudaStream_t);

}  // namespace p3m
