// Particle keys and counting sorts (PP cells and mesh bricks).
//
// The PP cell of a particle is floor(x / (L/floor(L/rc))) per axis, the same
// cell grid as yukawa_pp.py:17-28 and :44-52; positions are first folded by
// one box length into [0, L) (a particle at exactly x = L lands in cell 0,
// where the reference would index past its grid). The mesh brick is the
// BRICK^3 block of base indices floor(x/h) (yukawa_pm_ord6.py:17-27), folded
// into [0, M).
//
// The cell sort (the grid of the neighbour-list build, cells >= (rc + skin)/2)
// runs only on rebuild steps, per replica: each replica has its own rebuild
// flag, its cells are scanned within its own particle range, and the cell
// kernels skip the work of replicas whose flag is clear -- so a replica's
// lists, and its rounding, do not depend on the other replicas of a batch. It is deterministic: counts and offsets
// come from integer atomics and a scan; the order inside a cell is then
// fixed by sorting each cell's particle indices ascending (rank sort), so
// every rerun builds the same lists. The brick sort runs every step and puts
// each brick's particles in ascending index order, so the assignment adds
// them in a fixed order: a stable counting sort over chunks of `ch`
// consecutive particles of one replica (ch sized at context creation so that
// there are a few chunks per SM) (per-chunk counts per brick, a scan of
// each brick's counts over the chunks, then one warp per chunk placing its
// particles in index order). Its work is linear in the particle count however
// many particles share a brick.
#include "p3m_kernels.h"

namespace p3m {

template <typename T>
__global__ void k_keys(const RepDev *__restrict__ reps, const int *__restrict__ prep,
                       const double *__restrict__ pos, int ntot, int *__restrict__ cell_key,
                       int *__restrict__ cell_sub, int *__restrict__ cell_count,
                       int *__restrict__ brick_key, int *__restrict__ brick_count, int has_mesh,
                       int *status)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        const RepDev &R = reps[prep[i]];
        int c, b, sub;
        particle_keys(R, pos[3 * i + 0], pos[3 * i + 1], pos[3 * i + 2], has_mesh, &c, &b, status,
                      &sub);
        cell_key[i] = c;
        cell_sub[i] = sub;
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
                            int *__restrict__ cell_sub, int *__restrict__ cell_count,
                            const int *__restrict__ rebuild, int *status)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        const int r = prep[i];
        if (!rebuild[r]) continue;
        const RepDev &R = reps[r];
        int c, b, sub;
        particle_keys(R, pos[3 * i + 0], pos[3 * i + 1], pos[3 * i + 2], 0, &c, &b, status, &sub);
        cell_key[i] = c;
        cell_sub[i] = sub;
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
                       int *brick_cursor, int nbrick, const int *__restrict__ rebuild,
                       int *__restrict__ rb_list, int first_part)
{
    __shared__ int sm[64];
    if (blockIdx.x + first_part == 0) {
        int k = 0, cells = 0;
        for (int r = 0; r < nrep; ++r) {
            if (!rebuild[r]) continue;
            const RepDev &R = reps[r];
            const int c0 = R.cell_off, nc = R.nc * R.nc * R.nc;
            block_scan_array(cell_count + c0, cell_start + c0, cell_cursor + c0, nc, R.p_off, sm);
            if (threadIdx.x == 0) {
                rb_list[1 + k] = r;
                rb_list[nrep + 1 + k] = cells;
            }
            ++k;
            cells += nc;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            rb_list[0] = k;
            rb_list[nrep + 1 + k] = cells;
        }
    } else if (nbrick > 0) {
        block_scan_array(brick_count, brick_start, brick_cursor, nbrick, 0, sm);
    }
}

__global__ void k_scatter(const int *__restrict__ cell_key, const int *__restrict__ cell_start,
                          int *cell_cursor, int *__restrict__ cell_tmp, int ntot,
                          const int *__restrict__ prep, const int *__restrict__ rebuild)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        if (rebuild[prep[i]]) {
            int c = cell_key[i];
            cell_tmp[cell_start[c] + atomicAdd(&cell_cursor[c], 1)] = i;
        }
    }
}

// One warp per cell: order the cell's particles by (sub-cell Morton code,
// index) -- z-order inside the cell, so the particles of one warp of the PP
// kernel are neighbours in space and walk their (similar) lists in step,
// reading nearby coordinates -- and remember every particle's position at
// this rebuild (the reference point of the skin check).
__global__ void k_fix_cells(const RepDev *__restrict__ reps, int nrep,
                            const int *__restrict__ cell_start, const int *__restrict__ cell_tmp,
                            const int *__restrict__ cell_sub, const double *__restrict__ pos,
                            int *__restrict__ cell_perm, int *__restrict__ cell_slot,
                            double *__restrict__ pos_ref, int ncell,
                            const int *__restrict__ rebuild)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    auto key = [&](int i) { return ((unsigned long long)cell_sub[i] << 32) | (unsigned)i; };
    for (int c = blockIdx.x * wpb + (threadIdx.x >> 5); c < ncell; c += gridDim.x * wpb) {
        if (!rebuild[find_rep(c, nrep, [&](int k) { return reps[k].cell_off; })]) continue;
        const int start = cell_start[c], n = cell_start[c + 1] - start;
        for (int e0 = 0; e0 < n; e0 += 32) {
            int e = e0 + lane;
            int v = (e < n) ? cell_tmp[start + e] : 0;
            const unsigned long long kv = (e < n) ? key(v) : ~0ull;
            // rank = keys below kv: 32 keys loaded per pass, compared by shuffle
            int rank = 0;
            for (int f0 = 0; f0 < n; f0 += 32) {
                const int f = f0 + lane;
                const unsigned long long kf = (f < n) ? key(cell_tmp[start + f]) : ~0ull;
                const int m = min(32, n - f0);
                for (int t = 0; t < m; ++t)
                    rank += (__shfl_sync(0xffffffffu, kf, t) < kv) ? 1 : 0;
            }
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

// ---- brick sort ----------------------------------------------------------

__device__ __forceinline__ int sort_chunks(const RepDev &R, int ch) { return (R.n + ch - 1) / ch; }

// One block per chunk: hist[chunk][k] = particles of the chunk in the
// replica's brick k (shared-memory integer counts).
__global__ void __launch_bounds__(256)
k_brick_hist(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ brick_key,
             int *__restrict__ hist, int nchunk, int ch)
{
    extern __shared__ int hcount[];
    for (int c = blockIdx.x; c < nchunk; c += gridDim.x) {
        const RepDev &R = reps[find_rep(c, nrep, [&](int k) { return reps[k].sc_off; })];
        const int nbr = R.nb * R.nb * R.nb;
        const int cl = c - R.sc_off;
        const int p0 = R.p_off + cl * ch, n = min(ch, R.n - cl * ch);
        for (int k = threadIdx.x; k < nbr; k += blockDim.x) hcount[k] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            atomicAdd(&hcount[brick_key[p0 + i] - R.brick_off], 1);
        __syncthreads();
        int *row = hist + R.sh_off + (long long)cl * nbr;
        for (int k = threadIdx.x; k < nbr; k += blockDim.x) row[k] = hcount[k];
        __syncthreads();
    }
}

// One warp per brick: its counts over the replica's chunks become the
// chunks' first slots (exclusive scan from brick_start), 32 chunks a pass.
__global__ void k_brick_colscan(const RepDev *__restrict__ reps, int nrep,
                                const int *__restrict__ brick_start, int *__restrict__ hist,
                                int nbrick, int ch)
{
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int b = blockIdx.x * wpb + (threadIdx.x >> 5); b < nbrick; b += gridDim.x * wpb) {
        const RepDev &R = reps[find_rep(b, nrep, [&](int k) { return reps[k].brick_off; })];
        const int nbr = R.nb * R.nb * R.nb;
        const int nch = sort_chunks(R, ch);
        int *col = hist + R.sh_off + (b - R.brick_off);
        int carry = brick_start[b];
        for (int c0 = 0; c0 < nch; c0 += 32) {
            const int cl = c0 + lane;
            const int t = cl < nch ? col[(long long)cl * nbr] : 0;
            int x = t;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (cl < nch) col[(long long)cl * nbr] = carry + x - t;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
    }
}

// One warp per chunk, 32 particles at a time in index order: lanes with the
// same brick take consecutive slots in lane order (__match_any_sync), then
// the group's last lane advances the brick's next slot.
__global__ void __launch_bounds__(32)
k_brick_place(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ brick_key,
              const int *__restrict__ hist, int *__restrict__ brick_perm,
              int *__restrict__ brick_slot, int nchunk, int ch)
{
    extern __shared__ int next_slot[];
    const int lane = threadIdx.x;
    for (int c = blockIdx.x; c < nchunk; c += gridDim.x) {
        const RepDev &R = reps[find_rep(c, nrep, [&](int k) { return reps[k].sc_off; })];
        const int nbr = R.nb * R.nb * R.nb;
        const int cl = c - R.sc_off;
        const int p0 = R.p_off + cl * ch, n = min(ch, R.n - cl * ch);
        const int *row = hist + R.sh_off + (long long)cl * nbr;
        for (int k = lane; k < nbr; k += 32) next_slot[k] = row[k];
        __syncwarp();
        for (int e0 = 0; e0 < n; e0 += 32) {
            const int e = e0 + lane;
            const bool valid = e < n;
            const int key = valid ? brick_key[p0 + e] - R.brick_off : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            if (valid) {
                const int slot = next_slot[key] + __popc(peers & ((1u << lane) - 1u));
                brick_perm[slot] = p0 + e;
                brick_slot[p0 + e] = slot;
            }
            __syncwarp();
            if (valid && lane == 31 - __clz(peers)) next_slot[key] += __popc(peers);
            __syncwarp();
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
                                                      s.cell_sub, s.cell_count, s.brick_key,
                                                      s.brick_count, s.has_mesh, s.status);
}

void launch_cell_keys(const DevState &s, cudaStream_t st)
{
    k_cell_keys<<<grid_for(s.ntot, 256), 256, 0, st>>>(s.reps, s.prep, s.pos, s.ntot, s.cell_key,
                                                       s.cell_sub, s.cell_count, s.rebuild,
                                                       s.status);
}

// Both scans (block 0: the cells of the rebuilding replicas, block 1: the
// bricks), or one of them: part 0 / 1.
void launch_scan(const DevState &s, cudaStream_t st, int part)
{
    const int first = part == 1 ? 1 : 0, nblocks = part < 0 ? 2 : 1;
    k_scan<<<nblocks, 1024, 0, st>>>(s.reps, s.nrep, s.cell_count, s.cell_start, s.cell_cursor,
                                     s.brick_count, s.brick_start, s.brick_cursor,
                                     s.has_mesh ? s.nbrick : 0, s.rebuild, s.rb_list, first);
}

void launch_scatter(const DevState &s, cudaStream_t st)
{
    k_scatter<<<grid_for(s.ntot, 256), 256, 0, st>>>(s.cell_key, s.cell_start, s.cell_cursor,
                                                      s.cell_tmp, s.ntot, s.prep, s.rebuild);
}

void launch_sort_bricks(const DevState &s, cudaStream_t st)
{
    const size_t smem = (size_t)s.max_bricks * sizeof(int);
    k_brick_hist<<<grid_for(s.nchunk, 1), 256, smem, st>>>(s.reps, s.nrep, s.brick_key,
                                                            s.brick_hist, s.nchunk, s.sort_ch);
    k_brick_colscan<<<grid_for(s.nbrick, 8), 256, 0, st>>>(s.reps, s.nrep, s.brick_start,
                                                              s.brick_hist, s.nbrick, s.sort_ch);
    k_brick_place<<<grid_for(s.nchunk, 1), 32, smem, st>>>(s.reps, s.nrep, s.brick_key,
                                                           s.brick_hist, s.brick_perm,
                                                           s.brick_slot, s.nchunk, s.sort_ch);
}

template <typename T> void launch_fix_cells(const DevState &s, cudaStream_t st)
{
    const int wpb = 8;
    int blocks = (s.ncell + wpb - 1) / wpb;
    k_fix_cells<<<blocks, wpb * 32, 0, st>>>(s.reps, s.nrep, s.cell_start, s.cell_tmp, s.cell_sub,
                                             s.pos, s.cell_perm, s.cell_slot, s.pos_ref, s.ncell,
                                             s.rebuild);
}

template void launch_keys<float>(const DevState &, cudaStream_t);
template void launch_keys<double>(const DevState &, cudaStream_t);
template void launch_fix_cells<float>(const DevState &, cudaStream_t);
template void launch_fix_cells<double>(const DevState &, cudaStream_t);

}  // namespace p3m
