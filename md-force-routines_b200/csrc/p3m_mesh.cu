// Particle-mesh (PM) stages: order-6 charge assignment, 3-D FFT of the
// charge mesh, the influence-function multiply with ik differentiation, three
// inverse FFTs of the field components and the order-6 force gather.
//
// This computes what yukawa_pm_ord6.py:440-484 computes:
//   rho   = charge_assgn_6(pos)                       (:445, :6-95)
//   rho_k = fftshift(fftn(rho)); phi_k = G_k rho_k     (:447-451)
//   U_f   = 1/2 sum |rho_k|^2 G_k / V                  (:453-457)
//   E     = (M^3/V) real(ifftn(ifftshift(-i k phi_k))) (:459-480)
//   acc   = Z field_assgn_6(E, pos)                    (:482, :213-312)
// on half spectra (R2C / C2R). Two facts make that equal to the reference's
// full complex transforms: the real part of ifftn equals the C2R transform of
// the Hermitian part of the spectrum, and the -i k_a multiplier of field
// component a is anti-Hermitian on a's own Nyquist plane, where the
// reference's real() therefore cancels it -- so it is zeroed there. U_f sums
// the half spectrum with weight 2 off the kx = 0 and kx = M/2 planes.
//
// Layouts (per replica, concatenated over replicas):
//   tiles   T     [brick][TILE^3]   partial charge of each brick's particles
//   spec    C2<T> [kx][z][y]        kx in [0, M/2], y fastest
//   ek      C2<T> [3][kx][z][y]     field spectra
//   green   T     [kx][z][y]        G_k / V in the same layout
//   efield  T     [3][z][y][x]      real field meshes, x fastest
//
// Assignment is deterministic: each CTA owns one brick of BRICK^3 base
// cells and adds its particles' 216-node stencils into a shared-memory tile
// of TILE^3 nodes, in FP64 in a fixed particle order without atomics
// (k_assign), or in FP32 with order-independent integer atomics
// (k_assign_i32).
// Overlapping tile halos are summed in a fixed order when the first FFT pass
// reads the mesh.
//
// The FFT is an in-place radix-2 decimation-in-time transform of lines held
// in shared memory (padded strides), with up to three stages per register
// pass, the input permuted to bit-reversed order as it is loaded. Twiddles
// exp(-2 pi i k/256) come from an FP64-accurate table.
#include "p3m_kernels.h"

namespace p3m {

constexpr int FFT_THREADS = 256;  // a multiple of the largest mesh side (256)
constexpr int LS = PENCIL + 1;  // padded line stride of the shared tiles
constexpr int LSX = XL_MAX + 1;  // the same for the x passes

template <typename T> using cplx = typename C2<T>::t;

__device__ __forceinline__ int brev(int n, int logM) { return (int)(__brev((unsigned)n) >> (32 - logM)); }

// signed frequency of index n on an M-point axis
__device__ __forceinline__ int freq(int n, int M) { return n < (M >> 1) ? n : n - M; }

template <typename T>
__device__ __forceinline__ void load_twiddles(cplx<T> *tw, const cplx<T> *g)
{
    for (int k = threadIdx.x; k < 128; k += blockDim.x) tw[k] = g[k];
}

// In-place radix-2 decimation-in-time FFT of `nlines` lines of length 2^logM
// held in shared memory, element n of line l at buf[l * ls + n * es]; input
// in bit-reversed order, output natural; unnormalised, the inverse uses
// conjugate twiddles; nlines = 2^lognl. Up to three consecutive radix-2 stages are done in
// registers on groups of 8 (4, 2) elements, so the data passes through shared
// memory -- and the block through a barrier -- once per three stages. Thread
// b takes line b mod nlines, so consecutive threads touch consecutive lines.
// Ends with a barrier.
template <typename T, int LOGR>
__device__ __forceinline__ void fft_group_pass(cplx<T> *buf, int logM, int ls, int es, int lognl,
                                               const cplx<T> *tw, bool inverse, int s)
{
    constexpr int R = 1 << LOGR;
    const int half = 1 << s;           // distance of the first stage's pairs
    const int ngroups = 1 << (lognl + logM - LOGR);
    for (int b = threadIdx.x; b < ngroups; b += blockDim.x) {
        const int l = b & ((1 << lognl) - 1), g = b >> lognl;
        const int k = g & (half - 1), blk = g >> s;
        const int base = (blk << (s + LOGR)) + k;
        cplx<T> x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = buf[l * ls + (base + r * half) * es];
#pragma unroll
        for (int t = 0; t < LOGR; ++t) {
            // stage s + t: pairs (r, r + 2^t); twiddle W_{2^(s+t+1)}^{k + (r mod 2^t) half}
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (r & (1 << t)) continue;
                const int e = k + (r & ((1 << t) - 1)) * half;
                cplx<T> w = tw[e << (7 - (s + t))];
                if (inverse) w.y = -w.y;
                const cplx<T> a = x[r], c = cmul<T>(w, x[r + (1 << t)]);
                x[r] = make_c<T>(a.x + c.x, a.y + c.y);
                x[r + (1 << t)] = make_c<T>(a.x - c.x, a.y - c.y);
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) buf[l * ls + (base + r * half) * es] = x[r];
    }
    __syncthreads();
}

// The first three stages (a pass of fft_group_pass with s = 0): each group is
// an 8-point DFT of elements base + r, r < 8, whose twiddles are the eighth
// roots of unity 1, -i and (+-1 - i)/sqrt 2 (conjugated for the inverse), so
// no table reads and only two real products per non-trivial rotation.
template <typename T>
__device__ __forceinline__ void fft_first_pass8(cplx<T> *buf, int logM, int ls, int es, int lognl,
                                                bool inverse)
{
    const T h = (T)0.70710678118654752440L;  // cos(pi/4), as the twiddle table holds it
    const int ngroups = 1 << (lognl + logM - 3);
    for (int b = threadIdx.x; b < ngroups; b += blockDim.x) {
        const int l = b & ((1 << lognl) - 1), base = (b >> lognl) << 3;
        cplx<T> x[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) x[r] = buf[l * ls + (base + r) * es];
        // stage 0: pairs (r, r+1), twiddle 1
#pragma unroll
        for (int r = 0; r < 8; r += 2) {
            const cplx<T> a = x[r], c = x[r + 1];
            x[r] = make_c<T>(a.x + c.x, a.y + c.y);
            x[r + 1] = make_c<T>(a.x - c.x, a.y - c.y);
        }
        // stage 1: pairs (r, r+2); twiddle 1 for even r, -i (inverse: +i) for odd r
#pragma unroll
        for (int r = 0; r < 8; r += (r & 1) ? 3 : 1) {
            const cplx<T> a = x[r], v = x[r + 2];
            cplx<T> c = v;
            if (r & 1) c = inverse ? make_c<T>(-v.y, v.x) : make_c<T>(v.y, -v.x);
            x[r] = make_c<T>(a.x + c.x, a.y + c.y);
            x[r + 2] = make_c<T>(a.x - c.x, a.y - c.y);
        }
        // stage 2: pairs (r, r+4), twiddle W_8^r (inverse: conjugate)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const cplx<T> a = x[r], v = x[r + 4];
            cplx<T> c;
            if (r == 0) {
                c = v;
            } else if (r == 2) {
                c = inverse ? make_c<T>(-v.y, v.x) : make_c<T>(v.y, -v.x);
            } else if (r == 1) {  // (1 - i)/sqrt 2, inverse (1 + i)/sqrt 2
                c = inverse ? make_c<T>(h * (v.x - v.y), h * (v.x + v.y))
                            : make_c<T>(h * (v.x + v.y), h * (v.y - v.x));
            } else {              // (-1 - i)/sqrt 2, inverse (-1 + i)/sqrt 2
                c = inverse ? make_c<T>(-h * (v.x + v.y), h * (v.x - v.y))
                            : make_c<T>(h * (v.y - v.x), -h * (v.x + v.y));
            }
            x[r] = make_c<T>(a.x + c.x, a.y + c.y);
            x[r + 4] = make_c<T>(a.x - c.x, a.y - c.y);
        }
#pragma unroll
        for (int r = 0; r < 8; ++r) buf[l * ls + (base + r) * es] = x[r];
    }
    __syncthreads();
}

// The passes of one line length 2^LOGM from stage S on, unrolled at compile
// time (stage offsets, group counts and twiddle strides become constants).
template <typename T, int LOGM, int S = 0>
__device__ __forceinline__ void fft_lines_t(cplx<T> *buf, int ls, int es, int lognl,
                                            const cplx<T> *tw, bool inverse)
{
    if constexpr (S == 0 && LOGM >= 3) {
        fft_first_pass8<T>(buf, LOGM, ls, es, lognl, inverse);
        fft_lines_t<T, LOGM, 3>(buf, ls, es, lognl, tw, inverse);
    } else if constexpr (S + 3 <= LOGM) {
        fft_group_pass<T, 3>(buf, LOGM, ls, es, lognl, tw, inverse, S);
        fft_lines_t<T, LOGM, S + 3>(buf, ls, es, lognl, tw, inverse);
    } else if constexpr (LOGM - S == 2) {
        fft_group_pass<T, 2>(buf, LOGM, ls, es, lognl, tw, inverse, S);
    } else if constexpr (LOGM - S == 1) {
        fft_group_pass<T, 1>(buf, LOGM, ls, es, lognl, tw, inverse, S);
    }
}

// ---------------------------------------------------------------------------
// Charge assignment
// ---------------------------------------------------------------------------

// Order-6 weights at node offset x (yukawa_pm_ord6.py:29-34).
template <typename T>
__device__ __forceinline__ void weights6(T x, T *w)
{
    T x2 = x * x, x3 = x2 * x, x4 = x3 * x, x5 = x4 * x;
    w[0] = ((T)1 - (T)10 * x + (T)40 * x2 - (T)80 * x3 + (T)80 * x4 - (T)32 * x5) / (T)3840;
    w[1] = ((T)237 - (T)750 * x + (T)840 * x2 - (T)240 * x3 - (T)240 * x4 + (T)160 * x5) / (T)3840;
    w[2] = ((T)841 - (T)770 * x - (T)440 * x2 + (T)560 * x3 + (T)80 * x4 - (T)160 * x5) / (T)1920;
    w[3] = ((T)841 + (T)770 * x - (T)440 * x2 - (T)560 * x3 + (T)80 * x4 + (T)160 * x5) / (T)1920;
    w[4] = ((T)237 + (T)750 * x + (T)840 * x2 + (T)240 * x3 - (T)240 * x4 - (T)160 * x5) / (T)3840;
    w[5] = ((T)1 + (T)10 * x + (T)40 * x2 + (T)80 * x3 + (T)80 * x4 + (T)32 * x5) / (T)3840;
}

// Base index (unwrapped) and offset along one axis (yukawa_pm_ord6.py:17-27).
__device__ __forceinline__ int base_offset(double p, double h, double &off)
{
    int ix = (int)floor(p / h);
    off = (p - (ix + 0.5) * h) / h;
    return ix;
}

__device__ __forceinline__ int wrapM(int i, int M)
{
    i %= M;
    return i < 0 ? i + M : i;
}

// One CTA of A_WARPS warps per brick. The brick's particles come in a fixed
// order (ascending particle index, from the brick sort); their weights are
// computed once per chunk; then warp w adds the stencils of all particles,
// in that order, to the tile planes z = w (mod 6) only -- exactly one of each
// particle's six planes, 36 nodes, spread over the lanes. No two warps
// touch the same node and each warp adds its particles one after another, so
// every node receives its contributions in the same order on every run and
// no atomics are needed.
constexpr int A_WARPS = 6;
constexpr int A_THREADS = 32 * A_WARPS;
constexpr int A_CHUNK = 128;   // particles per weight chunk

template <typename T> struct AssignW {
    T wx[6], wy[6], wz[6];  // wx carries the charge
    int base;               // (lz * TILE + ly) * TILE + lx, or -1
    int lz;
};

template <typename T> constexpr size_t assign_smem()
{
    return (size_t)TILE3 * sizeof(T) + (size_t)A_CHUNK * sizeof(AssignW<T>);
}

template <typename T>
__global__ void __launch_bounds__(A_THREADS)
k_assign(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ brick_start,
         const int *__restrict__ brick_perm, const double *__restrict__ pos,
         const double *__restrict__ charge, T *__restrict__ tiles, int nbrick, int *status)
{
    extern __shared__ __align__(16) unsigned char a_smem[];
    T *tile = reinterpret_cast<T *>(a_smem);
    AssignW<T> *W = reinterpret_cast<AssignW<T> *>(a_smem + (size_t)TILE3 * sizeof(T));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // this lane's nodes (dy, dx) of a particle's plane: node = lane + 32 pass < 36
    const int n0 = lane, n1 = lane + 32;
    const int off0 = (n0 / 6) * TILE + n0 % 6, off1 = (n1 / 6) * TILE + n1 % 6;
    const bool has1 = n1 < 36;
    for (int b = blockIdx.x; b < nbrick; b += gridDim.x) {
        const int r = find_rep(b, nrep, [&](int k) { return reps[k].brick_off; });
        const RepDev &R = reps[r];
        const int nb = R.nb, M = R.M, local = b - R.brick_off;
        const int bx = (local % nb) * BRICK, by = ((local / nb) % nb) * BRICK,
                  bz = (local / (nb * nb)) * BRICK;
        const int p0 = brick_start[b];
        const int n = brick_start[b + 1] - p0;
        __syncthreads();
        for (int k = threadIdx.x; k < TILE3; k += A_THREADS) tile[k] = (T)0;
        for (int c0 = 0; c0 < n; c0 += A_CHUNK) {
            const int cn = min(A_CHUNK, n - c0);
            __syncthreads();
            for (int k = threadIdx.x; k < cn; k += A_THREADS) {
                const int i = brick_perm[p0 + c0 + k];
                double ox, oy, oz;
                const int ix = base_offset(pos[3 * i + 0], R.h, ox);
                const int iy = base_offset(pos[3 * i + 1], R.h, oy);
                const int iz = base_offset(pos[3 * i + 2], R.h, oz);
                const int lx = wrapM(ix, M) - bx, ly = wrapM(iy, M) - by, lz = wrapM(iz, M) - bz;
                AssignW<T> w;
                // a particle outside [-L, 2L) was filed under brick 0 and
                // flagged by the key pass; it must not reach outside the tile
                if ((unsigned)lx < (unsigned)BRICK && (unsigned)ly < (unsigned)BRICK &&
                    (unsigned)lz < (unsigned)BRICK) {
                    weights6<T>((T)ox, w.wx);
                    weights6<T>((T)oy, w.wy);
                    weights6<T>((T)oz, w.wz);
                    const T q = (T)charge[i];
#pragma unroll
                    for (int c = 0; c < 6; ++c) w.wx[c] *= q;
                    w.base = (lz * TILE + ly) * TILE + lx;
                    w.lz = lz;
                } else {
                    w.base = -1;
                    w.lz = 0;
                }
                W[k] = w;
            }
            __syncthreads();
            for (int k = 0; k < cn; ++k) {
                const AssignW<T> &w = W[k];
                if (w.base < 0) continue;  // uniform over the block
                // this warp's plane of the particle: lz <= lz + d < lz + 6
                const int d = ((warp - w.lz) % A_WARPS + A_WARPS) % A_WARPS;
                T *plane = tile + w.base + d * TILE * TILE;
                const T wz = w.wz[d];
                plane[off0] += wz * w.wy[n0 / 6] * w.wx[n0 % 6];
                if (has1) plane[off1] += wz * w.wy[n1 / 6] * w.wx[n1 % 6];
                __syncwarp();
            }
        }
        __syncthreads();
        T *dst = tiles + R.tile_off + (long long)local * TILE3;
        for (int k = threadIdx.x; k < TILE3; k += A_THREADS) dst[k] = tile[k];
    }
}

// FP32 path: one CTA of 256 threads per brick, thread per particle, the 216
// contributions added to a shared tile with 32-bit integer atomics -- integer
// sums do not depend on the order of the adds, so the result is the same on
// every run. Each contribution q w is scaled by S = 2^k, the largest power of
// two with 0.17 n |q|max S <= 2^22 for the brick's n particles (0.17 bounds a
// product of three order-6 weights), so no node sum can exceed 2^22 in
// magnitude. t = q w S is split exactly into an integer part and an fb-bit
// fraction with the 1.5 * 2^23 rounding constant (exact for |t| < 2^22, no
// float <-> int conversions) and the two parts go to two int32 tiles: the node
// value is (hi + lo / 2^fb) / S, resolved to 2^-fb / S. fb = 16, or fewer for
// bricks of more than 2^14 particles, so that the n fractions of a node (each
// at most 2^fb) cannot overflow: n 2^fb <= 2^30.
constexpr int A32_THREADS = 256;
constexpr float kRound = 12582912.0f;  // 1.5 * 2^23
constexpr int kRoundBits = 0x4B400000;

__global__ void __launch_bounds__(A32_THREADS)
k_assign_i32(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ brick_start,
             const int *__restrict__ brick_perm, const double *__restrict__ pos,
             const double *__restrict__ charge, float *__restrict__ tiles, int nbrick)
{
    extern __shared__ __align__(16) int a32_smem[];
    int *thi = a32_smem;
    int *tlo = a32_smem + TILE3;
    __shared__ int a_src[A32_THREADS];  // the chunk's particle slot of each thread, or -1
    __shared__ int a_cnt[32];
    const int lane = threadIdx.x & 31;
    for (int b = blockIdx.x; b < nbrick; b += gridDim.x) {
        const int r = find_rep(b, nrep, [&](int k) { return reps[k].brick_off; });
        const RepDev &R = reps[r];
        const int nb = R.nb, M = R.M, local = b - R.brick_off;
        const int bx = (local % nb) * BRICK, by = ((local / nb) % nb) * BRICK,
                  bz = (local / (nb * nb)) * BRICK;
        const int p0 = brick_start[b], n = brick_start[b + 1] - p0;
        // S = 2^k with 0.17 n qmax S <= 2^22
        const double bound = 0.17 * (double)(n > 0 ? n : 1) * R.qmax;
        const int kexp = (int)floor(22.0 - log2(bound > 1e-300 ? bound : 1e-300));
        const float S = ldexpf(1.0f, max(-100, min(kexp, 100)));
        int nbits = 0;
        while ((1 << nbits) <= n && nbits < 30) ++nbits;  // n < 2^nbits
        const int fb = max(0, min(16, 30 - nbits));
        const float F = ldexpf(1.0f, fb);
        __syncthreads();
        for (int k = threadIdx.x; k < TILE3; k += A32_THREADS) {
            thi[k] = 0;
            tlo[k] = 0;
        }
        __syncthreads();
        for (int c0 = p0; c0 < p0 + n; c0 += A32_THREADS) {
            // The lanes of a warp add at the same offsets from their
            // particles' stencil bases: lanes whose bases share a shared-memory
            // bank conflict on every atomic. The chunk's particles are ranked
            // by bank (from floor(x / h) by multiplication: only the balance
            // depends on it) and dealt round-robin to the warps. Integer sums
            // do not depend on which thread adds what.
            const int nch = min(A32_THREADS, p0 + n - c0);
            int bank = 0, rank = 0;
            if (threadIdx.x < nch) {
                const int i = brick_perm[c0 + threadIdx.x];
                const int qx = wrapM((int)floor(pos[3 * i + 0] * R.inv_h), M) - bx;
                const int qy = wrapM((int)floor(pos[3 * i + 1] * R.inv_h), M) - by;
                const int qz = wrapM((int)floor(pos[3 * i + 2] * R.inv_h), M) - bz;
                bank = (int)((((unsigned)qz * TILE + (unsigned)qy) * TILE + (unsigned)qx) & 31u);
            }
            __syncthreads();  // the previous chunk is done with a_src
            a_src[threadIdx.x] = -1;
            if (threadIdx.x < 32) a_cnt[threadIdx.x] = 0;
            __syncthreads();
            if (threadIdx.x < nch) rank = atomicAdd(&a_cnt[bank], 1);
            __syncthreads();
            if (threadIdx.x < 32) {  // exclusive scan of the bank counts
                const int v = a_cnt[lane];
                int x = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += t;
                }
                a_cnt[lane] = x - v;
            }
            __syncthreads();
            if (threadIdx.x < nch) {
                const int q = a_cnt[bank] + rank, nw = (nch + 31) >> 5;
                a_src[(q % nw) * 32 + q / nw] = c0 + threadIdx.x;
            }
            __syncthreads();
            const int p = a_src[threadIdx.x];
            if (p < 0) continue;
            const int i = brick_perm[p];
            double ox, oy, oz;
            const int ix = base_offset(pos[3 * i + 0], R.h, ox);
            const int iy = base_offset(pos[3 * i + 1], R.h, oy);
            const int iz = base_offset(pos[3 * i + 2], R.h, oz);
            const int lx = wrapM(ix, M) - bx, ly = wrapM(iy, M) - by, lz = wrapM(iz, M) - bz;
            // a particle outside [-L, 2L) was filed under brick 0 and flagged
            if ((unsigned)lx >= (unsigned)BRICK || (unsigned)ly >= (unsigned)BRICK ||
                (unsigned)lz >= (unsigned)BRICK)
                continue;
            float wx[6], wy[6], wz[6];
            weights6<float>((float)ox, wx);
            weights6<float>((float)oy, wy);
            weights6<float>((float)oz, wz);
            const float qs = (float)charge[i] * S;
            const int base = (lz * TILE + ly) * TILE + lx;
#pragma unroll
            for (int g = 0; g < 6; ++g) {
#pragma unroll
                for (int a = 0; a < 6; ++a) {
                    const float qzy = qs * wz[g] * wy[a];
                    const int row = base + (g * TILE + a) * TILE;
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        const float t = qzy * wx[c];
                        const float hb = (t - 0.5f) + kRound;       // floor(t), as a float
                        const int hi = __float_as_int(hb) - kRoundBits;
                        const float frac = t - (hb - kRound);         // in [0, 1], exact
                        const int lo = __float_as_int(frac * F + kRound) - kRoundBits;
                        atomicAdd(thi + row + c, hi);
                        atomicAdd(tlo + row + c, lo);
                    }
                }
            }
        }
        __syncthreads();
        float *dst = tiles + R.tile_off + (long long)local * TILE3;
        const double inv = 1.0 / (double)S;
        const double invF = 1.0 / (double)F;  // exact: F is a power of two
        for (int k = threadIdx.x; k < TILE3; k += A32_THREADS)
            dst[k] = (float)(((double)thi[k] + (double)tlo[k] * invF) * inv);
    }
}

// A node's charge is the sum of the (up to 8) brick tiles that cover it. Along
// each axis node n lies in the tile of brick n / BRICK at offset n mod BRICK
// and, when that offset is below HALO, also in the halo of the previous
// (periodic) brick's tile at offset + BRICK. A tile element's address is a sum
// of one term per axis, so each axis contributes two candidate offsets.
struct AxisOff {
    int a, b;  // offset in the own brick's tile, in the previous brick's halo
    bool two;  // the halo term exists
};

// sb: elements between consecutive bricks along the axis; st: between
// consecutive tile rows along the axis
__device__ __forceinline__ AxisOff axis_off(int n, int nb, int sb, int st)
{
    const int bk = n / BRICK, o = n - bk * BRICK;
    AxisOff r;
    r.a = bk * sb + o * st;
    r.b = (bk == 0 ? nb - 1 : bk - 1) * sb + (o + BRICK) * st;
    r.two = o < HALO;
    return r;
}
__device__ __forceinline__ AxisOff axis_x(int x, int nb) { return axis_off(x, nb, TILE3, 1); }
__device__ __forceinline__ AxisOff axis_y(int y, int nb) { return axis_off(y, nb, nb * TILE3, TILE); }
__device__ __forceinline__ AxisOff axis_z(int z, int nb)
{
    return axis_off(z, nb, nb * nb * TILE3, TILE * TILE);
}

// The sum over the covering tiles in a fixed order (dz, dy, dx), all loads
// independent; t = the replica's tiles.
template <typename T>
__device__ __forceinline__ T rho_sum(const T *__restrict__ t, const AxisOff &X, const AxisOff &Y,
                                     const AxisOff &Z)
{
    const int zy0 = Z.a + Y.a, zy1 = Z.a + Y.b, zy2 = Z.b + Y.a, zy3 = Z.b + Y.b;
    const bool y1 = Y.two, z1 = Z.two;
    const T v0 = __ldg(t + zy0 + X.a);
    const T v1 = X.two ? __ldg(t + zy0 + X.b) : (T)0;
    const T v2 = y1 ? __ldg(t + zy1 + X.a) : (T)0;
    const T v3 = (y1 && X.two) ? __ldg(t + zy1 + X.b) : (T)0;
    const T v4 = z1 ? __ldg(t + zy2 + X.a) : (T)0;
    const T v5 = (z1 && X.two) ? __ldg(t + zy2 + X.b) : (T)0;
    const T v6 = (z1 && y1) ? __ldg(t + zy3 + X.a) : (T)0;
    const T v7 = (z1 && y1 && X.two) ? __ldg(t + zy3 + X.b) : (T)0;
    return ((v0 + v1) + (v2 + v3)) + ((v4 + v5) + (v6 + v7));
}

// Charge on node (x,y,z) of replica R.
template <typename T>
__device__ __forceinline__ T rho_at(const RepDev &R, const T *__restrict__ tiles, int x, int y, int z)
{
    return rho_sum<T>(tiles + R.tile_off, axis_x(x, R.nb), axis_y(y, R.nb), axis_z(z, R.nb));
}

// ---------------------------------------------------------------------------
// FFT passes
// ---------------------------------------------------------------------------

// Pass A: rows of the charge mesh (reduced from the tiles) -> R2C along x,
// written transposed into spec[kx][z][y]. Item = (replica, z, tile of
// 2 x_lines rows); two real rows share one complex line. The item body is
// instantiated per mesh side, so its loop bounds, masks and shifts are
// compile-time constants.
template <typename T, int LOGM>
__device__ __forceinline__ void x_r2c_item(const RepDev &R, int w, const T *__restrict__ tiles,
                                           cplx<T> *__restrict__ spec, cplx<T> *buf,
                                           const cplx<T> *tw)
{
    constexpr int M = 1 << LOGM;
    constexpr int LNL = x_lines_log(LOGM), NROW = 2 << LNL;  // complex lines, real rows
    constexpr int NYT = M >> (LNL + 1), NK = (M >> 1) + 1;
    static_assert(FFT_THREADS % M == 0, "each thread keeps one x");
    const int z = w / NYT, y0 = (w % NYT) * NROW;
    const int x = threadIdx.x & (M - 1);
    const AxisOff ax = axis_x(x, R.nb), az = axis_z(z, R.nb);
    const T *t = tiles + R.tile_off;
    T *dst = reinterpret_cast<T *>(&buf[brev(x, LOGM) * LSX]);
    __syncthreads();
    for (int j = threadIdx.x >> LOGM; j < NROW; j += FFT_THREADS >> LOGM)
        dst[j] = rho_sum<T>(t, ax, axis_y(y0 + j, R.nb), az);  // line j/2, part j%2
    __syncthreads();
    fft_lines_t<T, LOGM>(buf, 1, LSX, LNL, tw, false);
    // split the two real rows: Xa = (Z[k] + conj Z[M-k])/2, Xb = (Z[k] - conj Z[M-k])/2i
    cplx<T> *out = spec + R.spec_off + (long long)z * M + y0;
    for (int e = threadIdx.x; e < NROW * NK; e += FFT_THREADS) {
        const int j = e & (NROW - 1), k = e >> (LNL + 1);
        const int l = j >> 1;
        const cplx<T> Z = buf[k * LSX + l];
        const cplx<T> Zm = buf[((M - k) & (M - 1)) * LSX + l];
        cplx<T> X;
        if ((j & 1) == 0) {
            X.x = (T)0.5 * (Z.x + Zm.x);
            X.y = (T)0.5 * (Z.y - Zm.y);
        } else {
            X.x = (T)0.5 * (Z.y + Zm.y);
            X.y = (T)0.5 * (Zm.x - Z.x);
        }
        out[(long long)k * M * M + j] = X;
    }
}

template <typename T>
__global__ void __launch_bounds__(FFT_THREADS, sizeof(T) == 4 ? 4 : 1)
k_fft_x_r2c(const RepDev *__restrict__ reps, int nrep, const T *__restrict__ tiles,
            cplx<T> *__restrict__ spec, const cplx<T> *__restrict__ twg, int nitems)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *tw = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *buf = tw + 128;
    load_twiddles<T>(tw, twg);
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int r = find_rep(item, nrep, [&](int k) { return reps[k].wa_off; });
        const RepDev &R = reps[r];
        const int w = item - R.wa_off;
        switch (R.logM) {  // block-uniform: one replica per item
        case 5: x_r2c_item<T, 5>(R, w, tiles, spec, buf, tw); break;
        case 6: x_r2c_item<T, 6>(R, w, tiles, spec, buf, tw); break;
        case 7: x_r2c_item<T, 7>(R, w, tiles, spec, buf, tw); break;
        default: x_r2c_item<T, 8>(R, w, tiles, spec, buf, tw); break;
        }
    }
}

// Passes B / D: FFT along y of contiguous lines spec[kx][z][:]. Item =
// (replica, [component,] kx, 16-line z tile). `ncomp` arrays of `stride`
// elements are processed (1 forward, 3 inverse). The item body is
// instantiated per mesh side.
template <typename T, int LOGM>
__device__ __forceinline__ void y_item(const RepDev &R, int w, cplx<T> *__restrict__ data,
                                       long long off, cplx<T> *buf, const cplx<T> *tw,
                                       bool inverse)
{
    constexpr int M = 1 << LOGM, NZT = M / PENCIL;
    const int kx = w / NZT, z0 = (w % NZT) * PENCIL;
    cplx<T> *base = data + off + R.spec_off + ((long long)kx * M + z0) * M;
    __syncthreads();
    for (int e = threadIdx.x; e < PENCIL * M; e += FFT_THREADS) {
        const int y = e & (M - 1), l = e >> LOGM;
        buf[brev(y, LOGM) * LS + l] = base[l * M + y];
    }
    __syncthreads();
    if (inverse) fft_lines_t<T, LOGM>(buf, 1, LS, LOG_PENCIL, tw, true);
    else fft_lines_t<T, LOGM>(buf, 1, LS, LOG_PENCIL, tw, false);
    for (int e = threadIdx.x; e < PENCIL * M; e += FFT_THREADS) {
        const int y = e & (M - 1), l = e >> LOGM;
        base[l * M + y] = buf[y * LS + l];
    }
}

template <typename T>
__global__ void __launch_bounds__(FFT_THREADS)
k_fft_y(const RepDev *__restrict__ reps, int nrep, cplx<T> *__restrict__ data, long long stride,
        int ncomp, const cplx<T> *__restrict__ twg, int nitems_per_comp, bool inverse)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *tw = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *buf = tw + 128;
    load_twiddles<T>(tw, twg);
    for (int item = blockIdx.x; item < nitems_per_comp * ncomp; item += gridDim.x) {
        const int comp = item / nitems_per_comp, it = item % nitems_per_comp;
        const int r = find_rep(it, nrep, [&](int k) { return reps[k].wb_off; });
        const RepDev &R = reps[r];
        const int w = it - R.wb_off;
        const long long off = comp * stride;
        switch (R.logM) {  // block-uniform: one replica per item
        case 5: y_item<T, 5>(R, w, data, off, buf, tw, inverse); break;
        case 6: y_item<T, 6>(R, w, data, off, buf, tw, inverse); break;
        case 7: y_item<T, 7>(R, w, data, off, buf, tw, inverse); break;
        default: y_item<T, 8>(R, w, data, off, buf, tw, inverse); break;
        }
    }
}

// Pass C: forward FFT along z, U_f partial, phi = (G/V) rho_k, then the three
// field spectra with their inverse z transforms. E_z = IFFT_z(-i kz phi);
// E_x and E_y use psi = IFFT_z(phi) since their multipliers are constant
// along z: E_x = -i kx psi, E_y = -i ky psi. Item = (replica, kx, 16-wide y
// tile); the item body is instantiated per mesh side.
template <typename T, int LOGM>
__device__ __forceinline__ void z_green_item(const RepDev &R, int w,
                                             const cplx<T> *__restrict__ spec,
                                             const T *__restrict__ green,
                                             cplx<T> *__restrict__ ek, long long nspec,
                                             double *__restrict__ u_out, cplx<T> *buf,
                                             const cplx<T> *tw, double *red)
{
    constexpr int M = 1 << LOGM, NYT = M / PENCIL;
    cplx<T> *buf2 = buf + M * LS;
    const int kx = w / NYT, y0 = (w % NYT) * PENCIL;
    const long long lbase = R.spec_off + (long long)kx * M * M + y0;  // + z*M + l
    __syncthreads();
    for (int e = threadIdx.x; e < PENCIL * M; e += FFT_THREADS) {
        const int l = e & (PENCIL - 1), z = e >> LOG_PENCIL;
        buf[brev(z, LOGM) * LS + l] = spec[lbase + z * M + l];
    }
    __syncthreads();
    fft_lines_t<T, LOGM>(buf, 1, LS, LOG_PENCIL, tw, false);
    const double wkx = (kx == 0 || kx == (M >> 1)) ? 1.0 : 2.0;
    double u = 0.0;
    for (int e = threadIdx.x; e < PENCIL * M; e += FFT_THREADS) {
        const int l = e & (PENCIL - 1), n = e >> LOG_PENCIL;
        const cplx<T> rk = buf[n * LS + l];
        const T g = green[lbase + n * M + l];
        u += wkx * (double)g * ((double)rk.x * rk.x + (double)rk.y * rk.y);
        buf2[brev(n, LOGM) * LS + l] = make_c<T>(g * rk.x, g * rk.y);
    }
    __syncthreads();
    const T twopi_L = (T)(6.283185307179586477 * R.inv_L);
    for (int e = threadIdx.x; e < PENCIL * M; e += FFT_THREADS) {
        const int l = e & (PENCIL - 1), n = e >> LOG_PENCIL;
        const int br = brev(n, LOGM);
        const cplx<T> ph = buf2[br * LS + l];
        const T kz = (n == (M >> 1)) ? (T)0 : twopi_L * (T)freq(n, M);
        // -i kz phi = (kz phi.y, -kz phi.x)
        buf[br * LS + l] = make_c<T>(kz * ph.y, -kz * ph.x);
    }
    __syncthreads();
    fft_lines_t<T, LOGM>(buf, 1, LS, LOG_PENCIL, tw, true);   // E_z
    fft_lines_t<T, LOGM>(buf2, 1, LS, LOG_PENCIL, tw, true);  // psi
    const T kxv = (kx == (M >> 1)) ? (T)0 : twopi_L * (T)kx;
    for (int e = threadIdx.x; e < PENCIL * M; e += FFT_THREADS) {
        const int l = e & (PENCIL - 1), z = e >> LOG_PENCIL;
        const int yy = y0 + l;
        const T kyv = (yy == (M >> 1)) ? (T)0 : twopi_L * (T)freq(yy, M);
        const cplx<T> ps = buf2[z * LS + l];
        const long long o = lbase + z * M + l;
        ek[o] = make_c<T>(kxv * ps.y, -kxv * ps.x);
        ek[nspec + o] = make_c<T>(kyv * ps.y, -kyv * ps.x);
        ek[2 * nspec + o] = buf[z * LS + l];
    }
    const double ut = block_sum(u, red);
    if (threadIdx.x == 0) *u_out = ut;
}

template <typename T>
__global__ void __launch_bounds__(FFT_THREADS)
k_fft_z_green(const RepDev *__restrict__ reps, int nrep, const cplx<T> *__restrict__ spec,
              const T *__restrict__ green, cplx<T> *__restrict__ ek, long long nspec,
              double *__restrict__ u_part, const cplx<T> *__restrict__ twg, int nitems)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *tw = reinterpret_cast<cplx<T> *>(smem_raw);
    __shared__ double red[32];
    load_twiddles<T>(tw, twg);
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int r = find_rep(item, nrep, [&](int k) { return reps[k].wc_off; });
        const RepDev &R = reps[r];
        const int w = item - R.wc_off;
        cplx<T> *buf = tw + 128;
        double *u_out = u_part + item;
        switch (R.logM) {  // block-uniform: one replica per item
        case 5: z_green_item<T, 5>(R, w, spec, green, ek, nspec, u_out, buf, tw, red); break;
        case 6: z_green_item<T, 6>(R, w, spec, green, ek, nspec, u_out, buf, tw, red); break;
        case 7: z_green_item<T, 7>(R, w, spec, green, ek, nspec, u_out, buf, tw, red); break;
        default: z_green_item<T, 8>(R, w, spec, green, ek, nspec, u_out, buf, tw, red); break;
        }
    }
}

// Passes B-D fused for meshes whose kx planes fit in shared memory
// (M <= PLANE_MAX): one CTA per (replica, kx) loads the plane rho_k(kx,z,y),
// transforms it along y and z, forms the U_f partial and phi = (G/V) rho_k,
// and transforms back: E_z = IFFT_y IFFT_z(-i kz phi), E_y = IFFT_y(-i ky
// IFFT_z(phi)), E_x = -i kx IFFT_y IFFT_z(phi) -- seven line-FFT sweeps in
// shared memory, one plane read and three plane writes. The plane is stored
// [z][y] with a padded row (M+1); radix-2 DIT needs bit-reversed input, so the
// load and the multiplies write bit-reversed positions.
constexpr int PLANE_MAX = 64;

template <typename T, int LOGM>
__device__ __forceinline__ void plane_item(const RepDev &R, int kx, const cplx<T> *__restrict__ spec,
                                           const T *__restrict__ green, cplx<T> *__restrict__ ek,
                                           long long nspec, double *__restrict__ u_out,
                                           cplx<T> *A, cplx<T> *B, const cplx<T> *tw,
                                           double *red)
{
    constexpr int M = 1 << LOGM, LD = M + 1, MM = M * M;
    const long long lbase = R.spec_off + (long long)kx * M * M;
    __syncthreads();
    for (int e = threadIdx.x; e < MM; e += FFT_THREADS) {
        const int z = e >> LOGM, y = e & (M - 1);
        A[brev(z, LOGM) * LD + brev(y, LOGM)] = spec[lbase + e];
    }
    // this thread's influence-function values, in flight during the sweeps
    constexpr int GPT = (MM + FFT_THREADS - 1) / FFT_THREADS;
    T gr[GPT];
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
        const int e = threadIdx.x + i * FFT_THREADS;
        gr[i] = e < MM ? __ldg(green + lbase + e) : (T)0;
    }
    __syncthreads();
    fft_lines_t<T, LOGM>(A, LD, 1, LOGM, tw, false);  // along y
    fft_lines_t<T, LOGM>(A, 1, LD, LOGM, tw, false);  // along z
    const double wkx = (kx == 0 || kx == (M >> 1)) ? 1.0 : 2.0;
    double u = 0.0;
#pragma unroll
    for (int i = 0; i < GPT; ++i) {
        const int e = threadIdx.x + i * FFT_THREADS;
        if (e >= MM) break;
        const int z = e >> LOGM, y = e & (M - 1);
        const cplx<T> rk = A[z * LD + y];
        const T g = gr[i];
        u += wkx * (double)g * ((double)rk.x * rk.x + (double)rk.y * rk.y);
        B[brev(z, LOGM) * LD + brev(y, LOGM)] = make_c<T>(g * rk.x, g * rk.y);
    }
    __syncthreads();
    const T twopi_L = (T)(6.283185307179586477 * R.inv_L);
    for (int e = threadIdx.x; e < MM; e += FFT_THREADS) {
        const int zb = e >> LOGM, yb = e & (M - 1);
        const int z = brev(zb, LOGM);
        const T kz = (z == (M >> 1)) ? (T)0 : twopi_L * (T)freq(z, M);
        const cplx<T> ph = B[zb * LD + yb];
        A[zb * LD + yb] = make_c<T>(kz * ph.y, -kz * ph.x);  // -i kz phi
    }
    __syncthreads();
    fft_lines_t<T, LOGM>(A, 1, LD, LOGM, tw, true);  // z, of -i kz phi
    fft_lines_t<T, LOGM>(B, 1, LD, LOGM, tw, true);  // z, of phi: psi
    fft_lines_t<T, LOGM>(A, LD, 1, LOGM, tw, true);  // y: E_z
    cplx<T> *Ez = ek + 2 * nspec + lbase;
    for (int e = threadIdx.x; e < MM; e += FFT_THREADS) {
        const int z = e >> LOGM, y = e & (M - 1);
        Ez[e] = A[z * LD + y];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < MM; e += FFT_THREADS) {
        const int z = e >> LOGM, yb = e & (M - 1);
        const int y = brev(yb, LOGM);
        const T ky = (y == (M >> 1)) ? (T)0 : twopi_L * (T)freq(y, M);
        const cplx<T> ps = B[z * LD + yb];
        A[z * LD + yb] = make_c<T>(ky * ps.y, -ky * ps.x);  // -i ky psi
    }
    __syncthreads();
    fft_lines_t<T, LOGM>(A, LD, 1, LOGM, tw, true);  // y: E_y
    fft_lines_t<T, LOGM>(B, LD, 1, LOGM, tw, true);  // y: IFFT(psi)
    const T kxv = (kx == (M >> 1)) ? (T)0 : twopi_L * (T)kx;
    cplx<T> *Ey = ek + nspec + lbase;
    cplx<T> *Ex = ek + lbase;
    for (int e = threadIdx.x; e < MM; e += FFT_THREADS) {
        const int z = e >> LOGM, y = e & (M - 1);
        Ey[e] = A[z * LD + y];
        const cplx<T> ps = B[z * LD + y];
        Ex[e] = make_c<T>(kxv * ps.y, -kxv * ps.x);
    }
    const double ut = block_sum(u, red);
    if (threadIdx.x == 0) *u_out = ut;
}

template <typename T>
__global__ void __launch_bounds__(FFT_THREADS)
k_fft_plane(const RepDev *__restrict__ reps, int nrep, const cplx<T> *__restrict__ spec,
            const T *__restrict__ green, cplx<T> *__restrict__ ek, long long nspec,
            double *__restrict__ u_part, const cplx<T> *__restrict__ twg, int nitems)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *tw = reinterpret_cast<cplx<T> *>(smem_raw);
    __shared__ double red[32];
    load_twiddles<T>(tw, twg);
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int r = find_rep(item, nrep, [&](int k) { return reps[k].wp_off; });
        const RepDev &R = reps[r];
        const int kx = item - R.wp_off;
        cplx<T> *A = tw + 128;
        cplx<T> *B = A + R.M * (R.M + 1);
        if (R.logM == 5)
            plane_item<T, 5>(R, kx, spec, green, ek, nspec, u_part + item, A, B, tw, red);
        else
            plane_item<T, 6>(R, kx, spec, green, ek, nspec, u_part + item, A, B, tw, red);
    }
}

// Two adjacent spectrum rows a, b of line l, wavenumber k, packed into the
// complex line of an inverse transform whose real and imaginary parts come
// out as the two real rows (k and M - k from Hermitian symmetry).
template <typename T, int LOGM>
__device__ __forceinline__ void c2r_split(cplx<T> *buf, int k, int l, cplx<T> a, cplx<T> b)
{
    constexpr int M = 1 << LOGM;
    if (k == 0 || k == (M >> 1)) {
        buf[brev(k, LOGM) * LSX + l] = make_c<T>(a.x, b.x);
    } else {
        buf[brev(k, LOGM) * LSX + l] = make_c<T>(a.x - b.y, a.y + b.x);
        buf[brev(M - k, LOGM) * LSX + l] = make_c<T>(a.x + b.y, b.x - a.y);
    }
}

// Pass E: C2R along x of the three field spectra, written as real meshes
// efield[c][z][y][x]. Item = (replica, component, z, tile of 2 x_lines rows); rows
// 2l and 2l+1 share complex line l: Z[k] = Xa[k] + i Xb[k] over the
// Hermitian extension, with the imaginary parts at k = 0 and M/2 dropped.
// Instantiated per mesh side like pass A.
template <typename T, int LOGM>
__device__ __forceinline__ void x_c2r_item(const RepDev &R, int comp, int w,
                                           const cplx<T> *__restrict__ ek, long long nspec,
                                           T *__restrict__ efield, long long nmesh, cplx<T> *buf,
                                           const cplx<T> *tw)
{
    constexpr int M = 1 << LOGM;
    constexpr int LNL = x_lines_log(LOGM), NROW = 2 << LNL;  // complex lines, real rows
    constexpr int NYT = M >> (LNL + 1), NK = (M >> 1) + 1;
    const int z = w / NYT, y0 = (w % NYT) * NROW;
    const cplx<T> *src = ek + comp * nspec + R.spec_off + (long long)z * M + y0;
    __syncthreads();
    if constexpr (sizeof(T) == 4) {
        for (int e = threadIdx.x; e < (NK << LNL); e += FFT_THREADS) {
            const int l = e & ((1 << LNL) - 1), k = e >> LNL;
            const long long o = (long long)k * M * M + 2 * l;
            // o is even: one 16-byte load
            const float4 ab = __ldg(reinterpret_cast<const float4 *>(src + o));
            const cplx<T> a = make_c<T>(ab.x, ab.y), b = make_c<T>(ab.z, ab.w);
            c2r_split<T, LOGM>(buf, k, l, a, b);
        }
    } else {
        for (int e = threadIdx.x; e < (NK << LNL); e += FFT_THREADS) {
            const int l = e & ((1 << LNL) - 1), k = e >> LNL;
            const long long o = (long long)k * M * M + 2 * l;
            c2r_split<T, LOGM>(buf, k, l, src[o], src[o + 1]);
        }
    }
    __syncthreads();
    fft_lines_t<T, LOGM>(buf, 1, LSX, LNL, tw, true);
    T *dst = efield + comp * nmesh + R.mesh_off + ((long long)z * M + y0) * M;
    for (int e = threadIdx.x; e < NROW * M; e += FFT_THREADS) {
        const int x = e & (M - 1), j = e >> LOGM;
        const cplx<T> v = buf[x * LSX + (j >> 1)];
        dst[j * M + x] = (j & 1) ? v.y : v.x;
    }
}

template <typename T>
__global__ void __launch_bounds__(FFT_THREADS)
k_fft_x_c2r(const RepDev *__restrict__ reps, int nrep, const cplx<T> *__restrict__ ek,
            long long nspec, T *__restrict__ efield, long long nmesh,
            const cplx<T> *__restrict__ twg, int nitems_per_comp)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<T> *tw = reinterpret_cast<cplx<T> *>(smem_raw);
    cplx<T> *buf = tw + 128;
    load_twiddles<T>(tw, twg);
    for (int item = blockIdx.x; item < nitems_per_comp * 3; item += gridDim.x) {
        const int comp = item / nitems_per_comp, it = item % nitems_per_comp;
        const int r = find_rep(it, nrep, [&](int k) { return reps[k].wa_off; });
        const RepDev &R = reps[r];
        const int w = it - R.wa_off;
        switch (R.logM) {  // block-uniform: one replica per item
        case 5: x_c2r_item<T, 5>(R, comp, w, ek, nspec, efield, nmesh, buf, tw); break;
        case 6: x_c2r_item<T, 6>(R, comp, w, ek, nspec, efield, nmesh, buf, tw); break;
        case 7: x_c2r_item<T, 7>(R, comp, w, ek, nspec, efield, nmesh, buf, tw); break;
        default: x_c2r_item<T, 8>(R, comp, w, ek, nspec, efield, nmesh, buf, tw); break;
        }
    }
}

// ---------------------------------------------------------------------------
// Gather
// ---------------------------------------------------------------------------

// Field at each particle (yukawa_pm_ord6.py:298-300): E = sum over the 216
// stencil nodes of E[node] wz wy wx, written as (Ex, Ey, Ez, Z) in
// brick-sorted order so the caller forms acc = Z E (:308-310). One CTA per
// brick: each field component's TILE^3 neighbourhood of the brick is staged
// in shared memory (coalesced rows), and every particle of the brick reads
// its 216 nodes from there; each thread keeps the weights of up to GPT
// particles across the three components.
constexpr int G_THREADS = 256;

// Gather tiles keep rows of GTX nodes (TILE padded up) so each row is filled
// with 16-byte copies: a brick starts on a multiple of 16 nodes and M is a
// multiple of 16, so every 16-byte chunk -- wrapped ones included -- is
// aligned in global and shared memory.
constexpr int GTX = 24;
constexpr int GTILE = TILE * TILE * GTX;

// NB field-tile buffers per CTA: with two, the copy of component c+1 is in
// flight while component c is summed; with one, the CTA is half the size and,
// held to 64 registers, four of them share an SM (FP32: 57 against 63 us on
// the 20 x 64^3 ensemble). The choice is the context's gather_mode.
//
// NC field components per CTA: 3 (a CTA per brick), or 1 (a CTA per brick and
// component: three times the work items, each staging one tile and repeating
// the weights, so the SMs' last wave is shorter and no CTA waits for its own
// next copy).
template <typename T, int NB, int NC>
__global__ void __launch_bounds__(G_THREADS, sizeof(T) == 4 ? (NB == 1 ? 4 : 1) : 2)
k_gather(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ brick_start,
         const int *__restrict__ brick_perm, const double *__restrict__ pos,
         const double *__restrict__ charge, const T *__restrict__ efield, long long nmesh,
         typename V4<T>::t *__restrict__ acc_pm, int nbrick)
{
    extern __shared__ __align__(16) unsigned char g_smem[];
    T *tile = reinterpret_cast<T *>(g_smem);
    // per thread of the chunk: its particle (slot p, or -1), node offsets,
    // local tile offset of the stencil's first node (or -1)
    __shared__ int g_src[G_THREADS];
    __shared__ T g_o[3][G_THREADS];
    __shared__ int g_base[G_THREADS];
    __shared__ int g_cnt[32];
    const int lane = threadIdx.x & 31;
    static_assert(NC == 3 || NC == 1, "a whole brick or one component per CTA");
    constexpr int IPB = 3 / NC;  // work items per brick
    for (int it = blockIdx.x; it < nbrick * IPB; it += gridDim.x) {
        const int b = it / IPB, cfirst = (it % IPB) * NC, cend = cfirst + NC;
        const int r = find_rep(b, nrep, [&](int k) { return reps[k].brick_off; });
        const RepDev &R = reps[r];
        const int nb = R.nb, M = R.M, local = b - R.brick_off;
        const int bx = (local % nb) * BRICK, by = ((local / nb) % nb) * BRICK,
                  bz = (local / (nb * nb)) * BRICK;
        const int p0 = brick_start[b], p1 = brick_start[b + 1];
        for (int c0 = p0; c0 < p1; c0 += G_THREADS) {
            // Lanes of a warp read their particles' stencils at the same
            // offsets from different bases, so two lanes whose bases share a
            // shared-memory bank conflict on every read. The chunk's particles
            // are ranked by bank (base mod 32) and dealt round-robin to the
            // warps: each warp gets bases spread over the banks. Which thread
            // handles a particle does not change its sums.
            const int nch = min(G_THREADS, p1 - c0);
            int bank = 0, rank = 0, base0 = -1;
            T ox0 = 0, oy0 = 0, oz0 = 0;
            if (threadIdx.x < nch) {
                const int i = brick_perm[c0 + threadIdx.x];
                double ox, oy, oz;
                const int ix = base_offset(pos[3 * i + 0], R.h, ox);
                const int iy = base_offset(pos[3 * i + 1], R.h, oy);
                const int iz = base_offset(pos[3 * i + 2], R.h, oz);
                const int lx = wrapM(ix, M) - bx, ly = wrapM(iy, M) - by, lz = wrapM(iz, M) - bz;
                // (a particle outside [-L, 2L) was flagged by the key pass)
                if ((unsigned)lx < (unsigned)BRICK && (unsigned)ly < (unsigned)BRICK &&
                    (unsigned)lz < (unsigned)BRICK) {
                    base0 = (lz * TILE + ly) * GTX + lx;
                    bank = base0 & 31;
                }
                ox0 = (T)ox;
                oy0 = (T)oy;
                oz0 = (T)oz;
            }
            __syncthreads();  // the previous chunk / brick is done with g_* and the buffers
            g_src[threadIdx.x] = -1;
            if (threadIdx.x < 32) g_cnt[threadIdx.x] = 0;
            __syncthreads();
            if (threadIdx.x < nch) rank = atomicAdd(&g_cnt[bank], 1);
            __syncthreads();
            if (threadIdx.x < 32) {  // exclusive scan of the bank counts
                const int v = g_cnt[lane];
                int x = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += t;
                }
                g_cnt[lane] = x - v;
            }
            __syncthreads();
            if (threadIdx.x < nch) {
                const int q = g_cnt[bank] + rank, nw = (nch + 31) >> 5;
                const int tgt = (q % nw) * 32 + q / nw;
                g_src[tgt] = c0 + threadIdx.x;
                g_o[0][tgt] = ox0;
                g_o[1][tgt] = oy0;
                g_o[2][tgt] = oz0;
                g_base[tgt] = base0;
            }
            __syncthreads();
            const int p = g_src[threadIdx.x];
            T wx[6], wy[6], wz[6];
            const int base = p >= 0 ? g_base[threadIdx.x] : -1;
            T e[3] = {(T)0, (T)0, (T)0};
            if (base >= 0) {
                weights6<T>(g_o[0][threadIdx.x], wx);
                weights6<T>(g_o[1][threadIdx.x], wy);
                weights6<T>(g_o[2][threadIdx.x], wz);
            }
            // component tiles through the NB buffers
            auto issue = [&](int comp) {
                constexpr int EPC = 16 / sizeof(T);   // elements per 16-byte chunk
                constexpr int CPR = GTX / EPC;        // chunks per tile row
                constexpr int RP = G_THREADS / CPR;   // tile rows per pass
                static_assert(RP % TILE == 0, "a thread keeps its row's y");
                if (threadIdx.x < RP * CPR) {
                    // thread: chunk ch of rows r0, r0 + RP, ... -- fixed x and
                    // y, z advancing by RP / TILE
                    const int ch = threadIdx.x % CPR, r0 = threadIdx.x / CPR;
                    const int gx = (bx + ch * EPC) & (M - 1), gy = (by + r0 % TILE) & (M - 1);
                    const T *exy = efield + comp * nmesh + R.mesh_off + (long long)gy * M + gx;
                    T *d = tile + (comp % NB) * GTILE + r0 * GTX + ch * EPC;
                    for (int tz = r0 / TILE; tz < TILE; tz += RP / TILE, d += RP * GTX)
                        cp_async16(d, exy + (long long)((bz + tz) & (M - 1)) * M * M);
                }
                asm volatile("cp.async.commit_group;\n" ::: "memory");
            };
            issue(cfirst);
            for (int comp = cfirst; comp < cend; ++comp) {
                if (NB == 2 && comp + 1 < cend) {
                    issue(comp + 1);
                    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
                } else {
                    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
                }
                __syncthreads();
                const T *tl = tile + (comp % NB) * GTILE;
                if (base >= 0) {
                    // separable contraction: sum_g wz sum_a wy sum_c wx E
                    T acc = 0;
#pragma unroll
                    for (int g = 0; g < 6; ++g) {
                        T sg = 0;
#pragma unroll
                        for (int a = 0; a < 6; ++a) {
                            const T *row = tl + base + (g * TILE + a) * GTX;
                            T sa = 0;
#pragma unroll
                            for (int c = 0; c < 6; ++c) sa += wx[c] * row[c];
                            sg += wy[a] * sa;
                        }
                        acc += wz[g] * sg;
                    }
                    e[comp] = acc;
                }
                if (NB == 1 && comp + 1 < cend) {
                    __syncthreads();
                    issue(comp + 1);
                } else if (comp + 2 < cend) {
                    __syncthreads();  // buffer (comp % 2) is refilled next
                }
            }
            if (p >= 0) {
                if constexpr (NC == 3) {
                    typename V4<T>::t out;
                    out.x = e[0];
                    out.y = e[1];
                    out.z = e[2];
                    out.w = (T)charge[brick_perm[p]];
                    acc_pm[p] = out;
                } else {
                    T *o = reinterpret_cast<T *>(acc_pm + p);  // (Ex, Ey, Ez, Z)
                    o[cfirst] = e[cfirst];
                    if (cfirst == 0) o[3] = (T)charge[brick_perm[p]];
                }
            }
        }
    }
}

// Per-replica U_f = 1/2 sum over the replica's pass-C partials.
__global__ void k_reduce_pm(const RepDev *__restrict__ reps, int nrep,
                            const double *__restrict__ u_part, int wc_total, int wp_total,
                            double *__restrict__ rep_out)
{
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nrep;
         r += gridDim.x * (blockDim.x >> 5)) {
        if (reps[r].M == 0) {
            if (lane == 0) rep_out[8 * r + RO_UPM] = 0.0;
            continue;
        }
        // multi-pass items [wc_off, ...) and plane items (stored after wc_total)
        const int b = reps[r].wc_off, e = (r + 1 < nrep) ? reps[r + 1].wc_off : wc_total;
        const int pb = wc_total + reps[r].wp_off,
                  pe = wc_total + ((r + 1 < nrep) ? reps[r + 1].wp_off : wp_total);
        double t = 0.0;
        for (int k = b + lane; k < e; k += 32) t += u_part[k];
        for (int k = pb + lane; k < pe; k += 32) t += u_part[k];
        t = warp_sum(t);
        if (lane == 0) rep_out[8 * r + RO_UPM] = 0.5 * t;
    }
}

// ---------------------------------------------------------------------------
// Conversions used by the compat entry points
// ---------------------------------------------------------------------------

// Influence function from the reference's fftshifted (M,M,M) FP64 layout
// (index n <-> k = 2 pi (n - M/2)/L) into green[kx][z][y] / V.
template <typename T>
__global__ void k_green_from_shifted(const RepDev *__restrict__ reps, int rep,
                                     const double *__restrict__ gk, T *__restrict__ green)
{
    const RepDev &R = reps[rep];
    const int M = R.M, h = M >> 1, nk = h + 1;
    const long long n = (long long)nk * M * M;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(e % M), z = (int)((e / M) % M), kx = (int)(e / ((long long)M * M));
        const int sx = (kx + h) & (M - 1), sy = (y + h) & (M - 1), sz = (z + h) & (M - 1);
        green[R.spec_off + e] = (T)(gk[((long long)sz * M + sy) * M + sx] * R.inv_V);
    }
}

template <typename T>
__global__ void k_tiles_to_mesh(const RepDev *__restrict__ reps, int rep,
                                const T *__restrict__ tiles, double *__restrict__ rho)
{
    const RepDev &R = reps[rep];
    const int M = R.M;
    const long long n = (long long)M * M * M;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e % M), y = (int)((e / M) % M), z = (int)(e / ((long long)M * M));
        rho[e] = (double)rho_at<T>(R, tiles, x, y, z);
    }
}

template <typename T>
__global__ void k_efield_from_mesh(const RepDev *__restrict__ reps, int rep,
                                   const double *__restrict__ ex, const double *__restrict__ ey,
                                   const double *__restrict__ ez, T *__restrict__ efield,
                                   long long nmesh)
{
    const RepDev &R = reps[rep];
    const long long n = (long long)R.M * R.M * R.M;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        efield[R.mesh_off + e] = (T)ex[e];
        efield[nmesh + R.mesh_off + e] = (T)ey[e];
        efield[2 * nmesh + R.mesh_off + e] = (T)ez[e];
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

template <typename T> static size_t fft_smem(int maxM, int nbuf)
{
    return (128 + (size_t)nbuf * maxM * LS) * sizeof(cplx<T>);
}

template <typename T> static size_t plane_smem(int M)
{
    return (128 + 2 * (size_t)M * (M + 1)) * sizeof(cplx<T>);
}

template <typename T> static size_t x_smem(int maxM)
{
    return (128 + (size_t)maxM * LSX) * sizeof(cplx<T>);
}

template <typename K> static void set_smem(K kernel, size_t bytes)
{
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static int grid_items(int n, int cap = 148 * 8) { return n < cap ? (n > 0 ? n : 1) : cap; }

template <typename T> void configure_mesh_kernels()
{
    set_smem(k_assign<T>, assign_smem<T>());
    set_smem(k_assign_i32, 2 * TILE3 * sizeof(int));
    set_smem(k_fft_x_r2c<T>, x_smem<T>(256));
    set_smem(k_fft_y<T>, fft_smem<T>(256, 1));
    set_smem(k_fft_z_green<T>, fft_smem<T>(256, 2));
    set_smem(k_fft_x_c2r<T>, x_smem<T>(256));
    set_smem(k_gather<T, 1, 3>, GTILE * sizeof(T));
    set_smem(k_gather<T, 1, 1>, GTILE * sizeof(T));
    if constexpr (sizeof(T) == 4) set_smem(k_gather<T, 2, 3>, 2 * GTILE * sizeof(T));
    set_smem(k_fft_plane<T>, plane_smem<T>(PLANE_MAX));
}

template <typename T> void launch_assign(const DevState &s, cudaStream_t st)
{
    if (sizeof(T) == 4) {
        k_assign_i32<<<grid_items(s.nbrick, 148 * 16), A32_THREADS, 2 * TILE3 * sizeof(int), st>>>(
            s.reps, s.nrep, s.brick_start, s.brick_perm, s.pos, s.charge, (float *)s.tiles,
            s.nbrick);
        return;
    }
    const size_t smem = assign_smem<T>();
    k_assign<T><<<grid_items(s.nbrick, 148 * 16), A_THREADS, smem, st>>>(
        s.reps, s.nrep, s.brick_start, s.brick_perm, s.pos, s.charge, (T *)s.tiles, s.nbrick,
        s.status);
}

template <typename T> void launch_fft_forward(const DevState &s, cudaStream_t st)
{
    using C = cplx<T>;
    const int maxM = s.max_mesh;
    const size_t sm1 = fft_smem<T>(maxM, 1), sm2 = fft_smem<T>(maxM, 2);
    k_fft_x_r2c<T><<<grid_items(s.wa), FFT_THREADS, x_smem<T>(maxM), st>>>(s.reps, s.nrep, (const T *)s.tiles,
                                                                (C *)s.spec, (const C *)s.twiddle, s.wa);
    if (s.wb > 0) {
        k_fft_y<T><<<grid_items(s.wb), FFT_THREADS, sm1, st>>>(s.reps, s.nrep, (C *)s.spec, s.nspec,
                                                                1, (const C *)s.twiddle, s.wb, false);
        k_fft_z_green<T><<<grid_items(s.wc), FFT_THREADS, sm2, st>>>(
            s.reps, s.nrep, (const C *)s.spec, (const T *)s.green, (C *)s.ek, s.nspec, s.u_pm_part,
            (const C *)s.twiddle, s.wc);
    }
    if (s.wp > 0) {
        k_fft_plane<T><<<grid_items(s.wp), FFT_THREADS, plane_smem<T>(s.max_plane), st>>>(
            s.reps, s.nrep, (const C *)s.spec, (const T *)s.green, (C *)s.ek, s.nspec,
            s.u_pm_part + s.wc, (const C *)s.twiddle, s.wp);
    }
}

int fft_kernel_count(const DevState &s) { return 2 + (s.wb > 0 ? 3 : 0) + (s.wp > 0 ? 1 : 0); }
int plane_max_mesh() { return PLANE_MAX; }  // the largest side the plane kernel takes

template <typename T> void launch_fft_inverse(const DevState &s, cudaStream_t st)
{
    using C = cplx<T>;
    const size_t sm1 = fft_smem<T>(s.max_mesh, 1);
    if (s.wb > 0)
        k_fft_y<T><<<grid_items(3 * s.wb), FFT_THREADS, sm1, st>>>(s.reps, s.nrep, (C *)s.ek, s.nspec,
                                                                    3, (const C *)s.twiddle, s.wb, true);
    k_fft_x_c2r<T><<<grid_items(3 * s.wa), FFT_THREADS, x_smem<T>(s.max_mesh), st>>>(
        s.reps, s.nrep, (const C *)s.ek, s.nspec, (T *)s.efield, s.nmesh, (const C *)s.twiddle,
        s.wa);
}

template <typename T> void launch_gather(const DevState &s, cudaStream_t st)
{
    using A = typename V4<T>::t;
    if (sizeof(T) == 4 && s.gather_mode == 2)
        k_gather<T, 2, 3><<<grid_items(s.nbrick, 148 * 16), G_THREADS, 2 * GTILE * sizeof(T), st>>>(
            s.reps, s.nrep, s.brick_start, s.brick_perm, s.pos, s.charge, (const T *)s.efield,
            s.nmesh, (A *)s.acc_pm, s.nbrick);
    else if (s.gather_mode == 0)
        k_gather<T, 1, 1><<<grid_items(3 * s.nbrick, 148 * 16), G_THREADS, GTILE * sizeof(T), st>>>(
            s.reps, s.nrep, s.brick_start, s.brick_perm, s.pos, s.charge, (const T *)s.efield,
            s.nmesh, (A *)s.acc_pm, s.nbrick);
    else
        k_gather<T, 1, 3><<<grid_items(s.nbrick, 148 * 16), G_THREADS, GTILE * sizeof(T), st>>>(
            s.reps, s.nrep, s.brick_start, s.brick_perm, s.pos, s.charge, (const T *)s.efield,
            s.nmesh, (A *)s.acc_pm, s.nbrick);
}

void launch_reduce_pm(const DevState &s, cudaStream_t st)
{
    k_reduce_pm<<<(s.nrep + 3) / 4, 128, 0, st>>>(s.reps, s.nrep, s.u_pm_part, s.wc, s.wp,
                                                  s.rep_out);
}

template <typename T>
void launch_green_from_host_layout(const DevState &s, int rep, const double *gk_dev, cudaStream_t st)
{
    k_green_from_shifted<T><<<592, 256, 0, st>>>(s.reps, rep, gk_dev, (T *)s.green);
}

template <typename T> void launch_tiles_to_mesh(const DevState &s, int rep, double *rho, cudaStream_t st)
{
    k_tiles_to_mesh<T><<<592, 256, 0, st>>>(s.reps, rep, (const T *)s.tiles, rho);
}

template <typename T>
void launch_efield_from_mesh(const DevState &s, int rep, const double *ex, const double *ey,
                             const double *ez, cudaStream_t st)
{
    k_efield_from_mesh<T><<<592, 256, 0, st>>>(s.reps, rep, ex, ey, ez, (T *)s.efield, s.nmesh);
}

#define P3M_INST(T)                                                                        \
    template void configure_mesh_kernels<T>();                                              \
    template void launch_assign<T>(const DevState &, cudaStream_t);                         \
    template void launch_fft_forward<T>(const DevState &, cudaStream_t);                    \
    template void launch_fft_inverse<T>(const DevState &, cudaStream_t);                    \
    template void launch_gather<T>(const DevState &, cudaStream_t);                         \
    template void launch_green_from_host_layout<T>(const DevState &, int, const double *,   \
                                                   cudaStream_t);                          \
    template void launch_tiles_to_mesh<T>(const DevState &, int, double *, cudaStream_t);   \
    template void launch_efield_from_mesh<T>(const DevState &, int, const double *,         \
                                             const double *, const double *, cudaStream_t);
P3M_INST(float)
P3M_INST(double)

}  // namespace p3m
