// Short-range (PP) Yukawa-Ewald forces over linked cells.
//
// Computes what yukawa_pp.py:6-139 computes: for every pair closer than r_c
// (minimum image through the 27-cell periodic stencil, :54-94)
//   phi(r) = (1/2r) [e^{kr} erfc(ar + k/2a) + e^{-kr} erfc(ar - k/2a)]   (:115)
//   F(r)   = f1 + f2 + f3                                               (:121-124)
// The energy is sum_{i<j} phi. The reference visits each pair once and
// applies Newton's third law; here every particle sums over all of its
// neighbours itself (full list), so each thread owns its particle's force and
// no atomics are needed. Z is ignored, as in the reference.
//
// Both exponentials share one factor: with u+- = ar +- k/2a,
//   e^{+-kr} erfc(u+-) = erfcx(u+-) exp(-(a^2 r^2 + k^2/4a^2))
// so a pair costs one exp and two erfcx (CUDA's exp/erfcx, no re-derived
// math), and f3 = (2a/sqrt(pi)) exp(...)/r.
//
// Layout of the work: one CTA per (home cell, split). The CTA stages the 27
// neighbour cells' particles, shifted into the home cell's frame, in shared
// memory; each thread first filters the staged particles by distance into a
// per-thread list of in-range neighbours (indices in shared memory), then
// evaluates the pair terms only for the listed ones, so a warp does not pay
// the transcendental cost for the ~85% of candidates outside the cutoff.
// Per-thread partial forces are added with Kahan compensation at flush
// granularity; energies are accumulated in FP64.
#include "p3m_kernels.h"

namespace p3m {

template <typename T> struct PairCoef {
    T a, a2, k, k2a, ce, c3, rc2;
};

__device__ __forceinline__ float p_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double p_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float p_exp(float x) { return expf(x); }
__device__ __forceinline__ double p_exp(double x) { return exp(x); }
__device__ __forceinline__ float p_erfcx(float x) { return erfcxf(x); }
__device__ __forceinline__ double p_erfcx(double x) { return erfcx(x); }

// Pair terms at squared distance r2: F(r)/r and phi(r).
template <typename T>
__device__ __forceinline__ void yukawa_ewald_pair(T r2, const PairCoef<T> &c, T &f_over_r, T &phi)
{
    T rinv = p_rsqrt(r2);
    T r = r2 * rinv;
    T ar = c.a * r;
    T E = p_exp(-(c.a2 * r2 + c.ce));
    T xp = p_erfcx(ar + c.k2a);
    T xm = p_erfcx(ar - c.k2a);
    T kr = c.k * r;
    T hE = (T)0.5 * rinv * E;
    phi = hE * (xp + xm);
    T fr = hE * rinv * (xp * ((T)1 - kr) + xm * ((T)1 + kr)) + c.c3 * rinv * E;
    f_over_r = fr * rinv;
}

template <typename T> struct PPCfg;
template <> struct PPCfg<float> { static constexpr int SCAP = 1536, LCAP = 96; };
template <> struct PPCfg<double> { static constexpr int SCAP = 1536, LCAP = 96; };

constexpr int PP_THREADS = 128;

// Shared-memory bytes of the PP kernel: staged neighbours (FP64: one double4;
// FP32: a hi and a lo float4 per particle) and the per-thread lists.
template <typename T> constexpr size_t pp_smem_bytes()
{
    return (size_t)PPCfg<T>::SCAP * 32 + (size_t)PPCfg<T>::LCAP * PP_THREADS * sizeof(unsigned short);
}

// Positions come in as FP64 offsets from the cell origin (double4). The FP64
// path stages them as they are. The FP32 path stages each coordinate as a
// pair of floats (hi = fl(x), lo = fl(x - hi)): the cutoff filter uses hi
// alone, and the pair terms use dx = (xi_hi - xj_hi) + (xi_lo - xj_lo), whose
// error is a rounding of dx itself rather than of the (larger) coordinates --
// with plain FP32 coordinates the position rounding alone gives a ~3e-6
// relative force error.
template <typename T, int TPI>
__global__ void __launch_bounds__(PP_THREADS)
k_pp(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ cell_start,
     const double4 *__restrict__ xs, typename V4<T>::t *__restrict__ acc_out,
     double *__restrict__ u_part, int ncell, int split)
{
    using T4 = typename V4<T>::t;
    constexpr bool F32 = sizeof(T) == 4;
    constexpr int SCAP = PPCfg<T>::SCAP, LCAP = PPCfg<T>::LCAP;
    constexpr int ICH = PP_THREADS / TPI;  // i-particles per CTA pass
    extern __shared__ __align__(16) unsigned char pp_smem[];
    T4 *stage = reinterpret_cast<T4 *>(pp_smem);               // FP64: double4; FP32: hi
    float4 *stage_lo = reinterpret_cast<float4 *>(pp_smem + (size_t)SCAP * 16);  // FP32 only
    unsigned short *list = reinterpret_cast<unsigned short *>(pp_smem + (size_t)SCAP * 32);
    __shared__ int pre[28];
    __shared__ int nstart[27];
    __shared__ double shx[27], shy[27], shz[27];
    __shared__ double red[32];

    const int tid = threadIdx.x;
    const int il = tid / TPI, sub = tid % TPI;

    for (int item = blockIdx.x; item < ncell * split; item += gridDim.x) {
        const int hc = item / split, part = item % split;
        const int r = find_rep(hc, nrep, [&](int k) { return reps[k].cell_off; });
        const RepDev &R = reps[r];
        const int nc = R.nc, local = hc - R.cell_off;
        const int cx = local % nc, cy = (local / nc) % nc, cz = local / (nc * nc);
        const int hstart = cell_start[hc], nhome = cell_start[hc + 1] - hstart;

        PairCoef<T> c;
        c.a = (T)R.alpha;
        c.a2 = (T)(R.alpha * R.alpha);
        c.k = (T)R.kappa;
        c.k2a = (T)(0.5 * R.kappa / R.alpha);
        c.ce = (T)(0.25 * R.kappa * R.kappa / (R.alpha * R.alpha));
        c.c3 = (T)(2.0 * R.alpha / 1.7724538509055160273);
        c.rc2 = (T)(R.rc * R.rc);

        __syncthreads();
        if (tid < 27) {
            int dx = tid % 3 - 1, dy = (tid / 3) % 3 - 1, dz = tid / 9 - 1;
            int nx = (cx + dx + nc) % nc, ny = (cy + dy + nc) % nc, nz = (cz + dz + nc) % nc;
            int nb = R.cell_off + nx + nc * (ny + nc * nz);
            nstart[tid] = cell_start[nb];
            pre[tid + 1] = cell_start[nb + 1] - cell_start[nb];
            shx[tid] = dx * R.cellw;
            shy[tid] = dy * R.cellw;
            shz[tid] = dz * R.cellw;
        }
        __syncthreads();
        if (tid == 0) {
            pre[0] = 0;
            for (int k = 0; k < 27; ++k) pre[k + 1] += pre[k];
        }
        __syncthreads();
        const int total = pre[27];

        double u_thread = 0.0;
        const int nchunks = (nhome + ICH - 1) / ICH;
        for (int ch = part; ch < nchunks; ch += split) {
            const int i = ch * ICH + il;
            const bool have_i = i < nhome;
            T4 xi;          // FP64: position; FP32: hi part
            float4 xl;      // FP32: lo part
            if (have_i) {
                const double4 p = xs[hstart + i];
                if constexpr (F32) {
                    xi.x = (float)p.x; xi.y = (float)p.y; xi.z = (float)p.z; xi.w = 0.f;
                    xl.x = (float)(p.x - (double)xi.x);
                    xl.y = (float)(p.y - (double)xi.y);
                    xl.z = (float)(p.z - (double)xi.z);
                    xl.w = 0.f;
                } else {
                    xi.x = p.x; xi.y = p.y; xi.z = p.z; xi.w = 0.0;
                }
            } else {
                xi.x = xi.y = xi.z = (T)1e18;
                xi.w = (T)0;
                xl.x = xl.y = xl.z = xl.w = 0.f;
            }
            T fx = 0, fy = 0, fz = 0, gx = 0, gy = 0, gz = 0;  // sums and Kahan terms

            for (int w0 = 0; w0 < total; w0 += SCAP) {
                const int wlen = min(SCAP, total - w0);
                __syncthreads();
                for (int k = tid; k < wlen; k += PP_THREADS) {
                    int g = w0 + k;
                    int cc = 0;
                    while (pre[cc + 1] <= g) ++cc;
                    const double4 p = xs[nstart[cc] + g - pre[cc]];
                    const double x = p.x + shx[cc], y = p.y + shy[cc], z = p.z + shz[cc];
                    T4 h;
                    h.x = (T)x; h.y = (T)y; h.z = (T)z; h.w = (T)0;
                    stage[k] = h;
                    if constexpr (F32) {
                        stage_lo[k] = make_float4((float)(x - (double)h.x), (float)(y - (double)h.y),
                                                  (float)(z - (double)h.z), 0.f);
                    }
                }
                __syncthreads();

                int cnt = 0;
                auto flush = [&]() {
                    int mmax = __reduce_max_sync(0xffffffffu, cnt);
                    T px = 0, py = 0, pz = 0;
                    T pu = 0;
                    for (int e = 0; e < mmax; ++e) {
                        if (e < cnt) {
                            const int k = list[e * PP_THREADS + tid];
                            const T4 q = stage[k];
                            T dx = xi.x - q.x, dy = xi.y - q.y, dz = xi.z - q.z;
                            if constexpr (F32) {
                                const float4 ql = stage_lo[k];
                                dx += xl.x - ql.x;
                                dy += xl.y - ql.y;
                                dz += xl.z - ql.z;
                            }
                            T r2 = dx * dx + dy * dy + dz * dz;
                            T fr, ph;
                            yukawa_ewald_pair<T>(r2, c, fr, ph);
                            px += fr * dx;
                            py += fr * dy;
                            pz += fr * dz;
                            pu += ph;
                        }
                    }
                    // Kahan-compensated add of the flush partials
                    T yx = px - gx, tx = fx + yx; gx = (tx - fx) - yx; fx = tx;
                    T yy = py - gy, ty = fy + yy; gy = (ty - fy) - yy; fy = ty;
                    T yz = pz - gz, tz = fz + yz; gz = (tz - fz) - yz; fz = tz;
                    u_thread += (double)pu;
                    cnt = 0;
                };
                for (int k0 = 0; k0 < wlen; k0 += 32) {
                    const int kmax = min(k0 + 32, wlen);
                    for (int k = k0 + sub; k < kmax; k += TPI) {
                        T4 q = stage[k];
                        T dx = xi.x - q.x, dy = xi.y - q.y, dz = xi.z - q.z;
                        T r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 < c.rc2 && r2 > (T)0) {
                            list[cnt * PP_THREADS + tid] = (unsigned short)k;
                            ++cnt;
                        }
                    }
                    if (__any_sync(0xffffffffu, cnt > LCAP - 32)) flush();
                }
                flush();
            }
            // combine the TPI partial sums of this i (fixed shuffle tree)
#pragma unroll
            for (int o = TPI / 2; o > 0; o >>= 1) {
                fx += __shfl_xor_sync(0xffffffffu, fx, o);
                fy += __shfl_xor_sync(0xffffffffu, fy, o);
                fz += __shfl_xor_sync(0xffffffffu, fz, o);
            }
            if (have_i && sub == 0) {
                T4 a;
                a.x = fx;
                a.y = fy;
                a.z = fz;
                a.w = (T)0;
                acc_out[hstart + i] = a;
            }
        }
        double u = block_sum(u_thread, red);
        if (tid == 0) u_part[item] = u;
    }
}

template <typename T, int TPI> static void launch_pp_tpi(const DevState &s, cudaStream_t st)
{
    using T4 = typename V4<T>::t;
    int grid = s.ncell * s.pp_split;
    k_pp<T, TPI><<<grid, PP_THREADS, pp_smem_bytes<T>(), st>>>(
        s.reps, s.nrep, s.cell_start, (const double4 *)s.xs_cell, (T4 *)s.acc_pp, s.u_pp_part,
        s.ncell, s.pp_split);
}

template <typename T> void configure_pp_kernels()
{
    const int smem = (int)pp_smem_bytes<T>();
    cudaFuncSetAttribute(k_pp<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_pp<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_pp<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <typename T> void launch_pp(const DevState &s, cudaStream_t st)
{
    switch (s.pp_tpi) {
    case 2: launch_pp_tpi<T, 2>(s, st); break;
    case 4: launch_pp_tpi<T, 4>(s, st); break;
    default: launch_pp_tpi<T, 1>(s, st);
    }
}

// Per-replica U_pp = 1/2 sum over the replica's (cell, split) partials, in
// index order (one warp per replica).
__global__ void k_reduce_pp(const RepDev *__restrict__ reps, int nrep,
                            const double *__restrict__ u_part, int split, int ncell_total,
                            double *__restrict__ rep_out)
{
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nrep;
         r += gridDim.x * (blockDim.x >> 5)) {
        int b = reps[r].cell_off * split;
        int e = (r + 1 < nrep ? reps[r + 1].cell_off : ncell_total) * split;
        double t = 0.0;
        for (int k = b + lane; k < e; k += 32) t += u_part[k];
        t = warp_sum(t);
        if (lane == 0) rep_out[8 * r + RO_UPP] = 0.5 * t;
    }
}

void launch_reduce_pp(const DevState &s, cudaStream_t st)
{
    k_reduce_pp<<<(s.nrep + 3) / 4, 128, 0, st>>>(s.reps, s.nrep, s.u_pp_part, s.pp_split,
                                                  s.ncell, s.rep_out);
}

template void configure_pp_kernels<float>();
template void configure_pp_kernels<double>();
template void launch_pp<float>(const DevState &, cudaStream_t);
template void launch_pp<double>(const DevState &, cudaStream_t);

}  // namespace p3m
