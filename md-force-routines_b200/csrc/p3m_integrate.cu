// Integrator, thermostat, energies, n(q,t) and the optimal influence function.
//
// One velocity-Verlet step (velocity_verlet_p3m_ord6.py:5-26) is split around
// the force evaluation:
//   k_kick_drift   v += 0.5 a dt; x += v dt; single periodic wrap (:7-19),
//                  fused with the PP-cell / mesh-brick keys of the new x
//   ... sort, PP, PM ...
//   k_kick_finish  a = af (a_pp + Z E) (yukawa_p3m_ord6.py:21); v += 0.5 a dt
//                  (:24); per-block sums of v^2 in FP64
//   k_step_reduce  per replica K = kf sum v^2, T = K/kf/N, U = uf (U_pp + U_pm
//                  + U_self) (yukawa_p3m_ord6.py:23-24) and, in thermostat
//                  mode, the factor of thermostat_p3m_ord6.py:9-23
//   k_scale_vel    v *= factor (thermostat mode only)
// The position and velocity updates use explicitly rounded FP64 operations in
// the reference's order (no FMA contraction), so a step reproduces the
// reference's rounding.
#include "p3m_kernels.h"

namespace p3m {

__device__ __forceinline__ double kick(double v, double a, double dt)
{
    // v + 0.5*a*dt, evaluated as v + ((0.5*a)*dt)
    return __dadd_rn(v, __dmul_rn(__dmul_rn(0.5, a), dt));
}

__device__ __forceinline__ double wrap_once(double x, double L)
{
    // velocity_verlet_p3m_ord6.py:16-19: if x > Lmax: x -= L; if x < Lmin: x += L
    if (x > L) x = __dsub_rn(x, L);
    if (x < 0.0) x = __dadd_rn(x, L);
    return x;
}

__global__ void k_kick_drift(const RepDev *__restrict__ reps, const int *__restrict__ prep,
                             double *__restrict__ pos, double *__restrict__ vel,
                             const double *__restrict__ acc, const double *__restrict__ pos_ref,
                             int ntot, int *__restrict__ brick_key, int *__restrict__ brick_count,
                             int has_mesh, int *rebuild, int *status,
                             const double *__restrict__ pos_pref, int *prune)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        const int r = prep[i];
        const RepDev &R = reps[r];
        double x[3];
        double d2 = 0.0, d2p = 0.0;
        bool vfin = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double v = kick(vel[3 * i + d], acc[3 * i + d], R.dt);
            vfin = vfin && isfinite(v);
            vel[3 * i + d] = v;
            x[d] = wrap_once(__dadd_rn(pos[3 * i + d], __dmul_rn(v, R.dt)), R.L);
            pos[3 * i + d] = x[d];
            // displacement since the last list rebuild, minimum image
            double dd = x[d] - pos_ref[3 * i + d];
            dd -= R.L * rint(dd * R.inv_L);
            d2 += dd * dd;
            if (pos_pref) {  // and since the last inner-list build
                double dp = x[d] - pos_pref[3 * i + d];
                dp -= R.L * rint(dp * R.inv_L);
                d2p += dp * dp;
            }
        }
        // a non-finite velocity (or acceleration) is reported as such; the
        // position it makes is also flagged by particle_keys below
        if (!vfin) raise_status(status, ST_NONFINITE);
        if (d2 > 0.25 * R.skin * R.skin && !rebuild[r]) atomicOr(rebuild + r, 1);
        if (pos_pref && d2p > 0.25 * R.pbuf * R.pbuf && !prune[r]) atomicOr(prune + r, 1);
        int b;
        particle_keys(R, x[0], x[1], x[2], has_mesh, nullptr, &b, status);
        if (b >= 0) {
            brick_key[i] = b;
            atomicAdd(&brick_count[b], 1);
        }
    }
}

// Replica-aligned particle blocks: block b belongs to replica r and covers
// particles p_off + (b - blk_off) * PBLK + [0, PBLK).
__device__ __forceinline__ int block_replica(const RepDev *reps, int nrep, int b)
{
    return find_rep(b, nrep, [&](int k) { return reps[k].blk_off; });
}

// acc = af (a_pp + Z E) for every particle; with do_kick the second half kick
// and the per-block FP64 sum of v^2.
template <typename T>
__global__ void __launch_bounds__(PBLK)
k_kick_finish(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ cell_slot,
              const int *__restrict__ brick_slot, const typename V4<T>::t *__restrict__ acc_pp,
              const typename V4<T>::t *__restrict__ acc_pm, int has_mesh,
              double *__restrict__ acc, double *__restrict__ vel, double *__restrict__ kin_part,
              int do_kick, double *__restrict__ ep_out, int *status)
{
    __shared__ double red[32];
    const int b = blockIdx.x;
    const int r = block_replica(reps, nrep, b);
    const RepDev &R = reps[r];
    const int i = R.p_off + (b - R.blk_off) * PBLK + threadIdx.x;
    double kin = 0.0;
    if (i < R.p_off + R.n) {
        const typename V4<T>::t ap = acc_pp[cell_slot[i]];
        double a[3] = {(double)ap.x, (double)ap.y, (double)ap.z};
        if (has_mesh) {
            const typename V4<T>::t e = acc_pm[brick_slot[i]];
            const double q = (double)e.w;
            const double E[3] = {(double)e.x, (double)e.y, (double)e.z};
#pragma unroll
            for (int d = 0; d < 3; ++d) a[d] = a[d] + q * E[d];
            if (ep_out) {
                ep_out[3 * i + 0] = E[0];
                ep_out[3 * i + 1] = E[1];
                ep_out[3 * i + 2] = E[2];
            }
        }
        bool finite = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double ad = R.af * a[d];
            finite = finite && isfinite(ad);
            acc[3 * i + d] = ad;
            if (do_kick) {
                const double v = kick(vel[3 * i + d], ad, R.dt);
                vel[3 * i + d] = v;
                kin += v * v;
            }
        }
        if (!finite) raise_status(status, ST_NONFINITE);
    }
    const double t = block_sum(kin, red);
    if (threadIdx.x == 0) kin_part[b] = t;
}

// Per replica: energies, temperature and the thermostat factor; one row of
// the energy ring; step counter advance. mode: 0 NVE, 1 thermostat, 2 force
// only (no kinetic terms). Single block.
__global__ void k_step_reduce(const RepDev *__restrict__ reps, int nrep, int nblk,
                              const double *__restrict__ kin_part, double *__restrict__ rep_out,
                              int mode, int *__restrict__ counters, double *__restrict__ ring,
                              int ring_cap, int recorded, int snap_interval, int snap_cap,
                              int *rebuild, int *status, StepSums sums, int *prune,
                              double *prune_count)
{
    // counters: [0] steps since the run started, [1] energy-ring position,
    // [2] step index of the run's first step (thermostat_p3m_ord6.py:15 tests
    // it <= 1999), [3] n(q,t) rows recorded, [4] snapshots taken, [5] the
    // snapshot slot this step writes (-1: none)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int it = counters[2] + counters[0];
    const int step = counters[1];
    for (int r = w; r < nrep; r += nw) {
        const RepDev &R = reps[r];
        if (sums.u_pp_part) {
            // k_reduce_pp and k_reduce_pm, in their order
            const int b0 = R.pp_blk_off, b1 = (r + 1 < nrep) ? reps[r + 1].pp_blk_off : sums.pp_nblk;
            double t = 0.0;
            for (int k = b0 + lane; k < b1; k += 32) t += sums.u_pp_part[k];
            t = warp_sum(t);
            double tm = 0.0;
            if (R.M > 0) {
                const int cb = R.wc_off, ce = (r + 1 < nrep) ? reps[r + 1].wc_off : sums.wc_total;
                const int pb = sums.wc_total + R.wp_off,
                          pe = sums.wc_total + ((r + 1 < nrep) ? reps[r + 1].wp_off : sums.wp_total);
                for (int k = cb + lane; k < ce; k += 32) tm += sums.u_pm_part[k];
                for (int k = pb + lane; k < pe; k += 32) tm += sums.u_pm_part[k];
                tm = warp_sum(tm);
            }
            if (lane == 0) {
                rep_out[8 * r + RO_UPP] = 0.5 * t;
                rep_out[8 * r + RO_UPM] = 0.5 * tm;
            }
        }
        const int b0 = R.blk_off, b1 = (r + 1 < nrep) ? reps[r + 1].blk_off : nblk;
        double s = 0.0;
        for (int k = b0 + lane; k < b1; k += 32) s += kin_part[k];
        s = warp_sum(s);
        if (lane == 0) {
            double *o = rep_out + 8 * r;
            const double u_self = -R.n * R.alpha / 1.7724538509055160273;
            const double U = R.uf * (o[RO_UPP] + o[RO_UPM] + u_self);
            const double K = R.kf * s;
            const double T = K / R.kf / (double)R.n;
            double fact = 1.0;
            if (mode == 1) {
                // thermostat_p3m_ord6.py:15-23
                fact = (it <= 1999) ? sqrt(R.t_desired / T)
                                    : sqrt((20.0 * R.t_desired / T - 1.0) / 20.0);
            }
            if (!isfinite(U)) raise_status(status, ST_NONFINITE);
            o[RO_USELF] = u_self;
            o[RO_U] = U;
            o[RO_K] = K;
            o[RO_T] = T;
            o[RO_FACT] = fact;
            if (ring && ring_cap > 0) {
                double *row = ring + ((long long)(step % ring_cap) * nrep + r) * 4;
                row[0] = U;
                row[1] = K;
                row[2] = T;
                row[3] = fact;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (mode != 2) {
            counters[0] += 1;
            counters[1] = step + 1;
            if (recorded) counters[3] += 1;
            // a snapshot after step `it` when (it + 1) % interval == 0, as the
            // reference writes its files (yukawa_MD_p3m_ord6.py:222)
            if (snap_interval > 0 && (it + 1) % snap_interval == 0) {
                counters[5] = counters[4] % snap_cap;
                counters[4] += 1;
            } else {
                counters[5] = -1;
            }
        }
    }
    // this step's lists are built (count them); the next drift decides again
    for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
        if (rebuild[r] && mode != 2) rep_out[8 * r + RO_REBUILDS] += 1.0;
        if (prune) {  // inner lists: count the builds that came without an outer rebuild
            if (prune[r] && !rebuild[r] && mode != 2) prune_count[r] += 1.0;
            prune[r] = 0;
        }
        rebuild[r] = 0;
    }
}

// The state after this step, [slot][particle][pos, vel, acc] (the rows of
// yukawa_MD_p3m_ord6.py:223), into the slot k_step_reduce chose; steps[slot]
// = the step index.
__global__ void k_snapshot(const double *__restrict__ pos, const double *__restrict__ vel,
                           const double *__restrict__ acc, int ntot,
                           const int *__restrict__ counters, double *__restrict__ snap,
                           int *__restrict__ steps)
{
    const int slot = counters[5];
    if (slot < 0) return;
    double *dst = snap + (long long)slot * ntot * 9;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            dst[9 * (long long)i + c] = pos[3 * (long long)i + c];
            dst[9 * (long long)i + 3 + c] = vel[3 * (long long)i + c];
            dst[9 * (long long)i + 6 + c] = acc[3 * (long long)i + c];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) steps[slot] = counters[2] + counters[0] - 1;
}

__global__ void k_set_flags(int *flag, int n, int value)
{
    for (int r = threadIdx.x; r < n; r += blockDim.x) flag[r] = value;
}

__global__ void k_set_counters(int *counters, int run_step, int ring_pos, int it0)
{
    if (run_step >= 0) counters[0] = run_step;
    if (ring_pos >= 0) {
        counters[1] = ring_pos;
        counters[3] = ring_pos;
    }
    counters[2] = it0;
}

// out[i] = scale (use_pp a_pp + use_pm Z E) in original particle order; ep_out
// (optional) receives E at the particle.
template <typename T>
__global__ void k_combine(const RepDev *__restrict__ reps, const int *__restrict__ prep,
                          const int *__restrict__ cell_slot, const int *__restrict__ brick_slot,
                          const typename V4<T>::t *__restrict__ acc_pp,
                          const typename V4<T>::t *__restrict__ acc_pm, int use_pp, int use_pm,
                          int scale_af, double *__restrict__ out, double *__restrict__ ep_out,
                          int ntot, int *status)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        double a[3] = {0.0, 0.0, 0.0};
        if (use_pp) {
            const typename V4<T>::t ap = acc_pp[cell_slot[i]];
            a[0] = (double)ap.x;
            a[1] = (double)ap.y;
            a[2] = (double)ap.z;
        }
        if (use_pm) {
            const typename V4<T>::t e = acc_pm[brick_slot[i]];
            const double q = (double)e.w;
            a[0] = a[0] + q * (double)e.x;
            a[1] = a[1] + q * (double)e.y;
            a[2] = a[2] + q * (double)e.z;
            if (ep_out) {
                ep_out[3 * i + 0] = (double)e.x;
                ep_out[3 * i + 1] = (double)e.y;
                ep_out[3 * i + 2] = (double)e.z;
            }
        }
        const double f = scale_af ? reps[prep[i]].af : 1.0;
        out[3 * i + 0] = scale_af ? f * a[0] : a[0];
        out[3 * i + 1] = scale_af ? f * a[1] : a[1];
        out[3 * i + 2] = scale_af ? f * a[2] : a[2];
        if (!(isfinite(a[0]) && isfinite(a[1]) && isfinite(a[2]))) raise_status(status, ST_NONFINITE);
    }
}

__global__ void k_scale_vel(const RepDev *__restrict__ reps, const int *__restrict__ prep,
                            const double *__restrict__ rep_out, double *__restrict__ vel, int ntot)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x) {
        const double f = rep_out[8 * prep[i] + RO_FACT];
        vel[3 * i + 0] *= f;
        vel[3 * i + 1] *= f;
        vel[3 * i + 2] *= f;
    }
}

// n(q,t) partial sums: per replica-aligned block of NQ_PPT * PBLK particles,
// for each wave number q_m = m 2 pi / L (m = qmult[iq]) and axis,
// sum_i exp(-i q x_i) (yukawa_MD_p3m_ord6.py:215-219). Each thread sums
// NQ_PPT particles, a warp its 32 threads' sums (in the bulk precision T: a
// warp's total holds 32 NQ_PPT terms), and the block its warps' totals in
// FP64. The phase is reduced in FP64
// as frac(m x / L) before the sine/cosine of the bulk precision T; when the
// multiples are 1, 2, ..., nq (`consecutive`), exp(-i m theta) follows from
// exp(-i theta) by complex multiplication instead.
constexpr int NQ_PPT = 4;

template <typename T>
__device__ __forceinline__ void sincospi_t(double two_t, T *s, T *c)
{
    if (sizeof(T) == 4) {
        float sf, cf;
        sincospif((float)two_t, &sf, &cf);
        *s = (T)sf;
        *c = (T)cf;
    } else {
        double sd, cd;
        sincospi(two_t, &sd, &cd);
        *s = (T)sd;
        *c = (T)cd;
    }
}

// Sum over the 32 lanes of a warp of eight values v[0..7] per lane, by
// recursive halving: at each of the first three levels a lane keeps half of
// its values, sends the other half to its partner (lane ^ 16, ^ 8, ^ 4) and
// adds the partner's copy of the half it keeps; two butterfly levels finish
// the one value left. Lane l returns the total of value (l >> 2) & 7. Nine
// shuffles for eight sums (five per value in a plain butterfly), in a fixed
// order.
template <typename T>
__device__ __forceinline__ T warp_sum8(const T (&v)[8])
{
    const int lane = threadIdx.x & 31;
    T a[4], b[2];
    const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const T send = h4 ? v[i] : v[i + 4];
        a[i] = (h4 ? v[i + 4] : v[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const T send = h3 ? a[i] : a[i + 2];
        b[i] = (h3 ? a[i + 2] : a[i]) + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const T send = h2 ? b[0] : b[1];
    T c = (h2 ? b[1] : b[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
    c += __shfl_xor_sync(0xffffffffu, c, 2);
    c += __shfl_xor_sync(0xffffffffu, c, 1);
    return c;
}

template <typename T, bool consecutive>
__global__ void __launch_bounds__(PBLK)
k_nqt_partial(const RepDev *__restrict__ reps, int nrep, const double *__restrict__ pos,
              const double *__restrict__ qmult, int nq, double *__restrict__ part)
{
    extern __shared__ double nsm[];  // [nwarps][nq*6]
    const int b = blockIdx.x;
    const int r = find_rep(b, nrep, [&](int k) { return reps[k].nq_blk_off; });
    const RepDev &R = reps[r];
    const int first = R.p_off + (b - R.nq_blk_off) * (PBLK * NQ_PPT);
    const int end = R.p_off + R.n;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double xl[NQ_PPT][3];
    bool have[NQ_PPT];
#pragma unroll
    for (int m = 0; m < NQ_PPT; ++m) {
        const int i = first + threadIdx.x + m * PBLK;
        have[m] = i < end;
#pragma unroll
        for (int d = 0; d < 3; ++d) xl[m][d] = have[m] ? pos[3 * i + d] * R.inv_L : 0.0;
    }
    // per-particle base rotation exp(-i 2 pi x/L) for the recurrence; a
    // missing particle rotates by 1 and is weighted by 0
    T c1[NQ_PPT][3], s1[NQ_PPT][3], cm[NQ_PPT][3], sm[NQ_PPT][3], wt[NQ_PPT];
#pragma unroll
    for (int m = 0; m < NQ_PPT; ++m) {
        wt[m] = have[m] ? (T)1 : (T)0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            T st = (T)0, ct = (T)1;
            if constexpr (consecutive) {
                const double t = xl[m][d] - floor(xl[m][d]);
                sincospi_t<T>(2.0 * t, &st, &ct);
            }
            c1[m][d] = ct;
            s1[m][d] = -st;
            cm[m][d] = (T)1;
            sm[m][d] = (T)0;
        }
    }
    for (int iq = 0; iq < nq; ++iq) {
        const double mq = consecutive ? 0.0 : qmult[iq];
        T acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = (T)0;
#pragma unroll
        for (int m = 0; m < NQ_PPT; ++m) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                T c, sn;
                if constexpr (consecutive) {
                    // exp(-i (k+1) theta) = exp(-i k theta) exp(-i theta)
                    const T nc = cm[m][d] * c1[m][d] - sm[m][d] * s1[m][d];
                    const T ns = cm[m][d] * s1[m][d] + sm[m][d] * c1[m][d];
                    cm[m][d] = nc;
                    sm[m][d] = ns;
                    c = nc;
                    sn = ns;
                } else {
                    double t = mq * xl[m][d];
                    t = t - floor(t);
                    T st, ct;
                    sincospi_t<T>(2.0 * t, &st, &ct);
                    c = ct;
                    sn = -st;
                }
                acc[2 * d + 0] += wt[m] * c;
                acc[2 * d + 1] += wt[m] * sn;
            }
        }
        // lane l holds the warp's total of value (l >> 2) & 7 (6, 7: padding)
        const T tot = warp_sum8<T>(acc);
        const int k = (lane >> 2) & 7;
        if ((lane & 3) == 0 && k < 6) nsm[w * nq * 6 + iq * 6 + k] = (double)tot;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nq * 6; k += blockDim.x) {
        double t = 0.0;
        for (int ww = 0; ww < nw; ++ww) t += nsm[ww * nq * 6 + k];
        part[(long long)b * nq * 6 + k] = t;
    }
}

// Per replica: sum the block partials into out[r][nq][3] complex (re, im).
// Block (r, c) sums values 32 c .. 32 c + 31 of replica r: warp w adds the
// partials of blocks b0 + w, b0 + w + 8, ... (lane = value), then the eight
// warp sums are added in warp order -- a fixed order, so the result does not
// depend on timing; a large replica's thousand partial blocks are summed by
// eight warps instead of one thread per value.
constexpr int NQR_WARPS = 8;

__global__ void __launch_bounds__(NQR_WARPS * 32)
k_nqt_reduce(const RepDev *__restrict__ reps, int nrep, int nblk,
             const double *__restrict__ part, int nq, double *__restrict__ out,
             const int *__restrict__ counters, int ring_cap)
{
    __shared__ double wsum[NQR_WARPS][32];
    const int r = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nv = nq * 6, k = blockIdx.y * 32 + lane;
    const RepDev &R = reps[r];
    const int b0 = R.nq_blk_off, b1 = (r + 1 < nrep) ? reps[r + 1].nq_blk_off : nblk;
    double s = 0.0;
    if (k < nv)
        for (int bb = b0 + w; bb < b1; bb += NQR_WARPS) s += part[(long long)bb * nv + k];
    wsum[w][lane] = s;
    __syncthreads();
    if (w == 0 && k < nv) {
        double t = 0.0;
        for (int j = 0; j < NQR_WARPS; ++j) t += wsum[j][lane];
        double *o = out;
        if (counters) {
            // ring layout [row][replica][nq][3][2]; this step's row
            const int step = counters[3] % ring_cap;
            o = out + (long long)step * nrep * nv;
        }
        o[(long long)r * nv + k] = t;
    }
}

// ---------------------------------------------------------------------------
// Optimal influence function (yukawa_gf_opt.py:5-98), FP64, fftshifted layout.
// ---------------------------------------------------------------------------
constexpr int GF_MAXA = 15;  // 2 * m_alias + 1 <= 15

__global__ void __launch_bounds__(256)
k_gf_opt(double kappa, double alpha, int p, int m, int M, double L, double *__restrict__ G_k,
         double *__restrict__ a_part)
{
    __shared__ double red[32];
    const double two_pi = 6.283185307179586477, four_pi = 12.566370614359172954;
    const double h = L / M;
    const int mid = (M % 2 == 0) ? M / 2 : (M - 1) / 2;
    const long long total = (long long)M * M * M;
    const double kappa_sq = kappa * kappa, a_sq = alpha * alpha;
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double acontrib = 0.0;
    if (e < total) {
        const int nx = (int)(e % M), ny = (int)((e / M) % M), nz = (int)(e / ((long long)M * M));
        const int sx = nx - mid, sy = ny - mid, sz = nz - mid;
        const double kx = two_pi * sx / L, ky = two_pi * sy / L, kz = two_pi * sz / L;
        const double k_sq = kx * kx + ky * ky + kz * kz;
        double g = 0.0;
        if (k_sq != 0.0) {
            double kmx[GF_MAXA], kmy[GF_MAXA], kmz[GF_MAXA];
            double ux[GF_MAXA], uy[GF_MAXA], uz[GF_MAXA];
            const int na = 2 * m + 1;
            for (int a = 0; a < na; ++a) {
                const int mm = a - m;
                kmx[a] = two_pi * (sx + mm * M) / L;
                kmy[a] = two_pi * (sy + mm * M) / L;
                kmz[a] = two_pi * (sz + mm * M) / L;
                ux[a] = (kmx[a] != 0.0) ? sin(0.5 * kmx[a] * h) / (0.5 * kmx[a] * h) : 1.0;
                uy[a] = (kmy[a] != 0.0) ? sin(0.5 * kmy[a] * h) / (0.5 * kmy[a] * h) : 1.0;
                uz[a] = (kmz[a] != 0.0) ? sin(0.5 * kmz[a] * h) / (0.5 * kmz[a] * h) : 1.0;
            }
            double U_k_sq = 0.0, U_G_k = 0.0;
            for (int az = 0; az < na; ++az)
                for (int ay = 0; ay < na; ++ay)
                    for (int ax = 0; ax < na; ++ax) {
                        const double k_M_sq =
                            kmx[ax] * kmx[ax] + kmy[ay] * kmy[ay] + kmz[az] * kmz[az];
                        double u = ux[ax] * uy[ay] * uz[az];
                        double up = 1.0;
                        for (int q = 0; q < p; ++q) up *= u;  // (Ux Uy Uz)^p
                        const double u2 = up * up;
                        const double gm = four_pi * exp(-0.25 * (kappa_sq + k_M_sq) / a_sq) /
                                          (kappa_sq + k_M_sq);
                        const double kdot = kx * kmx[ax] + ky * kmy[ay] + kz * kmz[az];
                        U_G_k += u2 * gm * kdot;
                        U_k_sq += u2;
                    }
            g = U_G_k / ((U_k_sq * U_k_sq) * k_sq);
            acontrib = U_G_k * U_G_k / ((U_k_sq * U_k_sq) * k_sq);
        }
        G_k[e] = g;
    }
    const double t = block_sum(acontrib, red);
    if (threadIdx.x == 0) a_part[blockIdx.x] = t;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int pgrid(int n) { int g = (n + 255) / 256; return g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g); }

void launch_kick_drift(const DevState &s, cudaStream_t st)
{
    const bool inner = s.prune_buf > 0.0;
    k_kick_drift<<<pgrid(s.ntot), 256, 0, st>>>(s.reps, s.prep, s.pos, s.vel, s.acc, s.pos_ref,
                                                s.ntot, s.brick_key, s.brick_count, s.has_mesh,
                                                s.rebuild, s.status, inner ? s.pos_pref : nullptr,
                                                s.prune);
}

void launch_set_flags(int *flag, int n, int value, cudaStream_t st)
{
    k_set_flags<<<1, 256, 0, st>>>(flag, n, value);
}

template <typename T>
void launch_kick_finish(const DevState &s, int do_kick, double *ep_out, cudaStream_t st)
{
    using T4 = typename V4<T>::t;
    k_kick_finish<T><<<s.nblk, PBLK, 0, st>>>(s.reps, s.nrep, s.cell_slot, s.brick_slot,
                                              (const T4 *)s.acc_pp, (const T4 *)s.acc_pm,
                                              s.has_mesh, s.acc, s.vel, s.kin_part, do_kick,
                                              ep_out, s.status);
}

void launch_step_reduce(const DevState &s, int mode, int *counters, double *ring, int ring_cap,
                        cudaStream_t st, int recorded, int snap_interval, int snap_cap,
                        const StepSums &sums)
{
    k_step_reduce<<<1, 1024, 0, st>>>(s.reps, s.nrep, s.nblk, s.kin_part, s.rep_out, mode,
                                      counters, ring, ring_cap, recorded, snap_interval, snap_cap,
                                      s.rebuild, s.status, sums,
                                      s.prune_buf > 0.0 ? s.prune : nullptr, s.prune_count);
}

void launch_snapshot(const DevState &s, const int *counters, double *snap, int *steps,
                     cudaStream_t st)
{
    k_snapshot<<<pgrid(s.ntot), 256, 0, st>>>(s.pos, s.vel, s.acc, s.ntot, counters, snap, steps);
}

void launch_set_counters(int *counters, int run_step, int ring_pos, int it0, cudaStream_t st)
{
    k_set_counters<<<1, 1, 0, st>>>(counters, run_step, ring_pos, it0);
}

template <typename T>
void launch_combine(const DevState &s, int use_pp, int use_pm, int scale_af, double *out,
                    double *ep_out, cudaStream_t st)
{
    using T4 = typename V4<T>::t;
    k_combine<T><<<pgrid(s.ntot), 256, 0, st>>>(s.reps, s.prep, s.cell_slot, s.brick_slot,
                                                (const T4 *)s.acc_pp, (const T4 *)s.acc_pm,
                                                use_pp, use_pm, scale_af, out, ep_out, s.ntot,
                                                s.status);
}

void launch_scale_vel(const DevState &s, cudaStream_t st)
{
    k_scale_vel<<<pgrid(s.ntot), 256, 0, st>>>(s.reps, s.prep, s.rep_out, s.vel, s.ntot);
}

template <typename T>
void launch_nqt(const DevState &s, const double *pos, const double *qmult, int nq, int consecutive,
                double *part, double *out, const int *counters, int ring_cap, cudaStream_t st)
{
    const size_t smem = (size_t)(PBLK / 32) * nq * 6 * sizeof(double);
    if (consecutive)
        k_nqt_partial<T, true><<<s.nq_nblk, PBLK, smem, st>>>(s.reps, s.nrep, pos, qmult, nq, part);
    else
        k_nqt_partial<T, false><<<s.nq_nblk, PBLK, smem, st>>>(s.reps, s.nrep, pos, qmult, nq, part);
    const dim3 rgrid(s.nrep, (nq * 6 + 31) / 32);
    k_nqt_reduce<<<rgrid, NQR_WARPS * 32, 0, st>>>(s.reps, s.nrep, s.nq_nblk, part, nq, out,
                                                   counters, ring_cap);
}

int nqt_particles_per_block() { return PBLK * NQ_PPT; }

template <typename T> void configure_integrate_kernels(int max_nq)
{
    const int smem = (int)((PBLK / 32) * max_nq * 6 * sizeof(double));
    cudaFuncSetAttribute(k_nqt_partial<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_nqt_partial<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

void launch_gf_opt(double kappa, double alpha, int p, int m_alias, int M, double L, double *G_k,
                   double *a_part, cudaStream_t st)
{
    const long long total = (long long)M * M * M;
    const int blocks = (int)((total + 255) / 256);
    k_gf_opt<<<blocks, 256, 0, st>>>(kappa, alpha, p, m_alias, M, L, G_k, a_part);
}

int gf_opt_blocks(int M) { return (int)(((long long)M * M * M + 255) / 256); }

#define P3M_INST(T)                                                                             \
    template void launch_kick_finish<T>(const DevState &, int, double *, cudaStream_t);          \
    template void launch_nqt<T>(const DevState &, const double *, const double *, int, int,      \
                                double *, double *, const int *, int, cudaStream_t);            \
    template void configure_integrate_kernels<T>(int);                                          \
    template void launch_combine<T>(const DevState &, int, int, int, double *, double *,         \
                                    cudaStream_t);
P3M_INST(float)
P3M_INST(double)

}  // namespace p3m
