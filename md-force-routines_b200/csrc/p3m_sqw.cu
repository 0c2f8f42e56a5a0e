// Dynamic structure factor S(q, omega) from recorded n(q,t) series.
//
// Computes what s_of_q_w.py:3-20 computes for each series (time FFT of one
// axis' n(q,t), S = |dt FFT|^2 / (N T) with T = Nt dt) and what
// s_of_q_w_avg.py:5-20 and s_of_q_w_script.py:37 do with the result (mean over
// the three axes, then over runs). One CTA per (replica, q column) transforms
// the three axis series one after another in shared memory, in FP64: a
// radix-2 decimation-in-frequency pass (natural order in, bit-reversed out)
// for power-of-two lengths; other lengths go through Bluestein's chirp-z
// transform (a_n = x_n conj(c_n), c_n = exp(i pi n^2 / N); X_k = conj(c_k)
// (a (*) c)_k by a length-P convolution, P >= 2N - 1 a power of two) with the
// chirp's spectrum, in bit-reversed order, supplied by the host.
#include "p3m_kernels.h"

namespace p3m {

__device__ __forceinline__ double2 cmul2(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ int brev_n(int n, int logP) { return (int)(__brev((unsigned)n) >> (32 - logP)); }

// natural order in, bit-reversed order out; exp(-2 pi i k / 2h) twiddles
__device__ void fft_dif(double2 *x, int logP, bool inverse)
{
    const int P = 1 << logP;
    for (int s = logP - 1; s >= 0; --s) {
        const int half = 1 << s;
        for (int b = threadIdx.x; b < (P >> 1); b += blockDim.x) {
            const int k = b & (half - 1);
            const int i0 = ((b >> s) << (s + 1)) + k, i1 = i0 + half;
            double sn, cs;
            sincospi((double)k / half, &sn, &cs);
            const double2 w = make_double2(cs, inverse ? sn : -sn);
            const double2 a = x[i0], c = x[i1];
            x[i0] = make_double2(a.x + c.x, a.y + c.y);
            x[i1] = cmul2(make_double2(a.x - c.x, a.y - c.y), w);
        }
        __syncthreads();
    }
}

// bit-reversed order in, natural order out
__device__ void fft_dit(double2 *x, int logP, bool inverse)
{
    const int P = 1 << logP;
    for (int s = 0; s < logP; ++s) {
        const int half = 1 << s;
        for (int b = threadIdx.x; b < (P >> 1); b += blockDim.x) {
            const int k = b & (half - 1);
            const int i0 = ((b >> s) << (s + 1)) + k, i1 = i0 + half;
            double sn, cs;
            sincospi((double)k / half, &sn, &cs);
            const double2 w = make_double2(cs, inverse ? sn : -sn);
            const double2 a = x[i0], c = cmul2(w, x[i1]);
            x[i0] = make_double2(a.x + c.x, a.y + c.y);
            x[i1] = make_double2(a.x - c.x, a.y - c.y);
        }
        __syncthreads();
    }
}

// Series (r, col, ax) element t of replica (or run) r lives at
// src[row(t) * row_stride + r * rep_stride + col * 3 + ax] (complex elements),
// row(t) = (row0 + t) % cap. Block (c, y) handles replica r = r0 + y. With
// per_axis = 0, out[(r * ncols + c) * nt + k] receives the mean over axes of
// |dt X_k|^2 / (N_r T); with per_axis = 1, out[((r * ncols + c) * 3 + ax) *
// nt + k] receives each axis' value. T = nt dt. The transform works in
// shared memory, or, when gscratch is not NULL, in the block's own P-point
// slice of gscratch (long series; the slice stays in L2).
__global__ void k_sqw(const double2 *__restrict__ src, long long row_stride, long long rep_stride,
                      int cap, int row0, int r0, int col0, int col_stride, int ncols, int nt,
                      int logP, int bluestein, const double2 *__restrict__ chirp_fft_br,
                      const double *__restrict__ nrep_n, double dt, int per_axis,
                      double2 *gscratch, double *__restrict__ out_rep)
{
    extern __shared__ double2 smem_sqw[];
    const int c = blockIdx.x, r = r0 + blockIdx.y;
    const int col = col0 + c * col_stride;
    const int P = 1 << logP;
    double2 *xs = gscratch ? gscratch + ((long long)blockIdx.y * gridDim.x + c) * P : smem_sqw;
    const double T = nt * dt;
    const double norm = dt * dt / (nrep_n[r] * T) / (per_axis ? 1.0 : 3.0);
    double *o0 = out_rep + ((long long)r * ncols + c) * nt * (per_axis ? 3 : 1);
    for (int k = threadIdx.x; k < nt * (per_axis ? 3 : 1); k += blockDim.x) o0[k] = 0.0;
    for (int ax = 0; ax < 3; ++ax) {
        double *o = per_axis ? o0 + (long long)ax * nt : o0;
        __syncthreads();
        for (int n = threadIdx.x; n < P; n += blockDim.x) {
            double2 v = make_double2(0.0, 0.0);
            if (n < nt) {
                const int row = (row0 + n) % cap;
                v = src[row * row_stride + r * rep_stride + col * 3 + ax];
                if (bluestein) {
                    // a_n = x_n conj(c_n), c_n = exp(i pi (n^2 mod 2N) / N)
                    const long long m = ((long long)n * n) % (2LL * nt);
                    double sn, cs;
                    sincospi((double)m / nt, &sn, &cs);
                    v = cmul2(v, make_double2(cs, -sn));
                }
            }
            xs[n] = v;
        }
        __syncthreads();
        fft_dif(xs, logP, false);  // bit-reversed spectrum
        if (bluestein) {
            for (int j = threadIdx.x; j < P; j += blockDim.x) xs[j] = cmul2(xs[j], chirp_fft_br[j]);
            __syncthreads();
            fft_dit(xs, logP, true);  // natural: P (a (*) c)
            for (int k = threadIdx.x; k < nt; k += blockDim.x) {
                const long long m = ((long long)k * k) % (2LL * nt);
                double sn, cs;
                sincospi((double)m / nt, &sn, &cs);
                const double2 X = cmul2(xs[k], make_double2(cs / P, -sn / P));
                o[k] += norm * (X.x * X.x + X.y * X.y);
            }
        } else {
            for (int k = threadIdx.x; k < nt; k += blockDim.x) {
                const double2 X = xs[brev_n(k, logP)];
                o[k] += norm * (X.x * X.x + X.y * X.y);
            }
        }
    }
}

// out[c][k] = mean over replicas of out_rep[r][c][k]
__global__ void k_sqw_mean(const double *__restrict__ out_rep, int nrep, long long n,
                           double *__restrict__ out)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int r = 0; r < nrep; ++r) s += out_rep[(long long)r * n + e];
        out[e] = s / nrep;
    }
}

int sqw_max_points() { return 1 << 21; }
int sqw_smem_points() { return 8192; }

void launch_sqw(const SqwArgs &a, double2 *gscratch, cudaStream_t st)
{
    const bool in_smem = (1 << a.logP) <= sqw_smem_points();
    const size_t smem = in_smem ? ((size_t)1 << a.logP) * sizeof(double2) : 0;
    if (in_smem) cudaFuncSetAttribute(k_sqw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid(a.ncols, a.nrep_launch);
    k_sqw<<<grid, 512, smem, st>>>(a.src, a.row_stride, a.rep_stride, a.cap, a.row0, a.r0, a.col0,
                                   a.col_stride, a.ncols, a.nt, a.logP, a.bluestein, a.chirp_fft_br,
                                   a.nrep_n, a.dt, a.per_axis, in_smem ? nullptr : gscratch,
                                   a.out_rep);
}

void launch_sqw_mean(const double *out_rep, int nrep, long long n, double *out, cudaStream_t st)
{
    const long long nb = (n + 255) / 256;
    k_sqw_mean<<<(int)(nb < 1184 ? nb : 1184), 256, 0, st>>>(out_rep, nrep, n, out);
}

}  // namespace p3m
