// PPPM accuracy estimates and the parameter search they drive.
//
// The reference sets alpha, r_c and M by hand for each run
// (yukawa_MD_p3m_ord6.py:52-68, README.md:27); its only error measure is
// A_pm, the sum yukawa_gf_opt.py:96 returns. These estimate the RMS
// per-particle force error of each part for N unit charges at random
// positions, in the reference's reduced units (force per charge^2 / a_ws^2):
//
//  * PP (host, FP64): the force beyond r_c, integrated over a uniform
//    background (Kolafa & Perram, Mol. Sim. 9 (1992) 351) with the exact
//    Yukawa-Ewald short-range force of yukawa_pp.py:115-124:
//      dF_pp^2 = 4 pi n int_{r_c}^inf F(r)^2 r^2 dr,  n = N / L^3.
//  * PM (device, FP64): Hockney & Eastwood's Q functional at the optimal
//    influence function (Computer Simulation Using Particles, eq. 8-22):
//      dF_pm^2 = N / V^2 sum_{k != 0} [ sum_m |k_m|^2 G_m^2 - A(k) ],
//    G_m = 4 pi e^{-(kappa^2 + k_m^2)/(4 alpha^2)} / (kappa^2 + k_m^2), the
//    alias sum over |m_i| <= m_alias, and A(k) the term whose sum is the
//    reference's A_pm (yukawa_gf_opt.py:92-94).
#include <cmath>
#include <vector>

#include "p3m_kernels.h"

namespace p3m {

// ---- PP, host ---------------------------------------------------------------

// -d phi / dr of phi = (1/2r)[e^{k r} erfc(a r + b) + e^{-k r} erfc(a r - b)],
// b = k / (2 a): phi/r - (k/2r)[e^{kr} erfc(ar+b) - e^{-kr} erfc(ar-b)]
// + (2a / (r sqrt(pi))) e^{-a^2 r^2 - b^2}.
static double pair_force_sr(double r, double kappa, double alpha)
{
    const double b = kappa / (2.0 * alpha);
    const double ep = std::exp(kappa * r) * std::erfc(alpha * r + b);
    const double em = std::exp(-kappa * r) * std::erfc(alpha * r - b);
    const double phi = 0.5 * (ep + em) / r;
    return phi / r - 0.5 * kappa * (ep - em) / r +
           2.0 * alpha / (r * std::sqrt(M_PI)) * std::exp(-alpha * alpha * r * r - b * b);
}

// Simpson's rule on [r_c, sqrt(r_c^2 + 40/alpha^2)]: past the upper end the
// integrand has fallen by e^-80 against its value at r_c.
double pp_error_estimate(double n_particles, double box, double kappa, double alpha, double rc)
{
    const int n_int = 800;
    const double n = n_particles / (box * box * box);
    const double r_end = std::sqrt(rc * rc + 40.0 / (alpha * alpha));
    const double w = (r_end - rc) / n_int;
    double s = 0.0;
    for (int i = 0; i <= n_int; ++i) {
        const double r = rc + i * w;
        const double f = pair_force_sr(r, kappa, alpha);
        const double c = (i == 0 || i == n_int) ? 1.0 : ((i & 1) ? 4.0 : 2.0);
        s += c * f * f * r * r;
    }
    return std::sqrt(4.0 * M_PI * n * s * w / 3.0);
}

// Smallest r_c in (0, rc_max] with pp_error_estimate <= tol (bisection to a
// relative width of 1e-5; the estimate falls monotonically with r_c), or -1
// when even rc_max misses tol.
double pp_cutoff_for(double n_particles, double box, double kappa, double alpha, double tol,
                     double rc_max)
{
    if (pp_error_estimate(n_particles, box, kappa, alpha, rc_max) > tol) return -1.0;
    double lo = 0.0, hi = rc_max;
    while (hi - lo > 1e-5 * rc_max) {
        const double mid = 0.5 * (lo + hi);
        if (mid > 0.0 && pp_error_estimate(n_particles, box, kappa, alpha, mid) <= tol)
            hi = mid;
        else
            lo = mid;
    }
    return hi;
}

// ---- PM, device ---------------------------------------------------------------

constexpr int PME_MAXA = 2 * 7 + 1;

// One thread per first-zone k (index order of yukawa_gf_opt.py's loops:
// k = 2 pi (n - M/2) / L); per-block sums of sum_m |k_m|^2 G_m^2 - A(k) and of
// A(k), in block order on the host.
__global__ void __launch_bounds__(256)
k_pm_error(double kappa, double alpha, int p, int m, int M, double L, double *__restrict__ q_part,
           double *__restrict__ a_part)
{
    __shared__ double red[32];
    const double two_pi = 6.283185307179586477, four_pi = 12.566370614359172954;
    const double h = L / M;
    const int mid = M / 2;
    const long long total = (long long)M * M * M;
    const double kappa_sq = kappa * kappa, inv4a2 = 0.25 / (alpha * alpha);
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double qc = 0.0, ac = 0.0;
    if (e < total) {
        const int sx = (int)(e % M) - mid, sy = (int)((e / M) % M) - mid,
                  sz = (int)(e / ((long long)M * M)) - mid;
        const double kx = two_pi * sx / L, ky = two_pi * sy / L, kz = two_pi * sz / L;
        const double k_sq = kx * kx + ky * ky + kz * kz;
        if (k_sq != 0.0) {
            // per-axis factors: the Gaussian e^{-k_m^2/(4 alpha^2)} and U^{2p}
            // both separate over x, y, z
            double kmx[PME_MAXA], kmy[PME_MAXA], kmz[PME_MAXA];
            double gx[PME_MAXA], gy[PME_MAXA], gz[PME_MAXA];
            double ux[PME_MAXA], uy[PME_MAXA], uz[PME_MAXA];
            const int na = 2 * m + 1;
            for (int a = 0; a < na; ++a) {
                const int mm = a - m;
                kmx[a] = two_pi * (sx + mm * M) / L;
                kmy[a] = two_pi * (sy + mm * M) / L;
                kmz[a] = two_pi * (sz + mm * M) / L;
                gx[a] = exp(-kmx[a] * kmx[a] * inv4a2);
                gy[a] = exp(-kmy[a] * kmy[a] * inv4a2);
                gz[a] = exp(-kmz[a] * kmz[a] * inv4a2);
                double vx = (kmx[a] != 0.0) ? sin(0.5 * kmx[a] * h) / (0.5 * kmx[a] * h) : 1.0;
                double vy = (kmy[a] != 0.0) ? sin(0.5 * kmy[a] * h) / (0.5 * kmy[a] * h) : 1.0;
                double vz = (kmz[a] != 0.0) ? sin(0.5 * kmz[a] * h) / (0.5 * kmz[a] * h) : 1.0;
                double px = 1.0, py = 1.0, pz = 1.0;
                for (int q = 0; q < 2 * p; ++q) {
                    px *= vx;
                    py *= vy;
                    pz *= vz;
                }
                ux[a] = px;
                uy[a] = py;
                uz[a] = pz;
            }
            const double g0 = four_pi * exp(-kappa_sq * inv4a2);
            // Sums over the aliases m != 0 (primed) apart from the central
            // term: x = U_0^2, c = G_0 k^2. With S = x + S', T = x c + T',
            // R2 = c^2/k^2 + R2', the term R2 - T^2/(S^2 k^2) equals
            // R2' + (c S' - T')(c (2x + S') + T') / (S^2 k^2) exactly; the
            // second form has no cancellation between O(c^2/k^2) sums.
            double S1 = 0.0, T1 = 0.0, R1 = 0.0, x = 0.0, c = 0.0;
            for (int az = 0; az < na; ++az)
                for (int ay = 0; ay < na; ++ay) {
                    const double uyz = uy[ay] * uz[az], gyz = g0 * gy[ay] * gz[az];
                    const double kyz_sq = kmy[ay] * kmy[ay] + kmz[az] * kmz[az];
                    const double kdot_yz = ky * kmy[ay] + kz * kmz[az];
                    for (int ax = 0; ax < na; ++ax) {
                        const double k_M_sq = kmx[ax] * kmx[ax] + kyz_sq;
                        const double u2 = ux[ax] * uyz;
                        const double gm = gyz * gx[ax] / (kappa_sq + k_M_sq);
                        if (ax == m && ay == m && az == m) {
                            x = u2;
                            c = gm * k_sq;
                        } else {
                            S1 += u2;
                            T1 += u2 * gm * (kx * kmx[ax] + kdot_yz);
                            R1 += k_M_sq * gm * gm;
                        }
                    }
                }
            const double S = x + S1, T = x * c + T1;
            ac = T * T / ((S * S) * k_sq);
            qc = R1 + (c * S1 - T1) * (c * (2.0 * x + S1) + T1) / ((S * S) * k_sq);
        }
    }
    const double tq = block_sum(qc, red);
    __syncthreads();
    const double ta = block_sum(ac, red);
    if (threadIdx.x == 0) {
        q_part[blockIdx.x] = tq;
        a_part[blockIdx.x] = ta;
    }
}

int pm_error_blocks(int M) { return (int)(((long long)M * M * M + 255) / 256); }

void launch_pm_error(double kappa, double alpha, int p, int m_alias, int M, double L,
                     double *q_part, double *a_part, cudaStream_t st)
{
    k_pm_error<<<pm_error_blocks(M), 256, 0, st>>>(kappa, alpha, p, m_alias, M, L, q_part, a_part);
}

}  // namespace p3m
