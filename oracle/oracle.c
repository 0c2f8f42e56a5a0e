/*
 * CPU oracle for the P3M force step (TEST INFRASTRUCTURE ONLY).
 *
 * Plain-C restatement of the reference's FP64 arithmetic for the hot path of
 * xgdhar/MD-force-routines. Only the tests, the smoke check and the CPU-baseline
 * leg of the benchmark call into this file; the product path never does.
 *
 * Each function cites the reference lines whose algorithm it restates. Loop
 * order and the order of floating-point operations follow the reference so
 * that the results agree with its numba code to rounding (compiled with
 * -ffp-contract=off so no FMA contraction changes the rounding).
 *
 * Parity of this restatement is pinned by tests/golden/*.npz, which hold the
 * outputs of the reference's own numba functions run on identical inputs.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_EMPTY (-50)

/*
 * Linked-cell short-range Yukawa-Ewald sum.
 * Restates yukawa_pp.py:6-139 (particle_particle): cell grid floor(L/rc)
 * (:17-28), head/linked list built in particle order (:44-52), the 27-cell
 * periodic stencil with image shift (:54-94), the i<j test (:104), the cutoff
 * (:112), the energy term (:115) and the force f1+f2+f3 (:121-124) applied
 * with Newton's third law (:126-132). Z is ignored, as in the reference.
 *
 * pos: (n,3) row-major; acc: (n,3) output (zeroed here, as at :42).
 * Returns 0, or -1 when a particle lies outside the cell grid (the reference
 * would index out of bounds there).
 */
int oracle_pp(int n, const double *pos, double Lx, double Ly, double Lz,
              double kappa, double G, double rc, double *acc, double *U_out)
{
    int Lxd = (int)floor(Lx / rc), Lyd = (int)floor(Ly / rc), Lzd = (int)floor(Lz / rc);
    double rc_x = Lx / Lxd, rc_y = Ly / Lyd, rc_z = Lz / Lzd;
    int ncell = Lxd * Lyd * Lzd;
    int *head = (int *)malloc(sizeof(int) * (size_t)ncell);
    int *ls = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    double rshift[3];
    double U = 0.0;
    const double sqrt_pi = sqrt(M_PI);
    int rc_status = 0;

    for (int c = 0; c < ncell; ++c) head[c] = ORACLE_EMPTY;
    memset(acc, 0, sizeof(double) * 3 * (size_t)n);

    for (int i = 0; i < n; ++i) {
        int cx = (int)floor(pos[3 * i + 0] / rc_x);
        int cy = (int)floor(pos[3 * i + 1] / rc_y);
        int cz = (int)floor(pos[3 * i + 2] / rc_z);
        if (cx < 0 || cy < 0 || cz < 0 || cx >= Lxd || cy >= Lyd || cz >= Lzd) {
            rc_status = -1;
            goto done;
        }
        int c = cx + cy * Lxd + cz * Lxd * Lyd;
        ls[i] = head[c];
        head[c] = i;
    }

    for (int cx = 0; cx < Lxd; ++cx)
    for (int cy = 0; cy < Lyd; ++cy)
    for (int cz = 0; cz < Lzd; ++cz) {
        int c = cx + cy * Lxd + cz * Lxd * Lyd;
        for (int czn = cz - 1; czn < cz + 2; ++czn)
        for (int cyn = cy - 1; cyn < cy + 2; ++cyn)
        for (int cxn = cx - 1; cxn < cx + 2; ++cxn) {
            int sx, sy, sz;
            if (cxn < 0) { sx = Lxd; rshift[0] = -Lx; }
            else if (cxn >= Lxd) { sx = -Lxd; rshift[0] = Lx; }
            else { sx = 0; rshift[0] = 0.0; }
            if (cyn < 0) { sy = Lyd; rshift[1] = -Ly; }
            else if (cyn >= Lyd) { sy = -Lyd; rshift[1] = Ly; }
            else { sy = 0; rshift[1] = 0.0; }
            if (czn < 0) { sz = Lzd; rshift[2] = -Lz; }
            else if (czn >= Lzd) { sz = -Lzd; rshift[2] = Lz; }
            else { sz = 0; rshift[2] = 0.0; }
            int cN = (cxn + sx) + (cyn + sy) * Lxd + (czn + sz) * Lxd * Lyd;

            for (int i = head[c]; i != ORACLE_EMPTY; i = ls[i]) {
                for (int j = head[cN]; j != ORACLE_EMPTY; j = ls[j]) {
                    if (!(i < j)) continue;
                    double dx = pos[3 * i + 0] - (pos[3 * j + 0] + rshift[0]);
                    double dy = pos[3 * i + 1] - (pos[3 * j + 1] + rshift[1]);
                    double dz = pos[3 * i + 2] - (pos[3 * j + 2] + rshift[2]);
                    double r = sqrt(dx * dx + dy * dy + dz * dz);
                    if (r < rc) {
                        double ekp = exp(kappa * r), ekm = exp(-kappa * r);
                        double up = G * r + 0.5 * kappa / G, um = G * r - 0.5 * kappa / G;
                        double ecp = erfc(up), ecm = erfc(um);
                        U = U + (0.5 / r) * (ekp * ecp + ekm * ecm);
                        double f1 = (0.5 / (r * r)) * ekp * ecp * (1 - kappa * r);
                        double f2 = (0.5 / (r * r)) * ekm * ecm * (1 + kappa * r);
                        double f3 = (G / sqrt_pi / r) * (exp(-(up * up)) * ekp + exp(-(um * um)) * ekm);
                        double fr = f1 + f2 + f3;
                        acc[3 * i + 0] = acc[3 * i + 0] + fr * dx / r;
                        acc[3 * i + 1] = acc[3 * i + 1] + fr * dy / r;
                        acc[3 * i + 2] = acc[3 * i + 2] + fr * dz / r;
                        acc[3 * j + 0] = acc[3 * j + 0] - fr * dx / r;
                        acc[3 * j + 1] = acc[3 * j + 1] - fr * dy / r;
                        acc[3 * j + 2] = acc[3 * j + 2] - fr * dz / r;
                    }
                }
            }
        }
    }
done:
    *U_out = U;
    free(head);
    free(ls);
    return rc_status;
}

/*
 * Order-6 B-spline weights at offset x in [-0.5, 0.5) from the node centre.
 * The six polynomials are those of yukawa_pm_ord6.py:29-34 (the same set is
 * used for y and z at :36-48 and in the gather at :41-60 of its second copy).
 */
static void w6(double x, double *w)
{
    double x2 = x * x, x3 = x2 * x, x4 = x3 * x, x5 = x4 * x;
    w[0] = (1 - 10 * x + 40 * x2 - 80 * x3 + 80 * x4 - 32 * x5) / 3840;
    w[1] = (237 - 750 * x + 840 * x2 - 240 * x3 - 240 * x4 + 160 * x5) / 3840;
    w[2] = (841 - 770 * x - 440 * x2 + 560 * x3 + 80 * x4 - 160 * x5) / 1920;
    w[3] = (841 + 770 * x - 440 * x2 - 560 * x3 + 80 * x4 + 160 * x5) / 1920;
    w[4] = (237 + 750 * x + 840 * x2 + 240 * x3 - 240 * x4 - 160 * x5) / 3840;
    w[5] = (1 + 10 * x + 40 * x2 + 80 * x3 + 80 * x4 + 32 * x5) / 3840;
}

/* Single periodic wrap of a stencil index, as at yukawa_pm_ord6.py:56-61. */
static inline int wrap1(int i, int M)
{
    if (i < 0) return i + M;
    if (i > M - 1) return i - M;
    return i;
}

/* Base index and node offset along one axis, yukawa_pm_ord6.py:17-27. */
static inline void base6(double p, double h, int *ix, double *x)
{
    *ix = (int)floor(p / h);
    double t = p - (*ix + 0.5) * h;
    *x = t / h;
}

/*
 * Charge assignment, order 6. Restates charge_assgn_6_numba,
 * yukawa_pm_ord6.py:6-95: per particle the base index floor(x/h), the offset
 * x/h - (ix+0.5), and the scatter of Z*wz*wy*wx onto nodes ix..ix+5 (mod M)
 * of rho[z][y][x] (:52-93). rho is zeroed first (:13).
 */
int oracle_assign6(int n, const double *pos, const double *Z, int Mx, int My, int Mz,
                   double hx, double hy, double hz, double *rho)
{
    memset(rho, 0, sizeof(double) * (size_t)Mx * My * Mz);
    for (int p = 0; p < n; ++p) {
        int ix, iy, iz;
        double x, y, z, wx[6], wy[6], wz[6];
        base6(pos[3 * p + 0], hx, &ix, &x);
        base6(pos[3 * p + 1], hy, &iy, &y);
        base6(pos[3 * p + 2], hz, &iz, &z);
        if (ix < -Mx || iy < -My || iz < -Mz || ix + 5 > 2 * Mx - 1 ||
            iy + 5 > 2 * My - 1 || iz + 5 > 2 * Mz - 1)
            return -1;
        w6(x, wx); w6(y, wy); w6(z, wz);
        for (int g = 0; g < 6; ++g) {
            int rg = wrap1(iz + g, Mz);
            for (int i = 0; i < 6; ++i) {
                int ri = wrap1(iy + i, My);
                for (int j = 0; j < 6; ++j) {
                    int rj = wrap1(ix + j, Mx);
                    size_t k = ((size_t)rg * My + ri) * Mx + rj;
                    rho[k] = rho[k] + Z[p] * wz[g] * wy[i] * wx[j];
                }
            }
        }
    }
    return 0;
}

/*
 * Field gather, order 6. Restates field_assgn_6_numba,
 * yukawa_pm_ord6.py:213-312: the same weights and stencil as the assignment,
 * accumulation of E_x/E_y/E_z at the particle (:298-300) and acc = Z*E
 * (:308-310). Ep may be NULL; otherwise it receives (3,n) field values.
 */
int oracle_gather6(int n, const double *pos, const double *Z, int Mx, int My, int Mz,
                   double hx, double hy, double hz, const double *Ex, const double *Ey,
                   const double *Ez, double *acc, double *Ep)
{
    for (int p = 0; p < n; ++p) {
        int ix, iy, iz;
        double x, y, z, wx[6], wy[6], wz[6];
        base6(pos[3 * p + 0], hx, &ix, &x);
        base6(pos[3 * p + 1], hy, &iy, &y);
        base6(pos[3 * p + 2], hz, &iz, &z);
        if (ix < -Mx || iy < -My || iz < -Mz || ix + 5 > 2 * Mx - 1 ||
            iy + 5 > 2 * My - 1 || iz + 5 > 2 * Mz - 1)
            return -1;
        w6(x, wx); w6(y, wy); w6(z, wz);
        double ex = 0.0, ey = 0.0, ez = 0.0;
        for (int g = 0; g < 6; ++g) {
            int rg = wrap1(iz + g, Mz);
            for (int i = 0; i < 6; ++i) {
                int ri = wrap1(iy + i, My);
                for (int j = 0; j < 6; ++j) {
                    int rj = wrap1(ix + j, Mx);
                    size_t k = ((size_t)rg * My + ri) * Mx + rj;
                    ex = ex + Ex[k] * wz[g] * wy[i] * wx[j];
                    ey = ey + Ey[k] * wz[g] * wy[i] * wx[j];
                    ez = ez + Ez[k] * wz[g] * wy[i] * wx[j];
                }
            }
        }
        acc[3 * p + 0] = Z[p] * ex;
        acc[3 * p + 1] = Z[p] * ey;
        acc[3 * p + 2] = Z[p] * ez;
        if (Ep) { Ep[p] = ex; Ep[n + p] = ey; Ep[2 * n + p] = ez; }
    }
    return 0;
}

/*
 * Optimal influence function. Restates gf_opt, yukawa_gf_opt.py:5-98: for
 * every mesh wave vector k != 0 of the fftshifted layout (index n <-> k =
 * 2*pi*(n - M/2)/L, :12-33) the alias sum over m in [-m_max, m_max]^3 of
 * U^2(k_M) G_Yuk(k_M) (k . k_M) divided by (sum U^2)^2 k^2 (:56-94), with
 * U = prod sinc(k_M h/2)^p (:68-84) and G_Yuk = 4 pi exp(-(kappa^2+k_M^2)/(4
 * alpha^2)) / (kappa^2 + k_M^2) (:86). Also accumulates A_pm (:96).
 * G_k is (Mz,My,Mx) row-major.
 */
struct gf_setup {
    double kappa_sq, Gew_sq, hx, hy, hz, Lx, Ly, Lz;
    int p, mx_max, my_max, mz_max, Mx, My, Mz, nx_mid, ny_mid, nz_mid;
};

/* G_k at fftshifted index (nz, ny, nx) (0 at k = 0); *A_term receives the
 * point's contribution to A_pm. */
static double gf_point(const struct gf_setup *g, int nz, int ny, int nx, double *A_term)
{
    const double two_pi = 2 * M_PI, four_pi = 4 * M_PI;
    int nz_sh = nz - g->nz_mid, ny_sh = ny - g->ny_mid, nx_sh = nx - g->nx_mid;
    double kz = two_pi * nz_sh / g->Lz;
    double ky = two_pi * ny_sh / g->Ly;
    double kx = two_pi * nx_sh / g->Lx;
    double k_sq = kx * kx + ky * ky + kz * kz;
    *A_term = 0.0;
    if (k_sq == 0.0) return 0.0;
    double U_k_sq = 0.0, U_G_k = 0.0;
    for (int mz = -g->mz_max; mz < g->mz_max + 1; ++mz)
    for (int my = -g->my_max; my < g->my_max + 1; ++my)
    for (int mx = -g->mx_max; mx < g->mx_max + 1; ++mx) {
        double kx_M = two_pi * (nx_sh + mx * g->Mx) / g->Lx;
        double ky_M = two_pi * (ny_sh + my * g->My) / g->Ly;
        double kz_M = two_pi * (nz_sh + mz * g->Mz) / g->Lz;
        double k_M_sq = kx_M * kx_M + ky_M * ky_M + kz_M * kz_M;
        double Ux = (kx_M != 0.0) ? sin(0.5 * kx_M * g->hx) / (0.5 * kx_M * g->hx) : 1.0;
        double Uy = (ky_M != 0.0) ? sin(0.5 * ky_M * g->hy) / (0.5 * ky_M * g->hy) : 1.0;
        double Uz = (kz_M != 0.0) ? sin(0.5 * kz_M * g->hz) / (0.5 * kz_M * g->hz) : 1.0;
        double U_k_M = pow(Ux * Uy * Uz, g->p);
        double U_k_M_sq = U_k_M * U_k_M;
        double G_k_M = four_pi * exp(-0.25 * (g->kappa_sq + k_M_sq) / g->Gew_sq) /
                       (g->kappa_sq + k_M_sq);
        double k_dot_k_M = kx * kx_M + ky * ky_M + kz * kz_M;
        U_G_k += (U_k_M_sq * G_k_M * k_dot_k_M);
        U_k_sq += U_k_M_sq;
    }
    *A_term = U_G_k * U_G_k / ((U_k_sq * U_k_sq) * k_sq);
    return U_G_k / ((U_k_sq * U_k_sq) * k_sq);
}

static struct gf_setup gf_make(double kappa, double Gew, int p, int mx_max, int my_max,
                               int mz_max, int Mx, int My, int Mz, double hx, double hy,
                               double hz, double Lx, double Ly, double Lz)
{
    struct gf_setup g;
    g.kappa_sq = kappa * kappa;
    g.Gew_sq = Gew * Gew;
    g.hx = hx; g.hy = hy; g.hz = hz;
    g.Lx = Lx; g.Ly = Ly; g.Lz = Lz;
    g.p = p;
    g.mx_max = mx_max; g.my_max = my_max; g.mz_max = mz_max;
    g.Mx = Mx; g.My = My; g.Mz = Mz;
    g.nz_mid = (Mz % 2 == 0) ? Mz / 2 : (Mz - 1) / 2;
    g.ny_mid = (My % 2 == 0) ? My / 2 : (My - 1) / 2;
    g.nx_mid = (Mx % 2 == 0) ? Mx / 2 : (Mx - 1) / 2;
    return g;
}

void oracle_gf_opt(double kappa, double Gew, int p, int mx_max, int my_max, int mz_max,
                   int Mx, int My, int Mz, double hx, double hy, double hz,
                   double Lx, double Ly, double Lz, double *G_k, double *A_pm_out)
{
    struct gf_setup g = gf_make(kappa, Gew, p, mx_max, my_max, mz_max, Mx, My, Mz, hx, hy, hz,
                                Lx, Ly, Lz);
    double A_pm = 0.0;
    for (int nz = 0; nz < Mz; ++nz)
        for (int ny = 0; ny < My; ++ny)
            for (int nx = 0; nx < Mx; ++nx) {
                double a;
                G_k[((size_t)nz * My + ny) * Mx + nx] = gf_point(&g, nz, ny, nx, &a);
                A_pm = A_pm + a;
            }
    *A_pm_out = A_pm;
}

/* The same influence function at n chosen points only (idx: n triples nz, ny,
 * nx of the fftshifted layout), for meshes whose full alias sum takes the
 * CPU minutes (256^3: about 5.8e9 alias terms). */
void oracle_gf_opt_points(double kappa, double Gew, int p, int m_max, int M, double h, double L,
                          int n, const int *idx, double *G_out)
{
    struct gf_setup g = gf_make(kappa, Gew, p, m_max, m_max, m_max, M, M, M, h, h, h, L, L, L);
    for (int i = 0; i < n; ++i) {
        double a;
        G_out[i] = gf_point(&g, idx[3 * i], idx[3 * i + 1], idx[3 * i + 2], &a);
    }
}
