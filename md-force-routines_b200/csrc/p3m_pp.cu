// Short-range (PP) Yukawa-Ewald forces over Verlet neighbour lists.
//
// Computes what yukawa_pp.py:6-139 computes: for every pair closer than r_c
// (minimum image; the reference finds them through a 27-cell periodic
// stencil, :54-94)
//   phi(r) = (1/2r) [e^{kr} erfc(ar + k/2a) + e^{-kr} erfc(ar - k/2a)]   (:115)
//   F(r)   = f1 + f2 + f3                                               (:121-124)
// The energy is sum_{i<j} phi. Every particle sums over all its neighbours
// itself (full list), so each thread owns its particle's force: no atomics,
// and the summation order is fixed by the list.
//
// Positions enter as integer fixed-point coordinates, q = frac(x/L) 2^B
// (B = 32 on the FP32 path, 64 on the FP64 path). The difference of two
// coordinates is exact, and its two's-complement wrap-around is the minimum
// image, so no periodic shifts are needed anywhere; converting the (small)
// difference to floating point rounds it once, relative to dx itself.
//
// Lists are rebuilt only when some particle has moved more than skin/2 since
// the last rebuild (the check is fused into the drift kernel); the rebuild
// kernels run in every step's launch sequence and return at once otherwise.
// A list holds every pair closer than rc + skin at rebuild time, so it holds
// every pair closer than rc until the next rebuild.
//
// Inner lists (FP32, prune buffer b > 0): the entries of a particle's Verlet
// list closer than rc + b, built inside the pair kernel whenever some
// particle of the replica has moved more than b/2 since their last build (or
// the Verlet lists were rebuilt). A pair missing from an inner list was
// either farther than rc + b at its build or missing from the Verlet list, so
// it cannot come within rc before one of the two checks fires.
//
// Pair terms: the FP64 path evaluates the reference's formula directly,
// written with the shared Gaussian factor
//   e^{+-kr} erfc(u+-) = erfcx(u+-) exp(-(a^2 r^2 + k^2/4a^2)),  u+- = ar +- k/2a,
// using CUDA's exp and erfcx. The FP32 path interpolates psi(r) = phi(r) r
// (finite at r = 0), tabulated on [0, rc] from FP64 values computed on the
// host, cubic per interval, and takes the force from the same cubic:
//   g(r) = F(r) r^2 = -r^2 d(psi/r)/dr = psi - r psi',
// F/r = g/r^3 and phi = psi/r -- one table read per pair, and a force that is
// exactly minus the gradient of the interpolated potential.
#include "p3m_kernels.h"

namespace p3m {

// ---------------------------------------------------------------------------
// coordinates
// ---------------------------------------------------------------------------
template <typename T> struct Coord;
template <> struct Coord<float> {
    using Q = uint4;
    using U = unsigned int;
    using I = int;
    static constexpr double scale = 4294967296.0;  // 2^32
    __device__ static U q(double t) { return __double2uint_rz(t * scale); }
};
template <> struct Coord<double> {
    using Q = ulonglong4;
    using U = unsigned long long;
    using I = long long;
    static constexpr double scale = 18446744073709551616.0;  // 2^64
    __device__ static U q(double t) { return __double2ull_rz(t * scale); }
};

// frac(x / L) in [0, 1)
__device__ __forceinline__ double unit_coord(double x, double inv_L)
{
    double t = x * inv_L;
    t -= floor(t);
    return t < 1.0 ? t : 0.0;
}

// Sorted-order integer coordinates, every step: xq[s] = q(pos[cell_perm[s]]);
// .w holds the replica index.
template <typename T>
__global__ void k_quantize(const RepDev *__restrict__ reps, const int *__restrict__ prep,
                           const int *__restrict__ cell_perm, const double *__restrict__ pos,
                           typename Coord<T>::Q *__restrict__ xq, int ntot)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ntot; s += gridDim.x * blockDim.x) {
        const int i = cell_perm[s];
        const int r = prep[i];
        const double il = reps[r].inv_L;
        typename Coord<T>::Q q;
        q.x = Coord<T>::q(unit_coord(pos[3 * i + 0], il));
        q.y = Coord<T>::q(unit_coord(pos[3 * i + 1], il));
        q.z = Coord<T>::q(unit_coord(pos[3 * i + 2], il));
        q.w = r;
        xq[s] = q;
    }
}

// dx of two coordinates (minimum image) in units of L / 2^B
template <typename T>
__device__ __forceinline__ typename Coord<T>::I qdiff(typename Coord<T>::U a, typename Coord<T>::U b)
{
    return (typename Coord<T>::I)(a - b);
}

// The list layout (list_index for the writer; list_lane_at, list_pass_at,
// list_block and list_chunk for the readers) is in p3m_list_layout.h.

// ---------------------------------------------------------------------------
// list build (rebuild steps only)
// ---------------------------------------------------------------------------
constexpr int LB_THREADS = 256;
constexpr int LB_TPI = 16;                    // lanes per particle
constexpr int LB_PPB = LB_THREADS / LB_TPI;   // particles per pass
constexpr int LB_HC = 256;                    // home particles per chunk
constexpr int LB_SCAP = 1024;                 // candidates staged per window (16 KB)
static_assert(cell_stencil(CELL_DIV_MAX) <= LB_THREADS, "one thread per stencil cell");
static_assert(LB_TPI >= PP_LIST_PAD, "one pad entry per lane at most");

// One CTA per cell of the replicas rebuilding this step (the list k_scan
// wrote); cells are (rc + skin)/D wide (about 10 particles at D = 2 and unit
// density 3/(4 pi), 80 at D = 1). The (2D+1)^3 neighbour cells'
// coordinates are staged in shared memory in the fixed stencil order (x
// fastest, offsets -D .. D), a window of LB_SCAP candidates at a time, as
// FP32 offsets from the home cell's centre: the wrap-around integer
// difference, exact, then one rounding. A home particle lies within half a
// cell of the centre and a candidate in range within rc + skin <= D cells of
// it, so both offsets are minimum images (at most (D + 1/2) L / nc <= L/2,
// nc >= 3 D) and their difference is the pair's separation; a test is three
// subtractions and the squared length, against a cutoff with a 1e-5
// relative margin over the rounding, so the list holds every pair within
// rc + skin. The LB_TPI lanes of a particle test LB_TPI consecutive candidates per round,
// and a warp ballot gives each candidate in range its place: the list holds
// the in-range candidates in stencil order, as a scan by one thread would,
// then the particle's own index up to a whole block of PP_LIST_PAD entries.
template <typename T, int D, int LT>
__global__ void __launch_bounds__(LB_THREADS)
k_build_lists(const RepDev *__restrict__ reps, int nrep, const int *__restrict__ cell_start,
              const typename Coord<T>::Q *__restrict__ xq, int *__restrict__ nnb,
              int *__restrict__ nlist, int maxnb, const int *__restrict__ rb_list, int nrep_all,
              int *status)
{
    constexpr int lt = LT;  // the list layout of the pair kernel's TPI = 2^LT
    using Q = typename Coord<T>::Q;
    using U = typename Coord<T>::U;
    constexpr int SCAP = LB_SCAP;
    constexpr int CELL_SPAN = 2 * D + 1;
    constexpr int CELL_STENCIL = cell_stencil(D);
    extern __shared__ __align__(16) unsigned char lb_smem[];
    float4 *stage = reinterpret_cast<float4 *>(lb_smem);  // offsets from the centre, .w = index bits
    __shared__ int pre[CELL_STENCIL + 1];  // candidates before stencil cell k
    __shared__ int nstart[CELL_STENCIL];   // first sorted index of stencil cell k
    __shared__ int wsum[LB_THREADS / 32];
    __shared__ int cnt_sm[LB_HC];          // list length so far of each particle of the chunk
    const int tid = threadIdx.x, lane = tid & 31;
    const int sub = tid % LB_TPI;
    const int gshift = lane & ~(LB_TPI - 1);            // first lane of this particle's group
    const unsigned below = (1u << (lane & (LB_TPI - 1))) - 1u;
    const int nrb = rb_list[0];
    const int *rb_cells = rb_list + nrep_all + 1;
    for (int item = blockIdx.x; item < rb_cells[nrb]; item += gridDim.x) {
        const int k = find_rep(item, nrb, [&](int j) { return rb_cells[j]; });
        const int r = rb_list[1 + k];
        const int hc = reps[r].cell_off + item - rb_cells[k];
        const int hstart = cell_start[hc], nhome = cell_start[hc + 1] - hstart;
        if (nhome == 0) continue;
        const RepDev &R = reps[r];
        const int nc = R.nc, local = hc - R.cell_off;
        const int cx = local % nc, cy = (local / nc) % nc, cz = local / (nc * nc);
        const float sc = (float)(R.L / Coord<T>::scale);
        const float rl2 = (float)(R.rcl * R.rcl * (1.0 + 1e-5));
        // the home cell's centre in the integer coordinates
        const U ox = Coord<T>::q(((double)cx + 0.5) / nc), oy = Coord<T>::q(((double)cy + 0.5) / nc),
                oz = Coord<T>::q(((double)cz + 0.5) / nc);
        __syncthreads();  // the previous cell is done with pre, nstart and stage
        // stencil cell tid: its start and count; pre = exclusive prefix sum
        int cntc = 0;
        if (tid < CELL_STENCIL) {
            const int dx = tid % CELL_SPAN - D, dy = (tid / CELL_SPAN) % CELL_SPAN - D,
                      dz = tid / (CELL_SPAN * CELL_SPAN) - D;
            const int nx = (cx + dx + nc) % nc, ny = (cy + dy + nc) % nc, nz = (cz + dz + nc) % nc;
            const int nb = R.cell_off + nx + nc * (ny + nc * nz);
            nstart[tid] = cell_start[nb];
            cntc = cell_start[nb + 1] - cell_start[nb];
        }
        int v = cntc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) wsum[tid >> 5] = v;
        __syncthreads();
        for (int w = 0; w < (tid >> 5); ++w) v += wsum[w];
        if (tid < CELL_STENCIL) pre[tid + 1] = v;
        if (tid == 0) pre[0] = 0;
        __syncthreads();
        const int total = pre[CELL_STENCIL];
        // home particles in chunks of LB_HC: each window of candidates is
        // staged once per chunk, and every particle's count so far is kept
        // in shared memory between windows
        for (int c0 = 0; c0 < nhome; c0 += LB_HC) {
            const int nch = min(LB_HC, nhome - c0);
            for (int w0 = 0; w0 < total; w0 += SCAP) {
                const int wlen = min(SCAP, total - w0);
                __syncthreads();  // the previous window's tests (and counts) are done
                if (w0 == 0)
                    for (int i = tid; i < nch; i += LB_THREADS) cnt_sm[i] = 0;
                // candidate g of the window: the stencil cell holding it by
                // binary search over pre
                for (int g = tid; g < wlen; g += LB_THREADS) {
                    const int gg = w0 + g;
                    int lo = 0, hi = CELL_STENCIL - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (pre[mid] <= gg) lo = mid; else hi = mid - 1;
                    }
                    const int j = nstart[lo] + gg - pre[lo];
                    const Q q = xq[j];
                    // the staged copy carries the sorted index
                    stage[g] = make_float4((float)qdiff<T>(q.x, ox) * sc, (float)qdiff<T>(q.y, oy) * sc,
                                           (float)qdiff<T>(q.z, oz) * sc, __int_as_float(j));
                }
                // the window's last round filled with candidates out of range
                const int wpad = (wlen + LB_TPI - 1) & ~(LB_TPI - 1);
                for (int g = wlen + tid; g < wpad; g += LB_THREADS)
                    stage[g] = make_float4(1e30f, 1e30f, 1e30f, __int_as_float(-1));
                __syncthreads();
                for (int i0 = 0; i0 < nch; i0 += LB_PPB) {
                    const int i = i0 + tid / LB_TPI;
                    const bool have = i < nch;
                    const int s = hstart + c0 + i;
                    float xr = 0.f, yr = 0.f, zr = 0.f;  // this particle's offset from the centre
                    if (have) {
                        const Q xi = xq[s];
                        xr = (float)qdiff<T>(xi.x, ox) * sc;
                        yr = (float)qdiff<T>(xi.y, oy) * sc;
                        zr = (float)qdiff<T>(xi.z, oz) * sc;
                    }
                    int cnt = have ? cnt_sm[i] : 0;
                    int *lrow = nlist + list_row(have ? s : hstart, maxnb, lt);
                    for (int kb = 0; kb < wpad; kb += LB_TPI) {  // uniform over the block
                        const float4 q = stage[kb + sub];
                        const float dx = xr - q.x, dy = yr - q.y, dz = zr - q.z;
                        const int j = __float_as_int(q.w);
                        const bool in = have && (dx * dx + dy * dy + dz * dz < rl2) && j != s;
                        const unsigned grp = (__ballot_sync(0xffffffffu, in) >> gshift) &
                                             ((1u << LB_TPI) - 1u);
                        if (in) {
                            const int pos = cnt + __popc(grp & below);
                            if (pos < maxnb) lrow[list_col(pos, lt)] = j;
                        }
                        cnt += __popc(grp);
                    }
                    if (have && sub == 0) cnt_sm[i] = cnt;
                }
            }
            __syncthreads();  // the chunk's counts are complete
            for (int i = tid / LB_TPI; i < nch; i += LB_PPB) {
                const int s = hstart + c0 + i;
                const int cnt = cnt_sm[i], nn = min(cnt, maxnb);
                if (sub == 0) {
                    if (cnt > maxnb) raise_status(status, ST_NBOVF);
                    nnb[s] = nn;
                }
                // pad to a whole block of PP_LIST_PAD entries with the
                // particle itself (r = 0: no contribution); maxnb is a
                // multiple of PP_LIST_PAD, so the pad stays in the list
                const int pe = nn + sub;
                if (pe < ((nn + PP_LIST_PAD - 1) & ~(PP_LIST_PAD - 1)))
                    nlist[list_index(s, pe, maxnb, lt)] = s;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// pair terms
// ---------------------------------------------------------------------------

// FP64: the reference's pair terms (F(r)/r and phi(r)) at squared distance r2.
__device__ __forceinline__ void pair_direct(double r2, const RepDev &R, double &f_over_r, double &phi)
{
    const double a = R.alpha, k = R.kappa;
    const double rinv = rsqrt(r2);
    const double r = r2 * rinv;
    const double E = exp(-(a * a * r2 + 0.25 * k * k / (a * a)));
    const double xp = erfcx(a * r + 0.5 * k / a);
    const double xm = erfcx(a * r - 0.5 * k / a);
    const double kr = k * r;
    const double hE = 0.5 * rinv * E;
    phi = hE * (xp + xm);
    const double fr = hE * rinv * (xp * (1.0 - kr) + xm * (1.0 + kr)) +
                      (2.0 * a / 1.7724538509055160273) * rinv * E;
    f_over_r = fr * rinv;
}

// ---------------------------------------------------------------------------
// forces from the lists
// ---------------------------------------------------------------------------
constexpr int PPL_THREADS = 256;

// FP64 forces from the lists: the reference's pair terms (pair_direct) per
// entry, TPI threads per particle, Kahan-compensated sums.
template <int TPI>
__global__ void __launch_bounds__(PPL_THREADS)
k_pp_f64(const RepDev *__restrict__ reps, int nrep, const ulonglong4 *__restrict__ xq,
         const int *__restrict__ nnb, const int *__restrict__ nlist, int maxnb,
         double4 *__restrict__ acc_out, double *__restrict__ u_part)
{
    using T = double;
    using Q = ulonglong4;
    constexpr int PPB = PPL_THREADS / TPI;  // particles per block
    constexpr int CH = 32;                  // entries per Kahan flush
    __shared__ double red[32];
    const int b = blockIdx.x;
    const int r = find_rep(b, nrep, [&](int k) { return reps[k].pp_blk_off; });
    const RepDev &R = reps[r];
    const int sub = threadIdx.x % TPI;
    const int s = R.p_off + (b - R.pp_blk_off) * PPB + threadIdx.x / TPI;
    const bool have = s < R.p_off + R.n;
    // L / 2^64 as a hi + lo pair
    const double scd = R.L / Coord<T>::scale;
    const T sc = (T)scd, sc_lo = (T)(scd - (double)sc);
    const T rc2 = (T)(R.rc * R.rc);

    T fx = 0, fy = 0, fz = 0, gx = 0, gy = 0, gz = 0;
    double u = 0.0;
    if (have) {
        const Q xi = xq[s];
        // the padded list in passes of the layout (see list_index): lane sub
        // takes entries v TPI + sub of each pass, as chunks of C
        constexpr int UNR = pp_unr(TPI), STEP = UNR * TPI, C = pp_chunk(TPI), NCH = UNR / C;
        constexpr int CSTRIDE = list_cstride(TPI);
        const int nr = (nnb[s] + PP_LIST_PAD - 1) & ~(PP_LIST_PAD - 1);
        const int *lg = list_lane_at<TPI>(nlist, s >> 5, s & 31, sub, maxnb);
        for (int c0 = 0; c0 < nr; c0 += CH) {
            const int c1 = min(c0 + CH, nr);
            T px = 0, py = 0, pz = 0, pu = 0;
            for (int k0 = c0; k0 < c1; k0 += STEP) {
                // independent loads first (padding points at the particle
                // itself: r2 = 0 is skipped below)
                const int *lp = list_pass_at<TPI>(lg, k0);
                int j[UNR];
#pragma unroll
                for (int i = 0; i < NCH; ++i) {
                    if constexpr (C == 4) {
                        const int4 t = __ldg(reinterpret_cast<const int4 *>(lp + i * CSTRIDE));
                        j[4 * i + 0] = t.x; j[4 * i + 1] = t.y; j[4 * i + 2] = t.z; j[4 * i + 3] = t.w;
                    } else {
                        const int2 t = __ldg(reinterpret_cast<const int2 *>(lp + i * CSTRIDE));
                        j[2 * i + 0] = t.x; j[2 * i + 1] = t.y;
                    }
                }
                Q q[UNR];
#pragma unroll
                for (int v = 0; v < UNR; ++v) q[v] = xq[j[v]];
#pragma unroll
                for (int v = 0; v < UNR; ++v) {
                    const T ix = (T)qdiff<T>(xi.x, q[v].x), iy = (T)qdiff<T>(xi.y, q[v].y),
                            iz = (T)qdiff<T>(xi.z, q[v].z);
                    const T dx = ix * sc + ix * sc_lo;
                    const T dy = iy * sc + iy * sc_lo;
                    const T dz = iz * sc + iz * sc_lo;
                    const T r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 < rc2 && r2 > (T)0) {
                        T fr, ph;
                        pair_direct(r2, R, fr, ph);
                        px += fr * dx;
                        py += fr * dy;
                        pz += fr * dz;
                        pu += ph;
                    }
                }
            }
            T yx = px - gx, tx = fx + yx; gx = (tx - fx) - yx; fx = tx;
            T yy = py - gy, ty = fy + yy; gy = (ty - fy) - yy; fy = ty;
            T yz = pz - gz, tz = fz + yz; gz = (tz - fz) - yz; fz = tz;
            u += (double)pu;
        }
    }
#pragma unroll
    for (int o = TPI / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (have && sub == 0) acc_out[s] = make_double4(fx, fy, fz, 0.0);
    const double ut = block_sum(u, red);
    if (threadIdx.x == 0) u_part[b] = ut;
}

// ---------------------------------------------------------------------------
// FP32 forces from the padded lists
// ---------------------------------------------------------------------------
// Each thread evaluates its list entries two at a time. sm_100 can issue the
// FP32 arithmetic of such a pair as packed fma.rn.f32x2 / mul / add
// instructions (P3M_PP_PACK=1, the same rounding operand by operand); on the
// 20 x 1e4-particle ensemble that measured slower than the scalar form (pair
// loop 0.199 against 0.181 ms: the kernel is bound by L1 -- the scattered
// 16-byte coordinate gathers and the table reads -- not by issue, and the
// packed operands cost register moves), so the scalar form is the default.
// Lists are padded with the particle's own index to whole blocks of
// PP_LIST_PAD entries, so the loop reads them without a bounds test.
#ifndef P3M_PP_PACK
#define P3M_PP_PACK 0
#endif

// Copies of the pair table in shared memory. A warp's 128-bit table reads go
// through the banks eight lanes at a time; with random intervals two of
// those lanes often hit the same bank group (8.4 wavefronts per read measured
// on the ensemble, against 4 without conflicts). With 8 copies, copy c held
// in bank group c only (entry i at float4 index 8 i + c) and read by the
// lanes l with l mod 8 = c, no two lanes of a phase can conflict.
#ifndef P3M_PP_TABLE_COPIES
#define P3M_PP_TABLE_COPIES 1
#endif
constexpr int PP_TABLE_COPIES = P3M_PP_TABLE_COPIES;
static_assert(PP_TABLE_COPIES == 1 || PP_TABLE_COPIES == 8, "1 or 8 table copies");

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

template <bool P> __device__ __forceinline__ float2 v_fma(float2 a, float2 b, float2 c)
{
    if constexpr (P) return __ffma2_rn(a, b, c);
    else return f2(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y));
}
template <bool P> __device__ __forceinline__ float2 v_mul(float2 a, float2 b)
{
    if constexpr (P) return __fmul2_rn(a, b);
    else return f2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
}
template <bool P> __device__ __forceinline__ float2 v_add(float2 a, float2 b)
{
    if constexpr (P) return __fadd2_rn(a, b);
    else return f2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}

// Two candidates a, b of particle xi: adds F/r * (dx, dy, dz) and phi of the
// ones closer than rc (and not the particle itself) to p*. tab holds the
// cubic coefficients of psi = phi r in the interval coordinate u in [0,1),
// one float4 per interval of h = rc / PP_TABLE_N; with t = r / h, the
// interval i = round(t - 1/2) and float(i) come from the 1.5 * 2^23 rounding
// constant (exact for t < 2^22, no float <-> int conversions), and the force
// from the same cubic: g = F r^2 = psi - t dpsi/du, F/r = g / r^3, phi = psi / r.
// With KEEP, bits 0 / 1 of `keep` are set for a / b closer than sqrt(rin2)
// (self entries included; the caller masks them by index).
template <bool P, bool KEEP = false>
__device__ __forceinline__ void pair_table2(const uint4 &xi, const uint4 &qa, const uint4 &qb,
                                            float2 sc, float2 sc_lo, float rc2, float2 inv_h,
                                            const float4 *__restrict__ tab, float2 &px,
                                            float2 &py, float2 &pz, float2 &pu,
                                            float rin2 = 0.f, unsigned *keep = nullptr)
{
    constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: round-to-integer constant
    const float2 ix = f2((float)(int)(xi.x - qa.x), (float)(int)(xi.x - qb.x));
    const float2 iy = f2((float)(int)(xi.y - qa.y), (float)(int)(xi.y - qb.y));
    const float2 iz = f2((float)(int)(xi.z - qa.z), (float)(int)(xi.z - qb.z));
    const float2 dx = v_fma<P>(ix, sc_lo, v_mul<P>(ix, sc));
    const float2 dy = v_fma<P>(iy, sc_lo, v_mul<P>(iy, sc));
    const float2 dz = v_fma<P>(iz, sc_lo, v_mul<P>(iz, sc));
    const float2 r2 = v_fma<P>(dz, dz, v_fma<P>(dy, dy, v_mul<P>(dx, dx)));
    if constexpr (KEEP) *keep = (r2.x < rin2 ? 1u : 0u) | (r2.y < rin2 ? 2u : 0u);
    // r = 0 (the particle itself: list padding) would make r = 0 * inf: take
    // rc^2 there (a valid table interval) and mask the result; beyond rc the
    // last interval's cubic is extrapolated, finite, and masked as well
    const float2 rs = f2(r2.x > 0.f ? r2.x : rc2, r2.y > 0.f ? r2.y : rc2);
    const float2 m = f2((r2.x < rc2 && r2.x > 0.f) ? 1.f : 0.f, (r2.y < rc2 && r2.y > 0.f) ? 1.f : 0.f);
    const float2 rinv = f2(rsqrtf(rs.x), rsqrtf(rs.y));
    const float2 t = v_mul<P>(v_mul<P>(rs, rinv), inv_h);
    const float2 tb = v_add<P>(v_add<P>(t, f2(-0.5f, -0.5f)), f2(kMagic, kMagic));
    const int ia = min(__float_as_int(tb.x) - 0x4B400000, PP_TABLE_N - 1);
    const int ib = min(__float_as_int(tb.y) - 0x4B400000, PP_TABLE_N - 1);
    const float2 fl = v_add<P>(tb, f2(-kMagic, -kMagic));       // the interval index, exact
    const float2 u = v_fma<P>(fl, f2(-1.f, -1.f), t);            // t - fl, exact
    // reading the inner lists, entries beyond rc and list padding (masked
    // below) skip their table read: fewer shared-memory wavefronts in the
    // L1-bound loop (0.146 against 0.150 ms at cfg3). Over the Verlet lists
    // of a list-building pass the predication cost more than it saved.
    float4 ca, cb;
    if constexpr (KEEP) {
        ca = tab[ia * PP_TABLE_COPIES];
        cb = tab[ib * PP_TABLE_COPIES];
    } else {
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        ca = m.x != 0.f ? tab[ia * PP_TABLE_COPIES] : z4;
        cb = m.y != 0.f ? tab[ib * PP_TABLE_COPIES] : z4;
    }
    const float2 c0 = f2(ca.x, cb.x), c1 = f2(ca.y, cb.y), c2 = f2(ca.z, cb.z), c3 = f2(ca.w, cb.w);
    const float2 ps = v_fma<P>(v_fma<P>(v_fma<P>(c3, u, c2), u, c1), u, c0);
    const float2 dps = v_fma<P>(v_fma<P>(v_mul<P>(c3, f2(3.f, 3.f)), u, v_add<P>(c2, c2)), u, c1);
    const float2 g = v_fma<P>(v_mul<P>(t, f2(-1.f, -1.f)), dps, ps);  // psi - t psi'
    const float2 fr = v_mul<P>(v_mul<P>(v_mul<P>(g, v_mul<P>(rinv, rinv)), rinv), m);
    const float2 ph = v_mul<P>(v_mul<P>(ps, rinv), m);
    px = v_fma<P>(fr, dx, px);
    py = v_fma<P>(fr, dy, py);
    pz = v_fma<P>(fr, dz, pz);
    pu = v_add<P>(pu, ph);
}

#ifndef P3M_PP_MINB
#define P3M_PP_MINB 3
#endif

// List modes of the FP32 pair kernel. PP_OUTER (no inner lists, prune
// buffer 0) reads the Verlet lists. PP_DYN decides per block: a replica whose
// flag is set (Verlet rebuild or inner prune) has its outer lists read and
// each particle's inner list written on the way -- the entries closer than
// rc + pbuf, in outer-list order, padded like the outer ones -- with the
// positions they were taken at; the other replicas read their inner lists.
enum PpMode { PP_OUTER = 0, PP_DYN = 1 };

struct PruneArgs {
    const int *rebuild = nullptr, *prune = nullptr;  // per-replica flags
    int *nnb_in = nullptr, *nlist_in = nullptr;      // inner lists (written by pruning blocks)
    int maxnb_in = 0;
    const int *cell_perm = nullptr;                  // sorted -> original particle
    const double *pos = nullptr;
    double *pos_pref = nullptr;                      // positions of the inner-list build
    int *status = nullptr;
};

// Staging of the inner entries of a warp's particles while a block of 16
// fills: position q of the warp's particle w at stage[q * PPW + w] (PPW =
// 32 / TPI particles per warp), so the TPI lanes of a particle, which touch
// consecutive positions, and the warp's particles, one bank apart, never
// share a bank. 32 positions: up to 15 carried and 16 of a pass.
template <int TPI> struct Stage {
    static constexpr int PPW = 32 / TPI;
    int *w;  // this warp's area (32 PPW ints)
    int p;   // this particle's index in the warp
    __device__ __forceinline__ int &operator[](int q) const { return w[q * PPW + p]; }
};

// One particle's block of 16 staged entries, written by its TPI lanes in
// the list layout: og = the lane's first chunk of the block (list_lane_at
// plus list_block).
template <int TPI>
__device__ __forceinline__ void store_block(int *og, const Stage<TPI> &buf, int sub)
{
    constexpr int UNR = pp_unr(TPI), STEP = UNR * TPI, C = pp_chunk(TPI), NCH = UNR / C;
    constexpr int CSTRIDE = list_cstride(TPI);
#pragma unroll
    for (int pass = 0; pass < PP_LIST_PAD / STEP; ++pass)
#pragma unroll
        for (int i = 0; i < NCH; ++i) {
            const int e = pass * STEP + i * C * TPI + sub;  // entries (i C + c) TPI + sub
            int *dst = og + list_chunk<TPI>(pass, i);
            if constexpr (C == 4)
                *reinterpret_cast<int4 *>(dst) =
                    make_int4(buf[e], buf[e + TPI], buf[e + 2 * TPI], buf[e + 3 * TPI]);
            else
                *reinterpret_cast<int2 *>(dst) = make_int2(buf[e], buf[e + TPI]);
        }
}

// The pair loop of one particle slot s (have: s holds a particle of
// replica R) over the list (nnb, nlist, maxnb); PRUNE: also its inner list.
// Returns the energy partial; the force goes to acc_out.
template <int TPI, bool PRUNE>
__device__ __forceinline__ double pp_body(const RepDev &R, int s, bool have,
                                          const uint4 *__restrict__ xq,
                                          const int *__restrict__ nnb,
                                          const int *__restrict__ nlist, int maxnb,
                                          const float4 *__restrict__ tab,
                                          float4 *__restrict__ acc_out, const PruneArgs &pa,
                                          int *stage_warp)
{
    constexpr bool P = P3M_PP_PACK != 0;
    constexpr int UNR = pp_unr(TPI);                     // entries per lane per pass
    constexpr int STEP = UNR * TPI;                      // entries of a particle per pass
    constexpr int C = pp_chunk(TPI), NCH = UNR / C;      // list chunks of a lane per pass
    constexpr int CSTRIDE = list_cstride(TPI);                // between a lane's chunks (entries)
    static_assert(UNR % 2 == 0 && PP_LIST_PAD % STEP == 0, "whole pairs, whole pad blocks");
    static_assert(PP_LIST_PAD == 16 && STEP <= 16, "the list layout's blocks");
    const int sub = threadIdx.x % TPI;
    // L / 2^32 as a hi + lo pair (a plain FP32 scale would bias every dx of
    // the replica by the same relative rounding)
    const double scd = R.L / 4294967296.0;
    const float sch = (float)scd;
    const float2 sc = f2(sch, sch), sc_lo = f2((float)(scd - (double)sch), (float)(scd - (double)sch));
    const float rc2 = (float)(R.rc * R.rc);
    const float ih = (float)(PP_TABLE_N / R.rc);
    const float2 inv_h = f2(ih, ih);
    const float rin2 = PRUNE ? (float)((R.rc + R.pbuf) * (R.rc + R.pbuf)) : 0.f;
    const int gbase = (threadIdx.x & 31) & ~(TPI - 1);   // first lane of this particle's group
    const int p32 = s & 31;

    float fx = 0.f, fy = 0.f, fz = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    double u = 0.0;
    // pruning keeps the warp converged for its ballots and shared staging:
    // every lane runs the warp's longest list, lanes past their own (or
    // without a particle) evaluating their own slot, which adds nothing
    if (have || PRUNE) {
        const int sv = have ? s : R.p_off;
        const uint4 xi = xq[sv];
        const int nr = have ? (nnb[s] + PP_LIST_PAD - 1) & ~(PP_LIST_PAD - 1) : 0;
        const int nloop = PRUNE ? __reduce_max_sync(0xffffffffu, nr) : nr;
        // this lane's first chunk in the particle's group blocks
        const int *lg = list_lane_at<TPI>(nlist, sv >> 5, p32, sub, maxnb);
        const Stage<TPI> buf{stage_warp, (int)(threadIdx.x & 31) / TPI};
        int fill = 0, blk = 0;  // pruning: staged entries, blocks written
        int *og = PRUNE ? list_lane_at<TPI>(pa.nlist_in, sv >> 5, p32, sub, pa.maxnb_in) : nullptr;
        for (int k0 = 0; k0 < nloop; k0 += STEP) {
            const int *lp = list_pass_at<TPI>(lg, k0);
            int j[UNR];
            if (!PRUNE || k0 < nr) {
#pragma unroll
                for (int i = 0; i < NCH; ++i) {
                    if constexpr (C == 4) {
                        const int4 t = __ldg(reinterpret_cast<const int4 *>(lp + i * CSTRIDE));
                        j[4 * i + 0] = t.x; j[4 * i + 1] = t.y; j[4 * i + 2] = t.z; j[4 * i + 3] = t.w;
                    } else {
                        const int2 t = __ldg(reinterpret_cast<const int2 *>(lp + i * CSTRIDE));
                        j[2 * i + 0] = t.x; j[2 * i + 1] = t.y;
                    }
                }
            } else {
#pragma unroll
                for (int v = 0; v < UNR; ++v) j[v] = sv;
            }
            uint4 q[UNR];
#pragma unroll
            for (int v = 0; v < UNR; ++v) q[v] = xq[j[v]];
            float2 px = f2(0.f, 0.f), py = px, pz = px, pu = px;
            unsigned keep = 0;  // pruning: bit v = this lane's entry v goes to the inner list
#pragma unroll
            for (int v = 0; v < UNR; v += 2) {
                unsigned k2 = 0;
                pair_table2<P, PRUNE>(xi, q[v], q[v + 1], sc, sc_lo, rc2, inv_h, tab, px, py, pz,
                                      pu, rin2, &k2);
                if constexpr (PRUNE) keep |= k2 << v;
            }
            const float sx = px.x + px.y, sy = py.x + py.y, sz = pz.x + pz.y;
            float y = sx - gx, t = fx + y; gx = (t - fx) - y; fx = t;
            y = sy - gy; t = fy + y; gy = (t - fy) - y; fy = t;
            y = sz - gz; t = fz + y; gz = (t - fz) - y; fz = t;
            u += (double)(pu.x + pu.y);
            if constexpr (PRUNE) {
#pragma unroll
                for (int v = 0; v < UNR; ++v)
                    if (j[v] == sv) keep &= ~(1u << v);  // list padding, idle lanes
                // this lane's entry v is entry v TPI + sub of the pass: the
                // group's keep bits in entry order give each kept one its place
                unsigned mask = 0;
                if constexpr (TPI == 1) {
                    mask = keep;
                } else if constexpr (TPI == 2) {
                    // the partner's 8 bits by one shuffle, both spread to
                    // alternate bits (entry 2 v + sub)
                    const unsigned other = __shfl_xor_sync(0xffffffffu, keep, 1);
                    auto spread = [](unsigned x) {
                        x = (x | (x << 4)) & 0x0F0Fu;
                        x = (x | (x << 2)) & 0x3333u;
                        return (x | (x << 1)) & 0x5555u;
                    };
                    const unsigned k0 = sub ? other : keep, k1 = sub ? keep : other;
                    mask = spread(k0) | (spread(k1) << 1);
                } else {
#pragma unroll
                    for (int v = 0; v < UNR; ++v) {
                        const unsigned bal = __ballot_sync(0xffffffffu, (keep >> v) & 1u);
                        mask |= ((bal >> gbase) & ((1u << TPI) - 1u)) << (v * TPI);
                    }
                }
#pragma unroll
                for (int v = 0; v < UNR; ++v)
                    if ((keep >> v) & 1u) buf[fill + __popc(mask & ((1u << (v * TPI + sub)) - 1u))] = j[v];
                fill += __popc(mask);
                __syncwarp();
                // a whole block: out, in the list layout (group-uniform tests,
                // no synchronisation inside them)
                const bool full = fill >= PP_LIST_PAD;
                if (full && (blk + 1) * PP_LIST_PAD <= pa.maxnb_in)
                    store_block<TPI>(og + list_block(blk), buf, sub);
                __syncwarp();
                if (full)
                    for (int e = sub; e < fill - PP_LIST_PAD; e += TPI) buf[e] = buf[PP_LIST_PAD + e];
                __syncwarp();
                if (full) {
                    fill -= PP_LIST_PAD;
                    ++blk;
                }
            }
        }
        if constexpr (PRUNE) {
            const int cin = blk * PP_LIST_PAD + fill;
            // the last block, padded with the particle itself
            if (fill > 0)
                for (int e = fill + sub; e < PP_LIST_PAD; e += TPI) buf[e] = sv;
            __syncwarp();
            if (have && fill > 0 && (blk + 1) * PP_LIST_PAD <= pa.maxnb_in)
                store_block<TPI>(og + list_block(blk), buf, sub);
            if (have && sub == 0) {
                if (cin > pa.maxnb_in) raise_status(pa.status, ST_NBOVF);
                pa.nnb_in[s] = min(cin, pa.maxnb_in);
                const int o = pa.cell_perm[s];
                pa.pos_pref[3 * o + 0] = pa.pos[3 * o + 0];
                pa.pos_pref[3 * o + 1] = pa.pos[3 * o + 1];
                pa.pos_pref[3 * o + 2] = pa.pos[3 * o + 2];
            }
        }
    }
#pragma unroll
    for (int o = TPI / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
    }
    if (have && sub == 0) acc_out[s] = make_float4(fx, fy, fz, 0.f);
    return u;
}

template <int TPI, int PM>
__global__ void __launch_bounds__(PPL_THREADS, P3M_PP_MINB)
k_pp_f32(const RepDev *__restrict__ reps, int nrep, const uint4 *__restrict__ xq,
         const int *__restrict__ nnb, const int *__restrict__ nlist, int maxnb,
         const float4 *__restrict__ tables, float4 *__restrict__ acc_out,
         double *__restrict__ u_part, PruneArgs pa)
{
    constexpr int PPB = PPL_THREADS / TPI;  // particles per block
    __shared__ double red[32];
    __shared__ __align__(16) int pstage[PM == PP_DYN ? PPB * 32 : 1];  // 32 positions per particle
    extern __shared__ __align__(16) float4 ppl_tab[];
    const int b = blockIdx.x;
    const int r = find_rep(b, nrep, [&](int k) { return reps[k].pp_blk_off; });
    const RepDev &R = reps[r];
    {
        const float4 *src = tables + (long long)r * PP_TABLE_N;
        for (int k = threadIdx.x; k < PP_TABLE_N * PP_TABLE_COPIES; k += PPL_THREADS)
            cp_async16(ppl_tab + k, src + k / PP_TABLE_COPIES);
        cp_async_wait_all();
        __syncthreads();
    }
    const float4 *tab = ppl_tab + (threadIdx.x & (PP_TABLE_COPIES - 1));  // this lane's copy
    const int s = R.p_off + (b - R.pp_blk_off) * PPB + threadIdx.x / TPI;
    const bool have = s < R.p_off + R.n;
    int *stage_warp = pstage + (PM == PP_DYN ? (threadIdx.x >> 5) * 32 * (32 / TPI) : 0);
    double u;
    if constexpr (PM == PP_OUTER) {
        u = pp_body<TPI, false>(R, s, have, xq, nnb, nlist, maxnb, tab, acc_out, pa, stage_warp);
    } else if ((pa.rebuild[r] | pa.prune[r]) != 0) {  // block-uniform
        u = pp_body<TPI, true>(R, s, have, xq, nnb, nlist, maxnb, tab, acc_out, pa, stage_warp);
    } else {
        u = pp_body<TPI, false>(R, s, have, xq, pa.nnb_in, pa.nlist_in, pa.maxnb_in, tab,
                                acc_out, pa, stage_warp);
    }
    const double ut = block_sum(u, red);
    if (threadIdx.x == 0) u_part[b] = ut;
}

// Per-replica U_pp = 1/2 sum of the replica's block partials (index order).
__global__ void k_reduce_pp(const RepDev *__restrict__ reps, int nrep,
                            const double *__restrict__ u_part, int nblk_total,
                            double *__restrict__ rep_out)
{
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nrep;
         r += gridDim.x * (blockDim.x >> 5)) {
        const int b0 = reps[r].pp_blk_off;
        const int b1 = (r + 1 < nrep) ? reps[r + 1].pp_blk_off : nblk_total;
        double t = 0.0;
        for (int k = b0 + lane; k < b1; k += 32) t += u_part[k];
        t = warp_sum(t);
        if (lane == 0) rep_out[8 * r + RO_UPP] = 0.5 * t;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int qgrid(int n) { int g = (n + 255) / 256; return g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g); }

int pp_particles_per_block(int tpi) { return PPL_THREADS / tpi; }

template <typename T> void configure_pp_kernels()
{
    using Q = typename Coord<T>::Q;
    const int lbs = (int)(LB_SCAP * sizeof(float4));
    auto setl = [&](auto k) { cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, lbs); };
    setl(k_build_lists<T, 1, 0>); setl(k_build_lists<T, 1, 1>);
    setl(k_build_lists<T, 1, 2>); setl(k_build_lists<T, 1, 3>);
    setl(k_build_lists<T, 2, 0>); setl(k_build_lists<T, 2, 1>);
    setl(k_build_lists<T, 2, 2>); setl(k_build_lists<T, 2, 3>);
    if constexpr (sizeof(T) == 4) {
        const int tab = (int)(PP_TABLE_N * PP_TABLE_COPIES * sizeof(float4));
        auto set = [&](auto k) { cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, tab); };
        set(k_pp_f32<1, PP_OUTER>); set(k_pp_f32<2, PP_OUTER>);
        set(k_pp_f32<4, PP_OUTER>); set(k_pp_f32<8, PP_OUTER>);
        set(k_pp_f32<1, PP_DYN>); set(k_pp_f32<2, PP_DYN>);
        set(k_pp_f32<4, PP_DYN>); set(k_pp_f32<8, PP_DYN>);
    }
}

template <typename T> void launch_quantize(const DevState &s, cudaStream_t st)
{
    k_quantize<T><<<qgrid(s.ntot), 256, 0, st>>>(s.reps, s.prep, s.cell_perm, s.pos,
                                                 (typename Coord<T>::Q *)s.xq, s.ntot);
}

template <typename T> void launch_build_lists(const DevState &s, cudaStream_t st)
{
    using Q = typename Coord<T>::Q;
    const int grid = s.ncell < 148 * 16 ? s.ncell : 148 * 16;
    using K = void (*)(const RepDev *, int, const int *, const Q *, int *, int *, int, const int *,
                       int, int *);
    static const K kerns[2][4] = {
        {k_build_lists<T, 1, 0>, k_build_lists<T, 1, 1>, k_build_lists<T, 1, 2>, k_build_lists<T, 1, 3>},
        {k_build_lists<T, 2, 0>, k_build_lists<T, 2, 1>, k_build_lists<T, 2, 2>, k_build_lists<T, 2, 3>}};
    const K kern = kerns[s.cell_div == 1 ? 0 : 1][__builtin_ctz((unsigned)s.pp_tpi) & 3];
    kern<<<grid, LB_THREADS, LB_SCAP * sizeof(float4), st>>>(
        s.reps, s.nrep, s.cell_start, (const Q *)s.xq, s.nnb, s.nlist, s.maxnb, s.rb_list, s.nrep,
        s.status);
}

template <typename T, int TPI> static void launch_pp_tpi(const DevState &s, cudaStream_t st)
{
    using Q = typename Coord<T>::Q;
    if constexpr (sizeof(T) == 4) {
        const size_t tab = PP_TABLE_N * PP_TABLE_COPIES * sizeof(float4);
        PruneArgs pa;
        if (s.prune_buf <= 0.0) {
            k_pp_f32<TPI, PP_OUTER><<<s.pp_nblk, PPL_THREADS, tab, st>>>(
                s.reps, s.nrep, (const uint4 *)s.xq, s.nnb, s.nlist, s.maxnb, s.pp_tables,
                (float4 *)s.acc_pp, s.u_pp_part, pa);
            return;
        }
        pa.rebuild = s.rebuild;
        pa.prune = s.prune;
        pa.nnb_in = s.nnb_in;
        pa.nlist_in = s.nlist_in;
        pa.maxnb_in = s.maxnb_in;
        pa.cell_perm = s.cell_perm;
        pa.pos = s.pos;
        pa.pos_pref = s.pos_pref;
        pa.status = s.status;
        k_pp_f32<TPI, PP_DYN><<<s.pp_nblk, PPL_THREADS, tab, st>>>(
            s.reps, s.nrep, (const uint4 *)s.xq, s.nnb, s.nlist, s.maxnb, s.pp_tables,
            (float4 *)s.acc_pp, s.u_pp_part, pa);
    } else {
        k_pp_f64<TPI><<<s.pp_nblk, PPL_THREADS, 0, st>>>(s.reps, s.nrep, (const Q *)s.xq, s.nnb,
                                                         s.nlist, s.maxnb, (double4 *)s.acc_pp,
                                                         s.u_pp_part);
    }
}

template <typename T> void launch_pp(const DevState &s, cudaStream_t st)
{
    switch (s.pp_tpi) {
    case 2: launch_pp_tpi<T, 2>(s, st); break;
    case 4: launch_pp_tpi<T, 4>(s, st); break;
    case 8: launch_pp_tpi<T, 8>(s, st); break;
    default: launch_pp_tpi<T, 1>(s, st);
    }
}


void launch_reduce_pp(const DevState &s, cudaStream_t st)
{
    k_reduce_pp<<<(s.nrep + 3) / 4, 128, 0, st>>>(s.reps, s.nrep, s.u_pp_part, s.pp_nblk,
                                                  s.rep_out);
}

#define P3M_INST(T)                                                         \
    template void configure_pp_kernels<T>();                                 \
    template void launch_quantize<T>(const DevState &, cudaStream_t);        \
    template void launch_build_lists<T>(const DevState &, cudaStream_t);     \
    template void launch_pp<T>(const DevState &, cudaStream_t);
P3M_INST(float)
P3M_INST(double)

}  // namespace p3m
