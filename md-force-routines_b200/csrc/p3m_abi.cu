// C ABI of libp3m_b200: contexts, device buffers, the compat entry points that
// mirror the reference's Python functions, and the device-resident stepper.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "p3m_kernels.h"

using namespace p3m;

struct p3m_ctx {
    int device = 0;
    int prec = P3M_FP32;
    int nrep = 0;
    std::vector<p3m_replica_desc> desc;
    std::vector<RepDev> rh;
    std::vector<char> green_ready;
    double skin_override = -1.0;  // the skin of the last p3m_set_tuning (< 0: per replica)
    DevState s;
    cudaStream_t st = nullptr;
    cudaStream_t st2 = nullptr;   // the mesh branch of a step (joined back into st)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaStream_t st3 = nullptr;   // the n(q,t) branch of a step
    cudaEvent_t ev_join3 = nullptr;
    int *counters = nullptr;      // [0] run step, [1] ring position, [2] it0, [3] n(q,t) rows,
                                  // [4] snapshots taken, [5] this step's snapshot slot
    int snap_interval = 0, snap_cap = 0;
    double *snap = nullptr;       // [cap][ntot][9] state snapshots
    int *snap_steps = nullptr;    // [cap] step index of each snapshot
    long long snap_read = 0;      // snapshots handed to the caller
    double *ring = nullptr;       // energies [cap][nrep][4]
    int ring_cap = 0;
    int ring_rows = 0;            // rows written (host-side tally)
    double *qmult = nullptr;      // [nq]
    int nq = 0, nqt_cap = 0;
    int nq_consecutive = 0;       // qmult == 1, 2, ..., nq
    double *nqt_part = nullptr;   // [nblk][nq*6]
    double *nqt_ring = nullptr;   // [cap][nrep][nq*6]
    int nqt_rows = 0;
    double *scratch = nullptr;    // FP64 staging: max(3 M^3, gf partials)
    double *ep = nullptr;         // FP64 field at particles (ntot,3)
    double *tmp_nq = nullptr;     // one n(q) row for the compat call [nrep][nq*6]
    int tmp_nq_cap = 0;
    double *hbuf = nullptr;       // pinned host staging
    size_t hbuf_bytes = 0;
    // p3m_get_step_async: pinned copy of rep_out ([R][8]) and the status word
    double *h_step = nullptr;
    double *step_out = nullptr;   // caller's (R, 4) energies, filled at p3m_sync
    bool step_pending = false;
    long long step_launches = 0;  // launches when the copies were queued
    bool state_set = false;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    // kGraphSteps steps per graph (launched for whole groups of steps)
    cudaGraphExec_t graphK[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    long long graph_kernels[2][2] = {{0, 0}, {0, 0}};  // kernels per step of the captured graphs
    int ncell_cap = 0;            // cells allocated (grid with skin 0)
    long long nlist_cap = 0;      // list entries allocated
    long long nlist_in_cap = 0;   // inner-list entries allocated
    int pp_nblk_cap = 0;          // PP blocks allocated (tpi = 8)
    long long launches = 0;
    std::string err;
};

static thread_local std::string g_err;

// Steps captured in one multi-step graph on the FP32 path: fewer graph
// launches, and no gap between them, for small systems whose steps last tens
// of microseconds (cfg1: 0.0781 against 0.0810 ms per step). The FP64 path's
// steps measured 3.5 % slower as groups, so it launches them one at a time.
static const int kGraphSteps = 8;
static int graph_steps(const p3m_ctx *ctx) { return ctx->prec == P3M_FP32 ? kGraphSteps : 1; }

// Drop the captured step graphs (all, or only those recording n(q,t)).
static void drop_graphs(p3m_ctx *ctx, bool rec_only = false)
{
    for (int a = 0; a < 2; ++a)
        for (int b = rec_only ? 1 : 0; b < 2; ++b) {
            if (ctx->graph[a][b]) { cudaGraphExecDestroy(ctx->graph[a][b]); ctx->graph[a][b] = nullptr; }
            if (ctx->graphK[a][b]) { cudaGraphExecDestroy(ctx->graphK[a][b]); ctx->graphK[a][b] = nullptr; }
        }
}

#define P3M_VERSION 200

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) return fail(ctx, P3M_ECUDA, #call, cudaGetErrorString(e_)); \
    } while (0)

static int fail(p3m_ctx *ctx, int code, const char *what, const char *why)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s", what, why ? why : "");
    if (ctx) ctx->err = buf; else g_err = buf;
    return code;
}

static bool is_pow2(int m) { return m > 0 && (m & (m - 1)) == 0; }

static int ilog2(int m)
{
    int l = 0;
    while ((1 << l) < m) ++l;
    return l;
}

template <typename X> static cudaError_t dalloc(X **p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(X));
    if (e == cudaSuccess) e = cudaMemset(*p, 0, count * sizeof(X));
    return e;
}

static cudaError_t valloc(void **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    return e;
}

static int check_device(p3m_ctx *ctx, int device)
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(ctx, P3M_ENODEV, "no CUDA device", e != cudaSuccess ? cudaGetErrorString(e) : "");
    if (device < 0 || device >= n) return fail(ctx, P3M_ENODEV, "device index out of range", "");
    cudaDeviceProp pr;
    CK(cudaGetDeviceProperties(&pr, device));
    if (pr.major != 10)
        return fail(ctx, P3M_ENODEV, "library is built for sm_100a (B200)", pr.name);
    CK(cudaSetDevice(device));
    return P3M_OK;
}

template <typename T> static size_t tsize() { return sizeof(T); }

// Default Verlet skin (a_ws): a list rebuild when a particle has moved skin/2.
static const double kDefaultSkin = 0.5;

// Yukawa-Ewald pair functions on the host, in FP64: g(r) = F(r) r^2 and
// psi(r) = phi(r) r (F and phi of yukawa_pp.py:115,121-124, multiplied out so
// both are finite at r = 0).
static void pair_g_psi(double r, double kappa, double a, double *g, double *psi)
{
    const double up = a * r + 0.5 * kappa / a, um = a * r - 0.5 * kappa / a;
    const double ep = exp(kappa * r) * erfc(up), em = exp(-kappa * r) * erfc(um);
    *psi = 0.5 * (ep + em);
    *g = 0.5 * (ep * (1.0 - kappa * r) + em * (1.0 + kappa * r)) +
         (a / sqrt(M_PI)) * r * (exp(-up * up) * exp(kappa * r) + exp(-um * um) * exp(-kappa * r));
}

// Cubic of psi per interval through the samples at u = 0, 1/3, 2/3, 1
// (monomial coefficients in u): PP_TABLE_N float4 (the FP32 kernel derives
// the force from the same cubic).
static void build_pp_table(const p3m_replica_desc &d, float4 *out)
{
    const double h = d.rc / PP_TABLE_N;
    for (int i = 0; i < PP_TABLE_N; ++i) {
        double fg[4], fp[4];
        for (int k = 0; k < 4; ++k) pair_g_psi((i + k / 3.0) * h, d.kappa, d.alpha, &fg[k], &fp[k]);
        float4 &c = out[i];
        c.x = (float)fp[0];
        c.y = (float)((-11.0 * fp[0] + 18.0 * fp[1] - 9.0 * fp[2] + 2.0 * fp[3]) / 2.0);
        c.z = (float)((18.0 * fp[0] - 45.0 * fp[1] + 36.0 * fp[2] - 9.0 * fp[3]) / 2.0);
        c.w = (float)((-9.0 * fp[0] + 27.0 * fp[1] - 27.0 * fp[2] + 9.0 * fp[3]) / 2.0);
    }
}

// Work items of the mesh passes of every replica: x-pass items, and either
// plane items (sides up to s.plane_max: the fused y/z plane kernel) or y and
// z pencil items. Updates ctx->rh offsets and ctx->s totals; the caller
// uploads.
static void plan_mesh_passes(p3m_ctx *ctx)
{
    DevState &s = ctx->s;
    int wa = 0, wb = 0, wc = 0, wp = 0, maxp = 0;
    for (int r = 0; r < ctx->nrep; ++r) {
        RepDev &R = ctx->rh[r];
        R.wa_off = wa;
        R.wb_off = wb;
        R.wc_off = wc;
        R.wp_off = wp;
        const int M = R.M;
        if (M == 0) continue;
        wa += M * (M >> (x_lines_log(R.logM) + 1));
        if (M <= s.plane_max) {
            wp += M / 2 + 1;
            if (M > maxp) maxp = M;
        } else {
            wb += (M / 2 + 1) * (M / PENCIL);
            wc += (M / 2 + 1) * (M / PENCIL);
        }
    }
    s.wa = wa;
    s.wb = wb;
    s.wc = wc;
    s.wp = wp;
    s.max_plane = maxp;
}

// Cell grid (cells >= (rc + skin) / cell_div, at least 3 cell_div per side), list capacity and
// PP block layout of every replica for a given skin and threads-per-particle.
// Updates ctx->rh and ctx->s counts; the caller uploads and (re)allocates.
static void plan_lists(p3m_ctx *ctx, double skin_override, int tpi)
{
    DevState &s = ctx->s;
    int cell = 0, blk = 0;
    double maxmean = 0.0, maxmean_in = 0.0;
    const int ppb = pp_particles_per_block(tpi);
    for (int r = 0; r < ctx->nrep; ++r) {
        const p3m_replica_desc &d = ctx->desc[r];
        RepDev &R = ctx->rh[r];
        double skin = skin_override >= 0.0 ? skin_override : (d.skin >= 0.0 ? d.skin : kDefaultSkin);
        // rc + skin <= L/3 keeps >= 3 cell_div cells per side, more than
        // the stencil spans (no cell is visited twice)
        const double smax = d.box / 3.0 * (1.0 - 1e-12) - d.rc;
        if (skin > smax) skin = smax > 0.0 ? smax : 0.0;
        R.skin = skin;
        R.rcl = d.rc + skin;
        R.nc = (int)floor(s.cell_div * d.box / R.rcl);  // >= 3 cell_div
        R.cellw = d.box / R.nc;
        R.inv_cellw = 1.0 / R.cellw;
        R.cell_off = cell;
        cell += R.nc * R.nc * R.nc;
        R.pp_blk_off = blk;
        blk += (d.n + ppb - 1) / ppb;
        const double dens = 4.0 / 3.0 * M_PI * d.n / (d.box * d.box * d.box);
        const double mean = dens * R.rcl * R.rcl * R.rcl;
        if (mean > maxmean) maxmean = mean;
        R.pbuf = s.prune_buf;
        const double rin = d.rc + R.pbuf;
        if (dens * rin * rin * rin > maxmean_in) maxmean_in = dens * rin * rin * rin;
    }
    s.ncell = cell;
    s.pp_tpi = tpi;
    s.pp_nblk = blk;
    // a multiple of PP_LIST_PAD: the builder pads every list to one
    s.maxnb = ((int)ceil(1.5 * maxmean + 64.0) + PP_LIST_PAD - 1) / PP_LIST_PAD * PP_LIST_PAD;
    s.maxnb_in = s.prune_buf > 0.0
                     ? ((int)ceil(1.5 * maxmean_in + 64.0) + PP_LIST_PAD - 1) / PP_LIST_PAD * PP_LIST_PAD
                     : 0;
    if (s.maxnb_in > s.maxnb) s.maxnb_in = s.maxnb;  // a subset of the outer list
}

extern "C" int p3m_version(void) { return P3M_VERSION; }

extern "C" const char *p3m_last_error(const p3m_ctx *ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

extern "C" int64_t p3m_launch_count(const p3m_ctx *ctx) { return ctx ? ctx->launches : 0; }

extern "C" void *p3m_stream(p3m_ctx *ctx) { return ctx ? (void *)ctx->st : nullptr; }

extern "C" int p3m_destroy(p3m_ctx *ctx)
{
    if (!ctx) return P3M_OK;
    cudaSetDevice(ctx->device);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    drop_graphs(ctx);
    DevState &s = ctx->s;
    void *ptrs[] = {s.reps, s.pos, s.vel, s.acc, s.charge, s.prep, s.cell_key, s.cell_count,
                    s.cell_start, s.cell_cursor, s.cell_tmp, s.cell_perm, s.cell_slot, s.xq, s.nnb,
                    s.cell_sub,
                    s.nlist, s.rebuild, s.rb_list, s.pos_ref, s.pp_tables,
                    s.nnb_in, s.nlist_in, s.prune, s.pos_pref, s.prune_count,
                    s.acc_pp, s.brick_key, s.brick_count, s.brick_start, s.brick_cursor,
                    s.brick_perm, s.brick_slot, s.brick_hist, s.tiles, s.spec, s.ek, s.green, s.efield,
                    s.acc_pm, s.twiddle, s.u_pp_part, s.u_pm_part, s.kin_part, s.rep_out,
                    s.status, ctx->counters, ctx->ring, ctx->qmult, ctx->nqt_part, ctx->snap,
                    ctx->snap_steps,
                    ctx->nqt_ring, ctx->scratch, ctx->ep, ctx->tmp_nq};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (ctx->hbuf) cudaFreeHost(ctx->hbuf);
    if (ctx->h_step) cudaFreeHost(ctx->h_step);
    if (ctx->st2) {
        cudaStreamSynchronize(ctx->st2);
        cudaStreamDestroy(ctx->st2);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->st3) {
        cudaStreamSynchronize(ctx->st3);
        cudaStreamDestroy(ctx->st3);
    }
    if (ctx->ev_join3) cudaEventDestroy(ctx->ev_join3);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
    return P3M_OK;
}

template <typename T> static int alloc_bulk(p3m_ctx *ctx)
{
    using T4 = typename V4<T>::t;
    using C = typename C2<T>::t;
    DevState &s = ctx->s;
    CK(valloc(&s.xq, (size_t)s.ntot * (sizeof(T) == 4 ? sizeof(uint4) : sizeof(ulonglong4))));
    CK(valloc(&s.acc_pp, (size_t)s.ntot * sizeof(T4)));
    if (s.has_mesh) {
        CK(valloc(&s.acc_pm, (size_t)s.ntot * sizeof(T4)));
        CK(valloc(&s.spec, (size_t)s.nspec * sizeof(C)));
        CK(valloc(&s.ek, (size_t)3 * s.nspec * sizeof(C)));
        CK(valloc(&s.green, (size_t)s.nspec * sizeof(T)));
        CK(valloc(&s.efield, (size_t)3 * s.nmesh * sizeof(T)));
        // twiddles exp(-2 pi i k/256), k < 128, from long double
        std::vector<C> tw(128);
        for (int k = 0; k < 128; ++k) {
            long double a = -2.0L * 3.141592653589793238462643383279502884L * k / 256.0L;
            tw[k].x = (T)cosl(a);
            tw[k].y = (T)sinl(a);
        }
        CK(valloc(&s.twiddle, 128 * sizeof(C)));
        CK(cudaMemcpy(s.twiddle, tw.data(), 128 * sizeof(C), cudaMemcpyHostToDevice));
        configure_mesh_kernels<T>();
    }
    configure_pp_kernels<T>();
    configure_integrate_kernels<T>(64);
    return P3M_OK;
}

extern "C" int p3m_create(const p3m_replica_desc *reps, int n_reps, int precision, int device,
                          p3m_ctx **out)
{
    if (!out) return fail(nullptr, P3M_EARG, "p3m_create", "out is NULL");
    *out = nullptr;
    if (!reps || n_reps <= 0) return fail(nullptr, P3M_EARG, "p3m_create", "no replicas");
    if (precision != P3M_FP32 && precision != P3M_FP64)
        return fail(nullptr, P3M_EARG, "p3m_create", "precision must be P3M_FP32 or P3M_FP64");
    int with_mesh = reps[0].mesh > 0;
    for (int r = 0; r < n_reps; ++r) {
        const p3m_replica_desc &d = reps[r];
        char why[256];
        why[0] = 0;
        if (d.n <= 0) snprintf(why, sizeof why, "replica %d: n must be > 0", r);
        else if (!(d.box > 0) || !(d.rc > 0) || !(d.alpha > 0) || !(d.kappa >= 0))
            snprintf(why, sizeof why, "replica %d: box, rc, alpha must be > 0, kappa >= 0", r);
        else if ((int)floor(d.box / d.rc) < 3)
            snprintf(why, sizeof why,
                     "replica %d: floor(L/rc) = %d < 3 (the 27-cell stencil would count pairs twice)",
                     r, (int)floor(d.box / d.rc));
        else if ((d.mesh > 0) != with_mesh)
            snprintf(why, sizeof why, "replica %d: all replicas need a mesh, or none", r);
        else if (d.mesh > 0 && (!is_pow2(d.mesh) || d.mesh < 32 || d.mesh > 256))
            snprintf(why, sizeof why, "replica %d: mesh must be a power of two in [32, 256]", r);
        else if (d.mesh > 0 && d.order != 6)
            snprintf(why, sizeof why, "replica %d: only charge-assignment order 6 is supported", r);
        else if (d.m_alias < 0 || d.m_alias > 7)
            snprintf(why, sizeof why, "replica %d: m_alias must be in [0, 7]", r);
        else if (d.skin > 0.5 * d.rc)
            snprintf(why, sizeof why, "replica %d: skin must be <= rc/2 (negative: default)", r);
        if (why[0]) return fail(nullptr, P3M_EARG, "p3m_create", why);
    }
    p3m_ctx *ctx = new p3m_ctx();
    int rc = check_device(ctx, device);
    if (rc != P3M_OK) {
        g_err = ctx->err;
        delete ctx;
        return rc;
    }
    ctx->device = device;
    ctx->prec = precision;
    ctx->nrep = n_reps;
    ctx->desc.assign(reps, reps + n_reps);
    ctx->green_ready.assign(n_reps, 0);
    DevState &s = ctx->s;
    s.nrep = n_reps;
    s.has_mesh = with_mesh;
    ctx->rh.resize(n_reps);
    long long mesh = 0, spec = 0, tile = 0, hist = 0;
    int nchunk = 0, max_bricks = 0;
    // brick-sort chunks: about 4 per SM over the whole batch (one warp each
    // places its particles), 256 to 4096 particles, a multiple of 32
    long long ntot_all = 0;
    for (int r = 0; r < n_reps; ++r) ntot_all += reps[r].n;
    int sort_ch = (int)std::min<long long>(4096, std::max<long long>(256, (ntot_all + 591) / 592));
    sort_ch = (sort_ch + 31) / 32 * 32;
    s.sort_ch = sort_ch;
    int p = 0, cell = 0, brick = 0, wc_cap = 0, blk = 0, maxm = 0;
    for (int r = 0; r < n_reps; ++r) {
        const p3m_replica_desc &d = reps[r];
        RepDev &R = ctx->rh[r];
        memset(&R, 0, sizeof R);
        R.n = d.n;
        R.p_off = p;
        R.L = d.box;
        R.kappa = d.kappa;
        R.alpha = d.alpha;
        R.rc = d.rc;
        R.dt = d.dt;
        R.t_desired = d.t_desired;
        R.af = d.af;
        R.uf = d.uf;
        R.kf = d.kf;
        R.inv_L = 1.0 / d.box;
        R.qmax = 1.0;
        R.inv_V = 1.0 / (d.box * d.box * d.box);
        R.blk_off = blk;
        R.M = d.mesh;
        if (d.mesh > 0) {
            const int M = d.mesh;
            R.logM = ilog2(M);
            R.h = d.box / M;
            R.inv_h = 1.0 / R.h;
            R.nb = M / BRICK;
            R.brick_off = brick;
            R.mesh_off = mesh;
            R.spec_off = spec;
            R.tile_off = tile;
            R.sc_off = nchunk;
            R.sh_off = hist;
            nchunk += (d.n + sort_ch - 1) / sort_ch;
            hist += (long long)((d.n + sort_ch - 1) / sort_ch) * R.nb * R.nb * R.nb;
            if (R.nb * R.nb * R.nb > max_bricks) max_bricks = R.nb * R.nb * R.nb;
            brick += R.nb * R.nb * R.nb;
            mesh += (long long)M * M * M;
            spec += (long long)(M / 2 + 1) * M * M;
            tile += (long long)R.nb * R.nb * R.nb * TILE3;
            // U_f partials: one per pencil item, more than per plane item
            wc_cap += (M / 2 + 1) * (M / PENCIL > 1 ? M / PENCIL : 1);
            if (M > maxm) maxm = M;
        } else {
            R.brick_off = brick;
        }
        p += d.n;
        {
            const int ncmax = (int)floor(CELL_DIV_MAX * d.box / d.rc);  // the finest grid any setting asks for
            cell += ncmax * ncmax * ncmax;
        }
        blk += (d.n + PBLK - 1) / PBLK;
    }
    {
        int qb = 0;
        for (int r = 0; r < n_reps; ++r) {
            ctx->rh[r].nq_blk_off = qb;
            qb += (reps[r].n + nqt_particles_per_block() - 1) / nqt_particles_per_block();
        }
        s.nq_nblk = qb;
    }
    s.ntot = p;
    ctx->ncell_cap = cell;
    s.nbrick = brick;
    s.nmesh = mesh;
    s.nspec = spec;
    s.ntile = tile;
    s.plane_max = plane_max_mesh();
    s.gather_mode = 1;
    plan_mesh_passes(ctx);
    s.nblk = blk;
    s.max_mesh = maxm;
    plan_lists(ctx, -1.0, p >= 148 * 256 * 2 ? 1 : (p >= 148 * 64 ? 2 : 4));

    auto cleanup = [&](int code) {
        std::string e = ctx->err;
        p3m_destroy(ctx);
        g_err = e;
        return code;
    };
#define CKC(call)                                                            \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) {                                             \
            fail(ctx, P3M_ECUDA, #call, cudaGetErrorString(e_));             \
            return cleanup(P3M_ECUDA);                                       \
        }                                                                    \
    } while (0)
    CKC(cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking));
    CKC(cudaStreamCreateWithFlags(&ctx->st2, cudaStreamNonBlocking));
    CKC(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    CKC(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
    CKC(cudaStreamCreateWithFlags(&ctx->st3, cudaStreamNonBlocking));
    CKC(cudaEventCreateWithFlags(&ctx->ev_join3, cudaEventDisableTiming));
    CKC(dalloc(&s.reps, n_reps));
    CKC(cudaMemcpy(s.reps, ctx->rh.data(), sizeof(RepDev) * n_reps, cudaMemcpyHostToDevice));
    {
        std::vector<float4> tab((size_t)n_reps * PP_TABLE_N);
        for (int r = 0; r < n_reps; ++r) build_pp_table(reps[r], tab.data() + (size_t)r * PP_TABLE_N);
        CKC(dalloc(&s.pp_tables, tab.size()));
        CKC(cudaMemcpy(s.pp_tables, tab.data(), sizeof(float4) * tab.size(), cudaMemcpyHostToDevice));
    }
    CKC(dalloc(&s.pos, (size_t)3 * p));
    CKC(dalloc(&s.vel, (size_t)3 * p));
    CKC(dalloc(&s.acc, (size_t)3 * p));
    CKC(dalloc(&s.charge, (size_t)p));
    {
        std::vector<double> ones(p, 1.0);
        CKC(cudaMemcpy(s.charge, ones.data(), sizeof(double) * p, cudaMemcpyHostToDevice));
        std::vector<int> pr(p);
        for (int r = 0; r < n_reps; ++r)
            for (int i = 0; i < reps[r].n; ++i) pr[ctx->rh[r].p_off + i] = r;
        CKC(dalloc(&s.prep, (size_t)p));
        CKC(cudaMemcpy(s.prep, pr.data(), sizeof(int) * p, cudaMemcpyHostToDevice));
    }
    CKC(dalloc(&s.cell_key, (size_t)p));
    CKC(dalloc(&s.cell_count, (size_t)ctx->ncell_cap));
    CKC(dalloc(&s.cell_start, (size_t)ctx->ncell_cap + 1));
    CKC(dalloc(&s.cell_cursor, (size_t)ctx->ncell_cap));
    CKC(dalloc(&s.nnb, (size_t)p));
    CKC(dalloc(&s.cell_sub, (size_t)p));
    ctx->nlist_cap = (long long)((p + 31) / 32) * 32 * s.maxnb;
    CKC(dalloc(&s.nlist, (size_t)ctx->nlist_cap));
    CKC(dalloc(&s.rebuild, (size_t)n_reps));
    CKC(dalloc(&s.rb_list, (size_t)2 * n_reps + 2));
    CKC(dalloc(&s.pos_ref, (size_t)3 * p));
    CKC(dalloc(&s.prune, (size_t)n_reps));
    CKC(dalloc(&s.nnb_in, (size_t)p));
    CKC(dalloc(&s.pos_pref, (size_t)3 * p));
    CKC(dalloc(&s.prune_count, (size_t)n_reps));
    CKC(dalloc(&s.cell_tmp, (size_t)p));
    CKC(dalloc(&s.cell_perm, (size_t)p));
    CKC(dalloc(&s.cell_slot, (size_t)p));
    CKC(dalloc(&s.brick_key, (size_t)p));
    CKC(dalloc(&s.brick_count, (size_t)brick));
    CKC(dalloc(&s.brick_start, (size_t)brick + 1));
    CKC(dalloc(&s.brick_cursor, (size_t)brick));
    CKC(dalloc(&s.brick_perm, (size_t)p));
    s.nchunk = nchunk;
    s.max_bricks = max_bricks;
    CKC(dalloc(&s.brick_hist, (size_t)hist));
    CKC(dalloc(&s.brick_slot, (size_t)p));
    if (with_mesh)
        CKC(valloc(&s.tiles, (size_t)tile * (precision == P3M_FP32 ? sizeof(float) : sizeof(double))));
    {
        int nb8 = 0;
        for (int r = 0; r < n_reps; ++r) nb8 += (reps[r].n + pp_particles_per_block(8) - 1) / pp_particles_per_block(8);
        ctx->pp_nblk_cap = nb8;
        CKC(dalloc(&s.u_pp_part, (size_t)nb8));
    }
    CKC(dalloc(&s.u_pm_part, (size_t)wc_cap));
    CKC(dalloc(&s.kin_part, (size_t)blk));
    CKC(dalloc(&s.rep_out, (size_t)8 * n_reps));
    CKC(dalloc(&s.status, 1));
    CKC(dalloc(&ctx->counters, 8));
    ctx->ring_cap = 8192;
    CKC(dalloc(&ctx->ring, (size_t)ctx->ring_cap * n_reps * 4));
    {
        size_t sc = (size_t)3 * maxm * maxm * maxm;
        size_t gfb = (size_t)gf_opt_blocks(maxm > 0 ? maxm : 1);
        CKC(dalloc(&ctx->scratch, (sc > gfb ? sc : gfb) + gfb + 16));
    }
    CKC(dalloc(&ctx->ep, (size_t)3 * p));
    int arc = (precision == P3M_FP32) ? alloc_bulk<float>(ctx) : alloc_bulk<double>(ctx);
    if (arc != P3M_OK) return cleanup(arc);
    launch_set_flags(s.rebuild, n_reps, 1, ctx->st);  // no lists exist yet
    CKC(cudaGetLastError());
    CKC(cudaDeviceSynchronize());
#undef CKC
    *out = ctx;
    return P3M_OK;
}

// ---------------------------------------------------------------------------
// internal sequences (enqueue only)
// ---------------------------------------------------------------------------

// Cell sort and list build. keys = true (compat calls, initial forces):
// force a rebuild and key every particle here. keys = false (inside a step):
// the drift kernel keyed the bricks and raised the rebuild flag if needed;
// the cell part runs only when the flag is set.
template <typename T> static void seq_sort(p3m_ctx *ctx, bool keys)
{
    DevState &s = ctx->s;
    if (keys) {
        launch_set_flags(s.rebuild, s.nrep, 1, ctx->st);
        launch_keys<T>(s, ctx->st);
        ctx->launches += 2;
    } else {
        launch_cell_keys(s, ctx->st);
        ctx->launches++;
    }
    launch_scan(s, ctx->st);
    launch_scatter(s, ctx->st);
    launch_fix_cells<T>(s, ctx->st);
    launch_quantize<T>(s, ctx->st);     // sorted coordinates of this step
    launch_build_lists<T>(s, ctx->st);  // from those coordinates (rebuild steps)
    ctx->launches += 5;
    if (s.has_mesh) {
        launch_sort_bricks(s, ctx->st);
        ctx->launches += 3;
    }
}

// reduce = false: leave the energy partials to k_step_reduce (inside a step)
template <typename T> static void seq_pp(p3m_ctx *ctx, bool reduce = true, cudaStream_t st = nullptr)
{
    if (!st) st = ctx->st;
    launch_pp<T>(ctx->s, st);
    ctx->launches++;
    if (reduce) {
        launch_reduce_pp(ctx->s, st);
        ctx->launches++;
    }
}

template <typename T> static void seq_pm(p3m_ctx *ctx, bool reduce = true, cudaStream_t st = nullptr)
{
    if (!st) st = ctx->st;
    DevState &s = ctx->s;
    launch_assign<T>(s, st);
    launch_fft_forward<T>(s, st);
    if (reduce) {
        launch_reduce_pm(s, st);
        ctx->launches++;
    }
    launch_fft_inverse<T>(s, st);
    launch_gather<T>(s, st);
    ctx->launches += 2 + fft_kernel_count(s);
}

// Compute the influence function of every replica that has none yet.
template <typename T> static int ensure_green(p3m_ctx *ctx)
{
    for (int r = 0; r < ctx->nrep; ++r) {
        if (ctx->green_ready[r] || ctx->rh[r].M == 0) continue;
        const p3m_replica_desc &d = ctx->desc[r];
        launch_gf_opt(d.kappa, d.alpha, d.order, d.m_alias, d.mesh, d.box, ctx->scratch,
                      ctx->scratch + (size_t)3 * ctx->s.max_mesh * ctx->s.max_mesh * ctx->s.max_mesh,
                      ctx->st);
        launch_green_from_host_layout<T>(ctx->s, r, ctx->scratch, ctx->st);
        ctx->launches += 2;
        ctx->green_ready[r] = 1;
    }
    CK(cudaGetLastError());
    return P3M_OK;
}

// One full force evaluation of the current device positions: sort (with or
// without the key pass), PP, PM. Leaves acc_pp / acc_pm and U parts.
template <typename T> static int seq_force(p3m_ctx *ctx, bool keys)
{
    if (ctx->s.has_mesh) {
        int rc = ensure_green<T>(ctx);
        if (rc != P3M_OK) return rc;
    }
    seq_sort<T>(ctx, keys);
    seq_pp<T>(ctx);
    if (ctx->s.has_mesh) seq_pm<T>(ctx);
    return P3M_OK;
}

// One integrator step of every replica (mode 0 NVE, 1 thermostat). After the
// drift (which keys the particles' bricks) the step forks: the mesh branch
// (brick scan and sort, assignment, FFTs, gather) runs on a second stream and
// the n(q,t) sums of the new positions on a third, while the particle branch
// (cell keys and scan, cell sort, lists, PP) runs on the first -- they share
// no arrays -- and they join before the forces are combined, so the
// latency-bound kernels of each branch fill the SMs the others leave idle
// (one graph holds all branches).
template <typename T> static int seq_step(p3m_ctx *ctx, int mode, int record_nqt)
{
    DevState &s = ctx->s;
    cudaStream_t st = ctx->st, st2 = ctx->st2;
    launch_kick_drift(s, st);
    ctx->launches++;
    const int rec = (record_nqt && ctx->nq > 0) ? 1 : 0;
    const bool fork = s.has_mesh || rec;
    cudaError_t e = cudaSuccess;
    if (fork) {
        e = cudaEventRecord(ctx->ev_fork, st);
        if (e == cudaSuccess && s.has_mesh) {
            e = cudaStreamWaitEvent(st2, ctx->ev_fork, 0);
            if (e == cudaSuccess) {
                launch_scan(s, st2, 1);
                launch_sort_bricks(s, st2);
                ctx->launches += 4;
                seq_pm<T>(ctx, false, st2);
                e = cudaEventRecord(ctx->ev_join, st2);
            }
        }
        if (e == cudaSuccess && rec) {  // the new positions are final: ring row counters[3]
            // (the reduction advances counters[3] after the join)
            e = cudaStreamWaitEvent(ctx->st3, ctx->ev_fork, 0);
            if (e == cudaSuccess) {
                launch_nqt<T>(s, s.pos, ctx->qmult, ctx->nq, ctx->nq_consecutive, ctx->nqt_part,
                              ctx->nqt_ring, ctx->counters, ctx->nqt_cap, ctx->st3);
                ctx->launches += 2;
                e = cudaEventRecord(ctx->ev_join3, ctx->st3);
            }
        }
    }
    launch_cell_keys(s, st);
    launch_scan(s, st, s.has_mesh ? 0 : -1);  // without a mesh branch: the bricks here too
    launch_scatter(s, st);
    launch_fix_cells<T>(s, st);
    launch_quantize<T>(s, st);     // sorted coordinates of this step
    launch_build_lists<T>(s, st);  // from those coordinates (rebuild steps)
    ctx->launches += 6;
    seq_pp<T>(ctx, false, st);
    if (e == cudaSuccess && s.has_mesh) e = cudaStreamWaitEvent(st, ctx->ev_join, 0);
    if (e == cudaSuccess && rec) e = cudaStreamWaitEvent(st, ctx->ev_join3, 0);
    launch_kick_finish<T>(s, 1, nullptr, st);
    ctx->launches++;
    StepSums sums;  // the energy sums, in the reduction (the n(q,t) row is summed on its branch)
    sums.u_pp_part = s.u_pp_part;
    sums.pp_nblk = s.pp_nblk;
    sums.u_pm_part = s.u_pm_part;
    sums.wc_total = s.wc;
    sums.wp_total = s.wp;
    launch_step_reduce(s, mode, ctx->counters, ctx->ring, ctx->ring_cap, st, rec,
                       ctx->snap_interval, ctx->snap_cap, sums);
    ctx->launches++;
    if (mode == P3M_MODE_THERMOSTAT) {
        launch_scale_vel(s, st);
        ctx->launches++;
    }
    if (ctx->snap_interval > 0) {  // after the thermostat's rescale: the step's final state
        launch_snapshot(s, ctx->counters, ctx->snap, ctx->snap_steps, st);
        ctx->launches++;
    }
    if (e != cudaSuccess) return fail(ctx, P3M_ECUDA, "step fork/join", cudaGetErrorString(e));
    return P3M_OK;
}

// ---------------------------------------------------------------------------
// host staging helpers
// ---------------------------------------------------------------------------

// Host <-> device copies on the context's stream (callers synchronise in
// finish()).
static int h2d(p3m_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    if (!bytes) return P3M_OK;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->st));
    return P3M_OK;
}

static int d2h(p3m_ctx *ctx, void *dst, const void *src, size_t bytes)
{
    if (!bytes) return P3M_OK;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->st));
    return P3M_OK;
}

// A device status word read back: clear it on the device and report it.
static int status_error(p3m_ctx *ctx, int st)
{
    if (!st) return P3M_OK;
    CK(cudaMemset(ctx->s.status, 0, sizeof(int)));
    // a non-finite velocity also makes a non-finite position: name the cause
    if (st & ST_NONFINITE)
        return fail(ctx, P3M_ENONFINITE, "non-finite velocity, force or energy", "");
    if (st & ST_BOX) return fail(ctx, P3M_EBOX, "particle outside [-L, 2L) or non-finite position", "");
    if (st & ST_NBOVF)
        return fail(ctx, P3M_ENBOVF, "a particle has more neighbours than the list holds",
                    "raise the capacity with a smaller skin or report the density");
    return P3M_OK;
}

static int finish(p3m_ctx *ctx)
{
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    int st = 0;
    CK(cudaMemcpy(&st, ctx->s.status, sizeof(int), cudaMemcpyDeviceToHost));
    return status_error(ctx, st);
}

static int compat_check(p3m_ctx *ctx, int replica)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (ctx->nrep != 1 || replica != 0)
        return fail(ctx, P3M_EARG, "compat call", "needs a single-replica context and replica 0");
    CK(cudaSetDevice(ctx->device));
    return P3M_OK;
}

// Charges of a single-replica context (the compat calls); NULL keeps the
// current ones. The replica's largest |Z| bounds the assignment's fixed point.
static int upload_charge(p3m_ctx *ctx, const double *Z)
{
    const int n = ctx->s.ntot;
    if (!Z) return P3M_OK;
    double qmax = 0.0;
    for (int i = 0; i < n; ++i) {
        if (!std::isfinite(Z[i])) return fail(ctx, P3M_EARG, "charges", "not finite");
        qmax = fmax(qmax, fabs(Z[i]));
    }
    if (!(qmax < 1e300)) return fail(ctx, P3M_EARG, "charges", "too large");
    if (qmax != ctx->rh[0].qmax) {
        ctx->rh[0].qmax = qmax > 0.0 ? qmax : 1.0;
        CK(cudaMemcpyAsync(&ctx->s.reps[0].qmax, &ctx->rh[0].qmax, sizeof(double),
                           cudaMemcpyHostToDevice, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    return h2d(ctx, ctx->s.charge, Z, sizeof(double) * n);
}

#define DISPATCH(fn, ...) (ctx->prec == P3M_FP32 ? fn<float>(__VA_ARGS__) : fn<double>(__VA_ARGS__))
#define RET(x) do { int rc_ = (x); if (rc_ != P3M_OK) return rc_; } while (0)

// ---------------------------------------------------------------------------
// compat entry points
// ---------------------------------------------------------------------------

template <typename T> static int do_pp(p3m_ctx *ctx, const double *pos, double *acc, double *U)
{
    DevState &s = ctx->s;
    RET(h2d(ctx, s.pos, pos, sizeof(double) * 3 * s.ntot));
    seq_sort<T>(ctx, true);
    seq_pp<T>(ctx);
    launch_combine<T>(s, 1, 0, 0, s.acc, nullptr, ctx->st);
    ctx->launches++;
    RET(d2h(ctx, acc, s.acc, sizeof(double) * 3 * s.ntot));
    double ro[8];
    RET(d2h(ctx, ro, s.rep_out, sizeof ro));
    RET(finish(ctx));
    *U = ro[RO_UPP];
    return P3M_OK;
}

extern "C" int p3m_pp(p3m_ctx *ctx, int replica, const double *pos, double *acc, double *U)
{
    RET(compat_check(ctx, replica));
    if (!pos || !acc || !U) return fail(ctx, P3M_EARG, "p3m_pp", "NULL argument");
    return DISPATCH(do_pp, ctx, pos, acc, U);
}

static int need_mesh(p3m_ctx *ctx, const char *who)
{
    if (!ctx->s.has_mesh) return fail(ctx, P3M_EARG, who, "context has no mesh");
    return P3M_OK;
}

template <typename T> static int do_assign(p3m_ctx *ctx, const double *pos, const double *Z, double *rho)
{
    DevState &s = ctx->s;
    const int M = ctx->rh[0].M;
    RET(h2d(ctx, s.pos, pos, sizeof(double) * 3 * s.ntot));
    RET(upload_charge(ctx, Z));
    seq_sort<T>(ctx, true);
    launch_assign<T>(s, ctx->st);
    launch_tiles_to_mesh<T>(s, 0, ctx->scratch, ctx->st);
    ctx->launches += 2;
    RET(d2h(ctx, rho, ctx->scratch, sizeof(double) * M * M * M));
    return finish(ctx);
}

extern "C" int p3m_assign(p3m_ctx *ctx, int replica, const double *pos, const double *Z, double *rho)
{
    RET(compat_check(ctx, replica));
    RET(need_mesh(ctx, "p3m_assign"));
    if (!pos || !rho) return fail(ctx, P3M_EARG, "p3m_assign", "NULL argument");
    return DISPATCH(do_assign, ctx, pos, Z, rho);
}

template <typename T>
static int do_gather(p3m_ctx *ctx, const double *pos, const double *Z, const double *Ex,
                     const double *Ey, const double *Ez, double *acc, double *Ep)
{
    DevState &s = ctx->s;
    const size_t M3 = (size_t)ctx->rh[0].M * ctx->rh[0].M * ctx->rh[0].M;
    RET(h2d(ctx, s.pos, pos, sizeof(double) * 3 * s.ntot));
    RET(upload_charge(ctx, Z));
    RET(h2d(ctx, ctx->scratch, Ex, sizeof(double) * M3));
    RET(h2d(ctx, ctx->scratch + M3, Ey, sizeof(double) * M3));
    RET(h2d(ctx, ctx->scratch + 2 * M3, Ez, sizeof(double) * M3));
    launch_efield_from_mesh<T>(s, 0, ctx->scratch, ctx->scratch + M3, ctx->scratch + 2 * M3, ctx->st);
    ctx->launches++;
    seq_sort<T>(ctx, true);
    launch_gather<T>(s, ctx->st);
    launch_combine<T>(s, 0, 1, 0, s.acc, ctx->ep, ctx->st);
    ctx->launches += 2;
    RET(d2h(ctx, acc, s.acc, sizeof(double) * 3 * s.ntot));
    RET(finish(ctx));
    if (Ep) {
        std::vector<double> e(3 * (size_t)s.ntot);
        CK(cudaMemcpy(e.data(), ctx->ep, sizeof(double) * e.size(), cudaMemcpyDeviceToHost));
        for (int i = 0; i < s.ntot; ++i)
            for (int d = 0; d < 3; ++d) Ep[(size_t)d * s.ntot + i] = e[3 * (size_t)i + d];
    }
    return P3M_OK;
}

extern "C" int p3m_gather(p3m_ctx *ctx, int replica, const double *pos, const double *Z,
                          const double *Ex, const double *Ey, const double *Ez, double *acc,
                          double *Ep)
{
    RET(compat_check(ctx, replica));
    RET(need_mesh(ctx, "p3m_gather"));
    if (!pos || !Ex || !Ey || !Ez || !acc) return fail(ctx, P3M_EARG, "p3m_gather", "NULL argument");
    return DISPATCH(do_gather, ctx, pos, Z, Ex, Ey, Ez, acc, Ep);
}

extern "C" int p3m_gf_opt(int device, double kappa, double alpha, int p, int m_alias, int M,
                          double box, double *G_k, double *A_pm)
{
    p3m_ctx *ctx = nullptr;
    if (!G_k || !A_pm) return fail(nullptr, P3M_EARG, "p3m_gf_opt", "NULL argument");
    if (M < 2 || M > 1024 || !(box > 0) || !(alpha > 0) || p < 1 || m_alias < 0 || m_alias > 7)
        return fail(nullptr, P3M_EARG, "p3m_gf_opt", "bad size or parameter");
    int rc = check_device(nullptr, device);
    if (rc != P3M_OK) return rc;
    const size_t n = (size_t)M * M * M;
    const int nb = gf_opt_blocks(M);
    double *d_g = nullptr, *d_a = nullptr;
    CK(cudaMalloc(&d_g, n * sizeof(double)));
    cudaError_t e = cudaMalloc(&d_a, nb * sizeof(double));
    if (e != cudaSuccess) {
        cudaFree(d_g);
        return fail(nullptr, P3M_ECUDA, "cudaMalloc", cudaGetErrorString(e));
    }
    launch_gf_opt(kappa, alpha, p, m_alias, M, box, d_g, d_a, 0);
    std::vector<double> a(nb);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(G_k, d_g, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(a.data(), d_a, nb * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_g);
    cudaFree(d_a);
    if (e != cudaSuccess) return fail(nullptr, P3M_ECUDA, "p3m_gf_opt", cudaGetErrorString(e));
    double s = 0.0;
    for (int k = 0; k < nb; ++k) s += a[k];
    *A_pm = s;
    return P3M_OK;
}

template <typename T> static int do_set_green(p3m_ctx *ctx, int replica, const double *G_k)
{
    const RepDev &R = ctx->rh[replica];
    if (!G_k) {
        ctx->green_ready[replica] = 0;
        return ensure_green<T>(ctx);
    }
    const size_t M3 = (size_t)R.M * R.M * R.M;
    RET(h2d(ctx, ctx->scratch, G_k, sizeof(double) * M3));
    launch_green_from_host_layout<T>(ctx->s, replica, ctx->scratch, ctx->st);
    ctx->launches++;
    ctx->green_ready[replica] = 1;
    return finish(ctx);
}

extern "C" int p3m_set_green(p3m_ctx *ctx, int replica, const double *G_k)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (replica < 0 || replica >= ctx->nrep) return fail(ctx, P3M_EARG, "p3m_set_green", "replica");
    RET(need_mesh(ctx, "p3m_set_green"));
    CK(cudaSetDevice(ctx->device));
    return DISPATCH(do_set_green, ctx, replica, G_k);
}

template <typename T>
static int do_pm(p3m_ctx *ctx, const double *pos, const double *Z, double *acc, double *U,
                 double *Ep, double *rho)
{
    DevState &s = ctx->s;
    const int M = ctx->rh[0].M;
    RET(ensure_green<T>(ctx));
    RET(h2d(ctx, s.pos, pos, sizeof(double) * 3 * s.ntot));
    RET(upload_charge(ctx, Z));
    seq_sort<T>(ctx, true);
    seq_pm<T>(ctx);
    launch_combine<T>(s, 0, 1, 0, s.acc, ctx->ep, ctx->st);
    ctx->launches++;
    if (rho) {
        launch_tiles_to_mesh<T>(s, 0, ctx->scratch, ctx->st);
        ctx->launches++;
        RET(d2h(ctx, rho, ctx->scratch, sizeof(double) * M * M * M));
    }
    RET(d2h(ctx, acc, s.acc, sizeof(double) * 3 * s.ntot));
    double ro[8];
    RET(d2h(ctx, ro, s.rep_out, sizeof ro));
    RET(finish(ctx));
    *U = ro[RO_UPM];
    if (Ep) {
        std::vector<double> e(3 * (size_t)s.ntot);
        CK(cudaMemcpy(e.data(), ctx->ep, sizeof(double) * e.size(), cudaMemcpyDeviceToHost));
        for (int i = 0; i < s.ntot; ++i)
            for (int d = 0; d < 3; ++d) Ep[(size_t)d * s.ntot + i] = e[3 * (size_t)i + d];
    }
    return P3M_OK;
}

extern "C" int p3m_pm(p3m_ctx *ctx, int replica, const double *pos, const double *Z, double *acc,
                      double *U, double *Ep, double *rho)
{
    RET(compat_check(ctx, replica));
    RET(need_mesh(ctx, "p3m_pm"));
    if (!pos || !acc || !U) return fail(ctx, P3M_EARG, "p3m_pm", "NULL argument");
    return DISPATCH(do_pm, ctx, pos, Z, acc, U, Ep, rho);
}

template <typename T>
static int do_force(p3m_ctx *ctx, const double *pos, const double *Z, double *acc, double *U,
                    double *parts)
{
    DevState &s = ctx->s;
    RET(h2d(ctx, s.pos, pos, sizeof(double) * 3 * s.ntot));
    RET(upload_charge(ctx, Z));
    RET(seq_force<T>(ctx, true));
    launch_kick_finish<T>(s, 0, nullptr, ctx->st);
    launch_step_reduce(s, 2, ctx->counters, nullptr, 0, ctx->st);
    ctx->launches += 2;
    RET(d2h(ctx, acc, s.acc, sizeof(double) * 3 * s.ntot));
    double ro[8];
    RET(d2h(ctx, ro, s.rep_out, sizeof ro));
    RET(finish(ctx));
    *U = ro[RO_U];
    if (parts) {
        parts[0] = ro[RO_UPP];
        parts[1] = ro[RO_UPM];
        parts[2] = ro[RO_USELF];
    }
    return P3M_OK;
}

extern "C" int p3m_force(p3m_ctx *ctx, int replica, const double *pos, const double *Z,
                         double *acc, double *U, double *parts)
{
    RET(compat_check(ctx, replica));
    if (!pos || !acc || !U) return fail(ctx, P3M_EARG, "p3m_force", "NULL argument");
    return DISPATCH(do_force, ctx, pos, Z, acc, U, parts);
}

template <typename T>
static int do_update(p3m_ctx *ctx, int mode, int it, double *pos, double *vel, double *acc,
                     double *U, double *Tout)
{
    DevState &s = ctx->s;
    const size_t b = sizeof(double) * 3 * s.ntot;
    RET(h2d(ctx, s.pos, pos, b));
    RET(h2d(ctx, s.vel, vel, b));
    RET(h2d(ctx, s.acc, acc, b));
    if (s.has_mesh) RET(ensure_green<T>(ctx));
    launch_set_counters(ctx->counters, 0, -1, it, ctx->st);
    launch_set_flags(s.rebuild, s.nrep, 1, ctx->st);  // the caller's arrays may hold any state
    ctx->launches += 2;
    RET(seq_step<T>(ctx, mode, 0));
    RET(d2h(ctx, pos, s.pos, b));
    RET(d2h(ctx, vel, s.vel, b));
    RET(d2h(ctx, acc, s.acc, b));
    double ro[8];
    RET(d2h(ctx, ro, s.rep_out, sizeof ro));
    RET(finish(ctx));
    *U = ro[RO_U];
    if (Tout) *Tout = ro[RO_T];
    return P3M_OK;
}

extern "C" int p3m_update(p3m_ctx *ctx, int replica, double *pos, double *vel, double *acc, double *U)
{
    RET(compat_check(ctx, replica));
    if (!pos || !vel || !acc || !U) return fail(ctx, P3M_EARG, "p3m_update", "NULL argument");
    return DISPATCH(do_update, ctx, P3M_MODE_NVE, 0, pos, vel, acc, U, nullptr);
}

extern "C" int p3m_vscale(p3m_ctx *ctx, int replica, int it, double *pos, double *vel, double *acc,
                          double *U, double *T)
{
    RET(compat_check(ctx, replica));
    if (!pos || !vel || !acc || !U) return fail(ctx, P3M_EARG, "p3m_vscale", "NULL argument");
    return DISPATCH(do_update, ctx, P3M_MODE_THERMOSTAT, it, pos, vel, acc, U, T);
}

template <typename T>
static int do_nqt(p3m_ctx *ctx, int replica, const double *pos, const double *qv, int nq, double *out)
{
    DevState &s = ctx->s;
    const RepDev &R = ctx->rh[replica];
    if (nq > 64) return fail(ctx, P3M_EARG, "p3m_nqt", "nq must be <= 64");
    if (ctx->tmp_nq_cap < nq) {
        if (ctx->tmp_nq) cudaFree(ctx->tmp_nq);
        ctx->tmp_nq = nullptr;
        CK(dalloc(&ctx->tmp_nq, (size_t)ctx->nrep * 64 * 6 + (size_t)s.nblk * 64 * 6 + 64));
        ctx->tmp_nq_cap = 64;
    }
    double *qm = ctx->tmp_nq;
    double *part = qm + 64;
    double *o = part + (size_t)s.nblk * 64 * 6;
    std::vector<double> qmult(nq);
    for (int k = 0; k < nq; ++k) qmult[k] = qv[k] * R.L / (2.0 * 3.141592653589793238);
    RET(h2d(ctx, s.pos + 3 * (size_t)R.p_off, pos, sizeof(double) * 3 * R.n));
    CK(cudaMemcpyAsync(qm, qmult.data(), sizeof(double) * nq, cudaMemcpyHostToDevice, ctx->st));
    launch_nqt<T>(s, s.pos, qm, nq, 0, part, o, nullptr, 0, ctx->st);
    ctx->launches += 2;
    RET(d2h(ctx, out, o + (size_t)replica * nq * 6, sizeof(double) * nq * 6));
    RET(finish(ctx));
    // (nq, 3) complex: reorder [iq][axis][re,im] is already the layout
    return P3M_OK;
}

extern "C" int p3m_nqt(p3m_ctx *ctx, int replica, const double *pos, const double *qv, int nq,
                       double *out)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (replica < 0 || replica >= ctx->nrep || !pos || !qv || !out || nq <= 0)
        return fail(ctx, P3M_EARG, "p3m_nqt", "bad argument");
    CK(cudaSetDevice(ctx->device));
    return DISPATCH(do_nqt, ctx, replica, pos, qv, nq, out);
}

// ---------------------------------------------------------------------------
// device-resident path
// ---------------------------------------------------------------------------

extern "C" int p3m_set_state(p3m_ctx *ctx, int replica, const double *pos, const double *vel,
                             const double *acc)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (replica < 0 || replica >= ctx->nrep) return fail(ctx, P3M_EARG, "p3m_set_state", "replica");
    CK(cudaSetDevice(ctx->device));
    const RepDev &R = ctx->rh[replica];
    const size_t o = 3 * (size_t)R.p_off, b = sizeof(double) * 3 * R.n;
    if (pos) RET(h2d(ctx, ctx->s.pos + o, pos, b));
    if (vel) RET(h2d(ctx, ctx->s.vel + o, vel, b));
    if (acc) RET(h2d(ctx, ctx->s.acc + o, acc, b));
    if (pos) launch_set_flags(ctx->s.rebuild, ctx->s.nrep, 1, ctx->st);
    ctx->state_set = true;
    return finish(ctx);
}

extern "C" int p3m_get_state(p3m_ctx *ctx, int replica, double *pos, double *vel, double *acc)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (replica < 0 || replica >= ctx->nrep) return fail(ctx, P3M_EARG, "p3m_get_state", "replica");
    CK(cudaSetDevice(ctx->device));
    const RepDev &R = ctx->rh[replica];
    const size_t o = 3 * (size_t)R.p_off, b = sizeof(double) * 3 * R.n;
    if (pos) RET(d2h(ctx, pos, ctx->s.pos + o, b));
    if (vel) RET(d2h(ctx, vel, ctx->s.vel + o, b));
    if (acc) RET(d2h(ctx, acc, ctx->s.acc + o, b));
    return finish(ctx);
}

static int set_state_all(p3m_ctx *ctx, const double *pos, const double *vel, const double *acc,
                         int keep_lists, bool sync)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    CK(cudaSetDevice(ctx->device));
    const size_t b = sizeof(double) * 3 * (size_t)ctx->s.ntot;
    if (pos) RET(h2d(ctx, ctx->s.pos, pos, b));
    if (vel) RET(h2d(ctx, ctx->s.vel, vel, b));
    if (acc) RET(h2d(ctx, ctx->s.acc, acc, b));
    if (pos && !keep_lists) launch_set_flags(ctx->s.rebuild, ctx->s.nrep, 1, ctx->st);
    ctx->state_set = true;
    if (!sync) {
        CK(cudaGetLastError());
        return P3M_OK;
    }
    return finish(ctx);
}

static int get_state_all(p3m_ctx *ctx, double *pos, double *vel, double *acc, bool sync)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    CK(cudaSetDevice(ctx->device));
    const size_t b = sizeof(double) * 3 * (size_t)ctx->s.ntot;
    if (pos) RET(d2h(ctx, pos, ctx->s.pos, b));
    if (vel) RET(d2h(ctx, vel, ctx->s.vel, b));
    if (acc) RET(d2h(ctx, acc, ctx->s.acc, b));
    if (!sync) {
        CK(cudaGetLastError());
        return P3M_OK;
    }
    return finish(ctx);
}

extern "C" int p3m_set_state_all(p3m_ctx *ctx, const double *pos, const double *vel,
                                 const double *acc, int keep_lists)
{
    return set_state_all(ctx, pos, vel, acc, keep_lists, true);
}

extern "C" int p3m_get_state_all(p3m_ctx *ctx, double *pos, double *vel, double *acc)
{
    return get_state_all(ctx, pos, vel, acc, true);
}

extern "C" int p3m_set_state_all_async(p3m_ctx *ctx, const double *pos, const double *vel,
                                       const double *acc, int keep_lists)
{
    return set_state_all(ctx, pos, vel, acc, keep_lists, false);
}

extern "C" int p3m_get_state_all_async(p3m_ctx *ctx, double *pos, double *vel, double *acc)
{
    return get_state_all(ctx, pos, vel, acc, false);
}

extern "C" int p3m_get_step_async(p3m_ctx *ctx, double *pos, double *vel, double *acc,
                                  double *energies)
{
    RET(get_state_all(ctx, pos, vel, acc, false));
    const size_t nrep = (size_t)ctx->nrep;
    if (!ctx->h_step) CK(cudaHostAlloc(&ctx->h_step, sizeof(double) * (8 * nrep + 1), cudaHostAllocDefault));
    CK(cudaMemcpyAsync(ctx->h_step, ctx->s.rep_out, sizeof(double) * 8 * nrep, cudaMemcpyDeviceToHost,
                       ctx->st));
    CK(cudaMemcpyAsync(ctx->h_step + 8 * nrep, ctx->s.status, sizeof(int), cudaMemcpyDeviceToHost,
                       ctx->st));
    ctx->step_out = energies;
    ctx->step_pending = true;
    ctx->step_launches = ctx->launches;
    return P3M_OK;
}

template <typename T> static int do_init_forces(p3m_ctx *ctx)
{
    RET(seq_force<T>(ctx, true));
    launch_kick_finish<T>(ctx->s, 0, nullptr, ctx->st);
    launch_step_reduce(ctx->s, 2, ctx->counters, nullptr, 0, ctx->st);
    ctx->launches += 2;
    return finish(ctx);
}

extern "C" int p3m_init_forces(p3m_ctx *ctx)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    CK(cudaSetDevice(ctx->device));
    return DISPATCH(do_init_forces, ctx);
}

extern "C" int p3m_set_nqt(p3m_ctx *ctx, const double *qmult, int nq, int capacity)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (nq < 0 || nq > 64 || (nq > 0 && (!qmult || capacity <= 0)))
        return fail(ctx, P3M_EARG, "p3m_set_nqt", "need 0 <= nq <= 64 and capacity > 0");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    if (ctx->qmult) cudaFree(ctx->qmult);
    if (ctx->nqt_part) cudaFree(ctx->nqt_part);
    if (ctx->nqt_ring) cudaFree(ctx->nqt_ring);
    ctx->qmult = ctx->nqt_part = ctx->nqt_ring = nullptr;
    drop_graphs(ctx, true);
    ctx->nq = nq;
    ctx->nqt_cap = capacity;
    ctx->nqt_rows = 0;
    if (nq == 0) return P3M_OK;
    CK(dalloc(&ctx->qmult, (size_t)nq));
    CK(cudaMemcpy(ctx->qmult, qmult, sizeof(double) * nq, cudaMemcpyHostToDevice));
    ctx->nq_consecutive = 1;
    for (int k = 0; k < nq; ++k)
        if (qmult[k] != (double)(k + 1)) ctx->nq_consecutive = 0;
    CK(dalloc(&ctx->nqt_part, (size_t)ctx->s.nq_nblk * nq * 6));
    CK(dalloc(&ctx->nqt_ring, (size_t)capacity * ctx->nrep * nq * 6));
    // ring positions restart at 0
    launch_set_counters(ctx->counters, -1, 0, 0, ctx->st);
    ctx->ring_rows = 0;
    return finish(ctx);
}

template <typename T> static int do_run(p3m_ctx *ctx, int n_steps, int mode, int it0, int rec,
                                        int use_graph, int sync)
{
    DevState &s = ctx->s;
    if (s.has_mesh) RET(ensure_green<T>(ctx));
    launch_set_counters(ctx->counters, 0, -1, it0, ctx->st);
    ctx->launches++;
    const int gi = (mode == P3M_MODE_THERMOSTAT) ? 1 : 0, gr = rec ? 1 : 0;
    // capture `steps` steps into `*out` (the kernels of one step are counted)
    auto capture = [&](int steps, cudaGraphExec_t *out) -> int {
        cudaGraph_t g;
        const long long before = ctx->launches;
        CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
        int step_rc = P3M_OK;
        for (int k = 0; k < steps && step_rc == P3M_OK; ++k) step_rc = seq_step<T>(ctx, mode, rec);
        cudaError_t e = cudaStreamEndCapture(ctx->st, &g);
        ctx->graph_kernels[gi][gr] = (ctx->launches - before) / steps;  // kernels per step
        ctx->launches = before;
        if (step_rc != P3M_OK) {
            if (e == cudaSuccess) cudaGraphDestroy(g);
            return step_rc;
        }
        if (e != cudaSuccess) return fail(ctx, P3M_ECUDA, "cudaStreamEndCapture", cudaGetErrorString(e));
        e = cudaGraphInstantiate(out, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(ctx, P3M_ECUDA, "cudaGraphInstantiate", cudaGetErrorString(e));
        return P3M_OK;
    };
    // both graphs on first use, so that a warm-up of any length has captured
    // them before the runs it prepares
    const int gsteps = graph_steps(ctx);
    const int groups = (use_graph && gsteps > 1) ? n_steps / gsteps : 0;
    if (use_graph && !ctx->graph[gi][gr]) RET(capture(1, &ctx->graph[gi][gr]));
    if (use_graph && gsteps > 1 && !ctx->graphK[gi][gr]) RET(capture(gsteps, &ctx->graphK[gi][gr]));
    for (int k = 0; k < groups; ++k) {
        CK(cudaGraphLaunch(ctx->graphK[gi][gr], ctx->st));
        ctx->launches += (long long)gsteps * ctx->graph_kernels[gi][gr];
    }
    for (int k = groups * gsteps; k < n_steps; ++k) {
        if (use_graph) {
            CK(cudaGraphLaunch(ctx->graph[gi][gr], ctx->st));
            ctx->launches += ctx->graph_kernels[gi][gr];  // counted while capturing
        } else {
            RET(seq_step<T>(ctx, mode, rec));
        }
    }
    ctx->ring_rows += n_steps;
    if (rec) ctx->nqt_rows += n_steps;
    CK(cudaGetLastError());
    if (sync) return finish(ctx);
    return P3M_OK;
}

extern "C" int p3m_run(p3m_ctx *ctx, int n_steps, int mode, int it0, int record_nqt, int use_graph,
                       int sync)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (n_steps < 0 || (mode != P3M_MODE_NVE && mode != P3M_MODE_THERMOSTAT))
        return fail(ctx, P3M_EARG, "p3m_run", "bad n_steps or mode");
    if (record_nqt && ctx->nq == 0) return fail(ctx, P3M_EARG, "p3m_run", "n(q,t) not configured");
    CK(cudaSetDevice(ctx->device));
    return DISPATCH(do_run, ctx, n_steps, mode, it0, record_nqt, use_graph, sync);
}

extern "C" int p3m_get_energies(p3m_ctx *ctx, double *out, int max_steps, int *n_out)
{
    if (!ctx || !out || !n_out) return fail(ctx, P3M_EARG, "p3m_get_energies", "NULL argument");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    int pos[4];
    CK(cudaMemcpy(pos, ctx->counters, sizeof pos, cudaMemcpyDeviceToHost));
    const int total = pos[1];
    int n = total < ctx->ring_cap ? total : ctx->ring_cap;
    if (n > max_steps) n = max_steps;
    const size_t row = (size_t)ctx->nrep * 4;
    // rows total-n .. total-1 of the ring: at most two contiguous pieces
    for (int k = 0; k < n;) {
        const int slot = (total - n + k) % ctx->ring_cap;
        const int len = std::min(n - k, ctx->ring_cap - slot);
        CK(cudaMemcpy(out + (size_t)k * row, ctx->ring + (size_t)slot * row,
                      sizeof(double) * row * len, cudaMemcpyDeviceToHost));
        k += len;
    }
    *n_out = n;
    return P3M_OK;
}

extern "C" int p3m_get_nqt(p3m_ctx *ctx, int replica, double *out, int max_steps, int *n_out)
{
    if (!ctx || !out || !n_out) return fail(ctx, P3M_EARG, "p3m_get_nqt", "NULL argument");
    if (replica < 0 || replica >= ctx->nrep || ctx->nq == 0)
        return fail(ctx, P3M_EARG, "p3m_get_nqt", "bad replica or n(q,t) not configured");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    int pos[4];
    CK(cudaMemcpy(pos, ctx->counters, sizeof pos, cudaMemcpyDeviceToHost));
    const int total = pos[3];  // rows recorded since p3m_set_nqt
    int n = total < ctx->nqt_cap ? total : ctx->nqt_cap;
    if (n > max_steps) n = max_steps;
    const size_t rowlen = (size_t)ctx->nq * 6;
    // the replica's rows, strided by the ring's row of all replicas: at most
    // two 2-D copies (the ring wraps once)
    for (int k = 0; k < n;) {
        const int slot = (total - n + k) % ctx->nqt_cap;
        const int len = std::min(n - k, ctx->nqt_cap - slot);
        const double *src = ctx->nqt_ring + ((size_t)slot * ctx->nrep + replica) * rowlen;
        CK(cudaMemcpy2D(out + (size_t)k * rowlen, sizeof(double) * rowlen, src,
                        sizeof(double) * rowlen * ctx->nrep, sizeof(double) * rowlen, len,
                        cudaMemcpyDeviceToHost));
        k += len;
    }
    *n_out = n;
    return P3M_OK;
}

extern "C" int p3m_set_snapshots(p3m_ctx *ctx, int interval, int capacity)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (interval < 0 || (interval > 0 && capacity < 1))
        return fail(ctx, P3M_EARG, "p3m_set_snapshots", "interval must be >= 0 and capacity >= 1");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    // the step sequence changes: drop the captured graphs
    drop_graphs(ctx);
    if (capacity != ctx->snap_cap || interval == 0) {
        cudaFree(ctx->snap);
        cudaFree(ctx->snap_steps);
        ctx->snap = nullptr;
        ctx->snap_steps = nullptr;
        ctx->snap_cap = 0;
    }
    ctx->snap_interval = 0;
    if (interval > 0) {
        if (!ctx->snap) {
            CK(dalloc(&ctx->snap, (size_t)capacity * ctx->s.ntot * 9));
            CK(dalloc(&ctx->snap_steps, (size_t)capacity));
        }
        ctx->snap_cap = capacity;
        ctx->snap_interval = interval;
    }
    CK(cudaMemsetAsync(ctx->counters + 4, 0, 2 * sizeof(int), ctx->st));
    ctx->snap_read = 0;
    return finish(ctx);
}

extern "C" int p3m_get_snapshots(p3m_ctx *ctx, double *out, int *steps, int max_snaps, int *n_out)
{
    if (!ctx || !out || !n_out || max_snaps < 0)
        return fail(ctx, P3M_EARG, "p3m_get_snapshots", "NULL argument");
    *n_out = 0;
    if (ctx->snap_cap == 0) return fail(ctx, P3M_EARG, "p3m_get_snapshots", "snapshots not configured");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    int taken = 0;
    CK(cudaMemcpy(&taken, ctx->counters + 4, sizeof(int), cudaMemcpyDeviceToHost));
    const long long avail = taken - ctx->snap_read;
    if (avail > ctx->snap_cap) {
        ctx->snap_read = taken;
        return fail(ctx, P3M_ESTATE, "p3m_get_snapshots",
                    "the snapshot ring overflowed: read it at least every capacity x interval steps");
    }
    const int n = (int)std::min<long long>(avail, max_snaps);
    const size_t per = (size_t)ctx->s.ntot * 9;
    for (int k = 0; k < n;) {
        const int slot = (int)((ctx->snap_read + k) % ctx->snap_cap);
        const int len = std::min(n - k, ctx->snap_cap - slot);
        CK(cudaMemcpy(out + (size_t)k * per, ctx->snap + (size_t)slot * per,
                      sizeof(double) * per * len, cudaMemcpyDeviceToHost));
        if (steps)
            CK(cudaMemcpy(steps + k, ctx->snap_steps + slot, sizeof(int) * len,
                          cudaMemcpyDeviceToHost));
        k += len;
    }
    ctx->snap_read += n;
    *n_out = n;
    return P3M_OK;
}

extern "C" int p3m_get_replica_stats(p3m_ctx *ctx, int replica, double *out)
{
    if (!ctx || !out) return fail(ctx, P3M_EARG, "p3m_get_replica_stats", "NULL argument");
    if (replica < 0 || replica >= ctx->nrep) return fail(ctx, P3M_EARG, "p3m_get_replica_stats", "replica");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaMemcpy(out, ctx->s.rep_out + 8 * (size_t)replica, 8 * sizeof(double), cudaMemcpyDeviceToHost));
    return P3M_OK;
}

extern "C" int p3m_check(p3m_ctx *ctx)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    CK(cudaSetDevice(ctx->device));
    return finish(ctx);
}

extern "C" int p3m_sync(p3m_ctx *ctx)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    CK(cudaSetDevice(ctx->device));
    if (!ctx->step_pending) return finish(ctx);  // waits, then reports a device status
    // copies of p3m_get_step_async are queued: wait, deliver the energies
    ctx->step_pending = false;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));
    const double *h = ctx->h_step;
    if (ctx->step_out)
        for (int r = 0; r < ctx->nrep; ++r) {
            double *o = ctx->step_out + 4 * (size_t)r;
            o[0] = h[8 * r + RO_U];
            o[1] = h[8 * r + RO_K];
            o[2] = h[8 * r + RO_T];
            o[3] = h[8 * r + RO_FACT];
        }
    ctx->step_out = nullptr;
    if (ctx->launches != ctx->step_launches) return finish(ctx);  // later work: read the status now
    int st;
    memcpy(&st, h + 8 * (size_t)ctx->nrep, sizeof st);
    return status_error(ctx, st);
}

extern "C" int p3m_set_priority(p3m_ctx *ctx, int level)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    if (level < 0) return fail(ctx, P3M_EARG, "p3m_set_priority", "level must be >= 0");
    CK(cudaSetDevice(ctx->device));
    int least = 0, greatest = 0;
    CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int prio = (greatest + level < least) ? greatest + level : least;
    // the new streams first: on a failure the context keeps its old ones
    cudaStream_t fresh[3] = {nullptr, nullptr, nullptr};
    for (int k = 0; k < 3; ++k) {
        const cudaError_t e = cudaStreamCreateWithPriority(&fresh[k], cudaStreamNonBlocking, prio);
        if (e != cudaSuccess) {
            for (int j = 0; j < k; ++j) cudaStreamDestroy(fresh[j]);
            return fail(ctx, P3M_ECUDA, "cudaStreamCreateWithPriority", cudaGetErrorString(e));
        }
    }
    cudaStream_t *streams[3] = {&ctx->st, &ctx->st2, &ctx->st3};
    for (cudaStream_t *p : streams) {
        const cudaError_t e = cudaStreamSynchronize(*p);
        if (e != cudaSuccess) {  // keep the old streams and graphs; drop the new streams
            for (int k = 0; k < 3; ++k) cudaStreamDestroy(fresh[k]);
            return fail(ctx, P3M_ECUDA, "cudaStreamSynchronize", cudaGetErrorString(e));
        }
    }
    drop_graphs(ctx);
    for (int k = 0; k < 3; ++k) {
        cudaStreamDestroy(*streams[k]);
        *streams[k] = fresh[k];
    }
    return P3M_OK;
}

extern "C" int p3m_set_tuning(p3m_ctx *ctx, const p3m_tuning *t)
{
    if (!ctx || !t) return fail(ctx, P3M_EARG, "p3m_set_tuning", "NULL argument");
    const int tpi = t->pp_tpi;
    if (!(tpi == 1 || tpi == 2 || tpi == 4 || tpi == 8))
        return fail(ctx, P3M_EARG, "p3m_set_tuning", "pp_tpi must be 1, 2, 4 or 8");
    if (t->cell_div != 1 && t->cell_div != 2)
        return fail(ctx, P3M_EARG, "p3m_set_tuning", "cell_div must be 1 or 2");
    if (t->plane_max != 0 && t->plane_max != 32 && t->plane_max != plane_max_mesh())
        return fail(ctx, P3M_EARG, "p3m_set_tuning", "plane_max must be 0, 32 or 64");
    if (t->gather_mode < 0 || t->gather_mode > 2)
        return fail(ctx, P3M_EARG, "p3m_set_tuning", "gather_mode must be 0, 1 or 2");
    for (int r = 0; r < ctx->nrep; ++r)
        if (t->skin > 0.5 * ctx->desc[r].rc)
            return fail(ctx, P3M_EARG, "p3m_set_tuning", "skin must be <= rc/2 (negative: default)");
    if (!(t->prune_buf >= 0.0 && t->prune_buf <= 1e3))
        return fail(ctx, P3M_EARG, "p3m_set_tuning", "prune_buf must be >= 0");
    if (t->prune_buf > 0.0 && ctx->prec != P3M_FP32)
        return fail(ctx, P3M_EARG, "p3m_set_tuning", "inner lists (prune_buf > 0) are an FP32-path option");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    drop_graphs(ctx);
    DevState &s = ctx->s;
    // the new plan replaces the old one only once its list storage exists
    const DevState saved = s;
    const std::vector<RepDev> saved_rh = ctx->rh;
    s.cell_div = t->cell_div;
    s.plane_max = t->plane_max;
    s.gather_mode = (ctx->prec == P3M_FP64 && t->gather_mode == 2) ? 1 : t->gather_mode;
    s.prune_buf = t->prune_buf;
    plan_lists(ctx, t->skin, tpi);
    plan_mesh_passes(ctx);
    for (int r = 0; r < ctx->nrep; ++r)
        if (s.prune_buf > 0.0 && s.prune_buf >= ctx->rh[r].skin) {
            s = saved;
            ctx->rh = saved_rh;
            return fail(ctx, P3M_EARG, "p3m_set_tuning", "prune_buf must be below every replica's skin");
        }
    // list storage: the outer lists, then the inner ones (both keep their
    // old storage when it is large enough)
    const long long need = (long long)((s.ntot + 31) / 32) * 32 * s.maxnb;
    const long long need_in = (long long)((s.ntot + 31) / 32) * 32 * s.maxnb_in;
    int *fresh = nullptr, *fresh_in = nullptr;
    cudaError_t e = cudaSuccess;
    if (need > ctx->nlist_cap) e = dalloc(&fresh, (size_t)need);
    if (e == cudaSuccess && need_in > ctx->nlist_in_cap) e = dalloc(&fresh_in, (size_t)need_in);
    if (e != cudaSuccess) {
        cudaFree(fresh);
        s = saved;
        ctx->rh = saved_rh;
        return fail(ctx, P3M_ECUDA, "p3m_set_tuning: list storage", cudaGetErrorString(e));
    }
    if (fresh) {
        cudaFree(s.nlist);
        s.nlist = fresh;
        ctx->nlist_cap = need;
    }
    if (fresh_in) {
        cudaFree(s.nlist_in);
        s.nlist_in = fresh_in;
        ctx->nlist_in_cap = need_in;
    }
    ctx->skin_override = t->skin < 0.0 ? -1.0 : t->skin;
    CK(cudaMemcpy(s.reps, ctx->rh.data(), sizeof(RepDev) * ctx->nrep, cudaMemcpyHostToDevice));
    launch_set_flags(s.rebuild, s.nrep, 1, ctx->st);  // the next force evaluation builds both lists
    return finish(ctx);
}

extern "C" int p3m_get_tuning(p3m_ctx *ctx, p3m_tuning *t)
{
    if (!ctx || !t) return fail(ctx, P3M_EARG, "p3m_get_tuning", "NULL argument");
    t->pp_tpi = ctx->s.pp_tpi;
    t->cell_div = ctx->s.cell_div;
    t->plane_max = ctx->s.plane_max;
    t->gather_mode = ctx->s.gather_mode;
    t->skin = ctx->skin_override;
    t->prune_buf = ctx->s.prune_buf;
    return P3M_OK;
}

extern "C" int p3m_get_inner_builds(p3m_ctx *ctx, int replica, double *out)
{
    if (!ctx || !out) return fail(ctx, P3M_EARG, "p3m_get_inner_builds", "NULL argument");
    if (replica < 0 || replica >= ctx->nrep) return fail(ctx, P3M_EARG, "p3m_get_inner_builds", "replica");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaMemcpy(out, ctx->s.prune_count + replica, sizeof(double), cudaMemcpyDeviceToHost));
    return P3M_OK;
}

extern "C" int p3m_set_pp_config(p3m_ctx *ctx, int tpi, double skin)
{
    if (!ctx) return fail(nullptr, P3M_EARG, "context", "NULL");
    p3m_tuning t;
    p3m_get_tuning(ctx, &t);
    t.pp_tpi = tpi;
    t.skin = skin;
    return p3m_set_tuning(ctx, &t);
}

extern "C" int p3m_get_pp_config(p3m_ctx *ctx, int *tpi, double *skin, int *maxnb)
{
    if (!ctx || !tpi || !skin || !maxnb) return fail(ctx, P3M_EARG, "p3m_get_pp_config", "NULL argument");
    *tpi = ctx->s.pp_tpi;
    *skin = ctx->rh[0].skin;
    *maxnb = ctx->s.maxnb;
    return P3M_OK;
}

// ---------------------------------------------------------------------------
// measurement
// ---------------------------------------------------------------------------

// Each stage is idempotent when repeated (the inverse FFT works in place on
// the field spectra, so it is timed together with the forward pass that
// rebuilds them: fft_inverse = fft_both - fft_forward). With inner lists,
// "pp" is the pair kernel of a step without list work (inner lists) and
// "pp_prune" that of a step where every replica builds its inner lists.
static const char *kStageNames[] = {"drift_sort", "keys_sort", "pp", "assign", "fft_forward",
                                    "fft_both", "gather", "finish", "nqt", "step", "pp_prune"};
static const int kNumStages = 11;

extern "C" const char *p3m_stage_name(int i)
{
    return (i >= 0 && i < kNumStages) ? kStageNames[i] : "";
}

template <typename T> static void enqueue_stage(p3m_ctx *ctx, int k)
{
    DevState &s = ctx->s;
    switch (k) {
    case 0:
        launch_kick_drift(s, ctx->st);
        seq_sort<T>(ctx, false);
        break;
    case 1: seq_sort<T>(ctx, true); break;
    case 2: seq_pp<T>(ctx); break;
    case 3: launch_assign<T>(s, ctx->st); ctx->launches++; break;
    case 4:
        launch_fft_forward<T>(s, ctx->st);
        ctx->launches += fft_kernel_count(s) - 1 - (s.wb > 0 ? 1 : 0);
        break;
    case 5:
        launch_fft_forward<T>(s, ctx->st);
        launch_fft_inverse<T>(s, ctx->st);
        ctx->launches += fft_kernel_count(s);
        break;
    case 6: launch_gather<T>(s, ctx->st); ctx->launches++; break;
    case 7:
        launch_kick_finish<T>(s, 0, nullptr, ctx->st);
        launch_step_reduce(s, 2, ctx->counters, nullptr, 0, ctx->st);
        ctx->launches += 2;
        break;
    case 10:
        launch_set_flags(s.rebuild, s.nrep, 1, ctx->st);
        seq_pp<T>(ctx);
        ctx->launches++;
        break;
    case 8:
        if (ctx->nq > 0) {
            launch_nqt<T>(s, s.pos, ctx->qmult, ctx->nq, ctx->nq_consecutive, ctx->nqt_part,
                          ctx->tmp_nq ? ctx->tmp_nq : ctx->nqt_part, nullptr, 0, ctx->st);
            ctx->launches += 2;
        }
        break;
    default: break;
    }
}

// Average device time of each stage over `iters` back-to-back launches
// (CUDA events on the context's stream). The drift stage moves the
// particles, so this perturbs the state; call it after the run it measures.
template <typename T> static int do_profile(p3m_ctx *ctx, int iters, double *ms, int max_stages,
                                            int *n_out)
{
    DevState &s = ctx->s;
    if (s.has_mesh) RET(ensure_green<T>(ctx));
    if (ctx->nq > 0 && ctx->tmp_nq_cap == 0) {
        CK(dalloc(&ctx->tmp_nq, (size_t)ctx->nrep * 64 * 6 + (size_t)s.nblk * 64 * 6 + 64));
        ctx->tmp_nq_cap = 64;
    }
    // the drift stage kicks with stale forces on every repeat: keep a copy of
    // the state and put it back afterwards
    const size_t sb = sizeof(double) * 3 * (size_t)s.ntot;
    double *backup = nullptr;
    CK(cudaMalloc(&backup, 3 * sb));
    CK(cudaMemcpyAsync(backup, s.pos, sb, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(backup + 3 * (size_t)s.ntot, s.vel, sb, cudaMemcpyDeviceToDevice, ctx->st));
    CK(cudaMemcpyAsync(backup + 6 * (size_t)s.ntot, s.acc, sb, cudaMemcpyDeviceToDevice, ctx->st));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int n = 0;
    for (int k = 0; k < kNumStages && n < max_stages; ++k, ++n) {
        ms[n] = 0.0;
        if (!s.has_mesh && k >= 3 && k <= 6) continue;
        if (k == 8 && ctx->nq == 0) continue;
        // one untimed launch, then the timed loop
        if (k == 9) {
            if (!ctx->graph[0][0]) { RET(do_run<T>(ctx, 1, P3M_MODE_NVE, 0, 0, 1, 1)); }
            CK(cudaEventRecord(e0, ctx->st));
            for (int i = 0; i < iters; ++i) CK(cudaGraphLaunch(ctx->graph[0][0], ctx->st));
            CK(cudaEventRecord(e1, ctx->st));
        } else {
            enqueue_stage<T>(ctx, k);
            if (k == 2 && s.prune_buf > 0.0) {
                // that launch built the inner lists: time the steps that read them
                launch_set_flags(s.rebuild, s.nrep, 0, ctx->st);
                launch_set_flags(s.prune, s.nrep, 0, ctx->st);
                ctx->launches += 2;
            }
            CK(cudaEventRecord(e0, ctx->st));
            for (int i = 0; i < iters; ++i) enqueue_stage<T>(ctx, k);
            CK(cudaEventRecord(e1, ctx->st));
        }
        CK(cudaEventSynchronize(e1));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, e0, e1));
        ms[n] = (double)t / iters;
        {
            int stv = 0;
            CK(cudaMemcpy(&stv, s.status, sizeof(int), cudaMemcpyDeviceToHost));
            if (stv && k != 0) {
                char b[128];
                snprintf(b, sizeof b, "status %d raised while profiling stage %s", stv, kStageNames[k]);
                ctx->err = b;
                ms[n] = -ms[n];  // flagged
                CK(cudaMemset(s.status, 0, sizeof(int)));
            }
        }
        if (k == 0) {
            // restore the state, clear what the stale drifts may have flagged,
            // and re-sort for the stages that follow
            CK(cudaMemcpyAsync(s.pos, backup, sb, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(s.vel, backup + 3 * (size_t)s.ntot, sb, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemcpyAsync(s.acc, backup + 6 * (size_t)s.ntot, sb, cudaMemcpyDeviceToDevice, ctx->st));
            CK(cudaMemsetAsync(s.status, 0, sizeof(int), ctx->st));
            seq_sort<T>(ctx, true);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(cudaStreamSynchronize(ctx->st));
    cudaFree(backup);
    *n_out = n;
    return finish(ctx);
}

extern "C" int p3m_profile_stages(p3m_ctx *ctx, int iters, double *ms, int max_stages, int *n_out)
{
    if (!ctx || !ms || !n_out || iters <= 0) return fail(ctx, P3M_EARG, "p3m_profile_stages", "bad argument");
    CK(cudaSetDevice(ctx->device));
    return DISPATCH(do_profile, ctx, iters, ms, max_stages, n_out);
}

extern "C" int p3m_fp32_peak(int device, double *tflops)
{
    if (!tflops) return fail(nullptr, P3M_EARG, "p3m_fp32_peak", "NULL argument");
    int rc = check_device(nullptr, device);
    if (rc != P3M_OK) return rc;
    const double t = fp32_fma_tflops(device);
    if (t <= 0) return fail(nullptr, P3M_ECUDA, "p3m_fp32_peak", "probe kernel failed");
    *tflops = t;
    return P3M_OK;
}

// ---------------------------------------------------------------------------
// S(q, omega)
// ---------------------------------------------------------------------------

static int ilog2_ceil(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

// Chirp spectrum for Bluestein's transform of length nt with FFT length P,
// in bit-reversed order (host, FP64).
static void chirp_spectrum_br(int nt, int logP, std::vector<double2> &out)
{
    const int P = 1 << logP;
    std::vector<std::complex<long double>> b(P, 0.0L);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < nt; ++m) {
        const long long q = ((long long)m * m) % (2LL * nt);
        const std::complex<long double> c = std::polar(1.0L, pi * (long double)q / nt);
        b[m] = c;
        if (m > 0) b[P - m] = c;
    }
    // plain O(P log P) radix-2 DIT on the host (bit-reversed input)
    std::vector<std::complex<long double>> x(P);
    for (int n = 0; n < P; ++n) {
        int r = 0;
        for (int k = 0; k < logP; ++k) r |= ((n >> k) & 1) << (logP - 1 - k);
        x[r] = b[n];
    }
    for (int s = 1; s <= logP; ++s) {
        const int m = 1 << s, h = m >> 1;
        for (int k = 0; k < h; ++k) {
            const std::complex<long double> w = std::polar(1.0L, -2.0L * pi * k / m);
            for (int j = k; j < P; j += m) {
                const std::complex<long double> t = w * x[j + h];
                x[j + h] = x[j] - t;
                x[j] = x[j] + t;
            }
        }
    }
    out.resize(P);
    for (int j = 0; j < P; ++j) {
        int r = 0;
        for (int k = 0; k < logP; ++k) r |= ((j >> k) & 1) << (logP - 1 - k);
        out[j] = make_double2((double)x[r].real(), (double)x[r].imag());
    }
}

static int plan_sqw(int nt, int *logP, int *bluestein)
{
    const bool pow2 = nt > 0 && (nt & (nt - 1)) == 0;
    *bluestein = pow2 ? 0 : 1;
    *logP = pow2 ? ilog2_ceil(nt) : ilog2_ceil(2 * nt - 1);
    return (1 << *logP) <= sqw_max_points() ? P3M_OK : P3M_EARG;
}

static const char *kSqwLenMsg = "nt must be a power of two <= 2^21 or any length <= 2^20";

// Runs k_sqw over replicas 0..nrep-1 of the series described by `a` (src,
// strides, ring position, columns and nt set by the caller) on stream st:
// uploads the chirp spectrum and the particle counts, takes a global-memory
// transform scratch for lengths beyond shared memory (replicas in chunks of
// at most 1 GiB of scratch), and copies out_rep (nrep * ncols * nt [* 3])
// and, when `out` is not NULL, the mean over replicas to the host.
static cudaError_t sqw_device(SqwArgs a, int nrep, const double *n_per_rep, cudaStream_t st,
                              double *host_out_rep, double *host_out, long long *launches)
{
    std::vector<double2> chirp;
    if (a.bluestein) chirp_spectrum_br(a.nt, a.logP, chirp);
    const size_t P = (size_t)1 << a.logP;
    const size_t per_rep = (size_t)a.ncols * a.nt * (a.per_axis ? 3 : 1);
    int chunk = nrep;
    if ((int)P > sqw_smem_points()) {
        const size_t per = (size_t)a.ncols * P * sizeof(double2);
        chunk = (int)std::max<size_t>(1, std::min<size_t>(nrep, ((size_t)1 << 30) / per));
    }
    double *d_rep = nullptr, *d_out = nullptr, *d_n = nullptr;
    double2 *d_chirp = nullptr, *d_scr = nullptr;
    cudaError_t e = cudaMalloc(&d_rep, (size_t)nrep * per_rep * sizeof(double));
    if (e == cudaSuccess && host_out) e = cudaMalloc(&d_out, per_rep * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_n, (size_t)nrep * sizeof(double));
    if (e == cudaSuccess && a.bluestein) e = cudaMalloc(&d_chirp, P * sizeof(double2));
    if (e == cudaSuccess && (int)P > sqw_smem_points())
        e = cudaMalloc(&d_scr, (size_t)chunk * a.ncols * P * sizeof(double2));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_n, n_per_rep, (size_t)nrep * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && a.bluestein)
        e = cudaMemcpyAsync(d_chirp, chirp.data(), P * sizeof(double2), cudaMemcpyHostToDevice, st);
    a.chirp_fft_br = d_chirp;
    a.nrep_n = d_n;
    a.out_rep = d_rep;
    for (int r0 = 0; e == cudaSuccess && r0 < nrep; r0 += chunk) {
        a.r0 = r0;
        a.nrep_launch = std::min(chunk, nrep - r0);
        launch_sqw(a, d_scr, st);
        ++*launches;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && host_out) {
        launch_sqw_mean(d_rep, nrep, (long long)per_rep, d_out, st);
        ++*launches;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && host_out)
        e = cudaMemcpy(host_out, d_out, per_rep * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && host_out_rep)
        e = cudaMemcpy(host_out_rep, d_rep, (size_t)nrep * per_rep * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_rep);
    cudaFree(d_out);
    cudaFree(d_n);
    cudaFree(d_chirp);
    cudaFree(d_scr);
    return e;
}

extern "C" int p3m_sqw(p3m_ctx *ctx, double dt, int col0, int col_stride, int ncols, int nt,
                       double *out, double *out_rep)
{
    if (!ctx || (!out && !out_rep)) return fail(ctx, P3M_EARG, "p3m_sqw", "NULL argument");
    if (ctx->nq == 0) return fail(ctx, P3M_EARG, "p3m_sqw", "n(q,t) not configured");
    if (ncols <= 0 || col0 < 0 || col_stride < 1 || col0 + (long long)(ncols - 1) * col_stride >= ctx->nq)
        return fail(ctx, P3M_EARG, "p3m_sqw", "q columns out of range");
    if (!(dt > 0)) return fail(ctx, P3M_EARG, "p3m_sqw", "dt must be > 0");
    SqwArgs a{};
    if (nt < 2 || plan_sqw(nt, &a.logP, &a.bluestein) != P3M_OK)
        return fail(ctx, P3M_EARG, "p3m_sqw", kSqwLenMsg);
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    int pos[4];
    CK(cudaMemcpy(pos, ctx->counters, sizeof pos, cudaMemcpyDeviceToHost));
    const int total = pos[3];
    if (total < nt || nt > ctx->nqt_cap)
        return fail(ctx, P3M_EARG, "p3m_sqw", "fewer recorded n(q,t) rows than nt");
    std::vector<double> nr(ctx->nrep);
    for (int r = 0; r < ctx->nrep; ++r) nr[r] = ctx->desc[r].n;
    a.src = (const double2 *)ctx->nqt_ring;
    a.row_stride = (long long)ctx->nrep * ctx->nq * 3;
    a.rep_stride = (long long)ctx->nq * 3;
    a.cap = ctx->nqt_cap;
    a.row0 = (total - nt) % ctx->nqt_cap;
    a.col0 = col0;
    a.col_stride = col_stride;
    a.ncols = ncols;
    a.nt = nt;
    a.dt = dt;
    a.per_axis = 0;
    std::vector<double> rep;
    double *host_rep = out_rep;
    if (!host_rep) {
        rep.resize((size_t)ctx->nrep * ncols * nt);
        host_rep = rep.data();
    }
    long long nl = 0;
    cudaError_t e = sqw_device(a, ctx->nrep, nr.data(), ctx->st, host_rep, out, &nl);
    ctx->launches += nl;
    if (e != cudaSuccess) return fail(ctx, P3M_ECUDA, "p3m_sqw", cudaGetErrorString(e));
    return P3M_OK;
}

// Series held on the host as complex128 (re, im pairs): uploads them and runs
// sqw_device on the legacy default stream; then rescales from T = nt dt to
// the caller's T.
static int sqw_host(const char *who, int device, const double *src, int nrun, int nt, int nq,
                    int col0, int col_stride, int ncols, double N, double dt, double T, int per_axis,
                    double *out_rep)
{
    SqwArgs a{};
    if (nt < 2 || plan_sqw(nt, &a.logP, &a.bluestein) != P3M_OK)
        return fail(nullptr, P3M_EARG, who, kSqwLenMsg);
    int rc = check_device(nullptr, device);
    if (rc != P3M_OK) return rc;
    const size_t n_src = (size_t)nrun * nt * nq * 3;
    double2 *d_src = nullptr;
    cudaError_t e = cudaMalloc(&d_src, n_src * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemcpy(d_src, src, n_src * sizeof(double2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        a.src = d_src;
        a.row_stride = (long long)nq * 3;
        a.rep_stride = (long long)nt * nq * 3;
        a.cap = nt;
        a.row0 = 0;
        a.col0 = col0;
        a.col_stride = col_stride;
        a.ncols = ncols;
        a.nt = nt;
        a.dt = dt;
        a.per_axis = per_axis;
        std::vector<double> nr(nrun, N);
        long long nl = 0;
        e = sqw_device(a, nrun, nr.data(), 0, out_rep, nullptr, &nl);
    }
    cudaFree(d_src);
    if (e != cudaSuccess) return fail(nullptr, P3M_ECUDA, who, cudaGetErrorString(e));
    const double f = (nt * dt) / T;
    const size_t n_out = (size_t)nrun * ncols * nt * (per_axis ? 3 : 1);
    for (size_t i = 0; i < n_out; ++i) out_rep[i] *= f;
    return P3M_OK;
}

extern "C" int p3m_sqw_series(int device, const double *nqt, int nt, double N, double dt, double T,
                              double *out)
{
    if (!nqt || !out || !(N > 0) || !(T > 0) || !(dt > 0))
        return fail(nullptr, P3M_EARG, "p3m_sqw_series", "bad argument");
    std::vector<double> o((size_t)3 * (nt > 0 ? nt : 0));
    const int rc = sqw_host("p3m_sqw_series", device, nqt, 1, nt, 1, 0, 1, 1, N, dt, T, 1, o.data());
    if (rc != P3M_OK) return rc;
    for (int k = 0; k < nt; ++k)
        for (int ax = 0; ax < 3; ++ax) out[3 * (size_t)k + ax] = o[(size_t)ax * nt + k];
    return P3M_OK;
}

extern "C" int p3m_sqw_runs(int device, const double *nqt, int nrun, int nt, int nq, int col0,
                            int col_stride, int ncols, double N, double dt, double T, double *out)
{
    if (!nqt || !out || nrun < 1 || nq < 1 || !(N > 0) || !(T > 0) || !(dt > 0))
        return fail(nullptr, P3M_EARG, "p3m_sqw_runs", "bad argument");
    if (ncols <= 0 || col0 < 0 || col_stride < 1 || col0 + (long long)(ncols - 1) * col_stride >= nq)
        return fail(nullptr, P3M_EARG, "p3m_sqw_runs", "q columns out of range");
    return sqw_host("p3m_sqw_runs", device, nqt, nrun, nt, nq, col0, col_stride, ncols, N, dt, T, 0,
                    out);
}

// ---------------------------------------------------------------------------
// PPPM error estimates
// ---------------------------------------------------------------------------

extern "C" int p3m_pp_error(double n, double box, double kappa, double alpha, double rc, double *dF)
{
    if (!dF || !(n > 0) || !(box > 0) || !(kappa >= 0) || !(alpha > 0) || !(rc > 0))
        return fail(nullptr, P3M_EARG, "p3m_pp_error", "bad argument");
    *dF = pp_error_estimate(n, box, kappa, alpha, rc);
    return P3M_OK;
}

extern "C" int p3m_pp_cutoff(double n, double box, double kappa, double alpha, double tol,
                             double rc_max, double *rc)
{
    if (!rc || !(n > 0) || !(box > 0) || !(kappa >= 0) || !(alpha > 0) || !(tol > 0) || !(rc_max > 0))
        return fail(nullptr, P3M_EARG, "p3m_pp_cutoff", "bad argument");
    *rc = pp_cutoff_for(n, box, kappa, alpha, tol, rc_max);
    return P3M_OK;
}

extern "C" int p3m_pm_error(int device, int count, const double *n, const double *box,
                            const double *kappa, const double *alpha, const int *M, int p,
                            int m_alias, double *dF, double *a_pm)
{
    if (count < 0 || (count > 0 && (!n || !box || !kappa || !alpha || !M || !dF)))
        return fail(nullptr, P3M_EARG, "p3m_pm_error", "NULL argument");
    if (p < 1 || p > 7 || m_alias < 0 || m_alias > 7)
        return fail(nullptr, P3M_EARG, "p3m_pm_error", "p must be in [1, 7], m_alias in [0, 7]");
    int maxb = 1;
    for (int i = 0; i < count; ++i) {
        if (!(n[i] > 0) || !(box[i] > 0) || !(kappa[i] >= 0) || !(alpha[i] > 0) || M[i] < 2 ||
            M[i] > 512)
            return fail(nullptr, P3M_EARG, "p3m_pm_error", "bad parameter set");
        maxb = std::max(maxb, pm_error_blocks(M[i]));
    }
    if (count == 0) return P3M_OK;
    int rc = check_device(nullptr, device);
    if (rc != P3M_OK) return rc;
    // partial sums of every set, [set][2][block]
    const size_t stride = 2 * (size_t)maxb;
    double *d_part = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&d_part, (size_t)count * stride * sizeof(double));
    for (int i = 0; e == cudaSuccess && i < count; ++i) {
        double *q = d_part + (size_t)i * stride;
        launch_pm_error(kappa[i], alpha[i], p, m_alias, M[i], box[i], q, q + maxb, st);
        e = cudaGetLastError();
    }
    std::vector<double> h;
    if (e == cudaSuccess) {
        h.resize((size_t)count * stride);
        e = cudaMemcpyAsync(h.data(), d_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_part);
    if (st) cudaStreamDestroy(st);
    if (e != cudaSuccess) return fail(nullptr, P3M_ECUDA, "p3m_pm_error", cudaGetErrorString(e));
    for (int i = 0; i < count; ++i) {
        const double *q = h.data() + (size_t)i * stride;
        const int nb = pm_error_blocks(M[i]);
        double sq = 0.0, sa = 0.0;
        for (int b = 0; b < nb; ++b) {
            sq += q[b];
            sa += q[maxb + b];
        }
        const double V = box[i] * box[i] * box[i];
        dF[i] = std::sqrt(std::max(sq, 0.0) * n[i] / (V * V));
        if (a_pm) a_pm[i] = sa;
    }
    return P3M_OK;
}

extern "C" int p3m_set_t_desired(p3m_ctx *ctx, const double *t_desired)
{
    if (!ctx || !t_desired) return fail(ctx, P3M_EARG, "p3m_set_t_desired", "NULL argument");
    for (int r = 0; r < ctx->nrep; ++r)
        if (!(t_desired[r] > 0.0) || !(t_desired[r] < 1e300))
            return fail(ctx, P3M_EARG, "p3m_set_t_desired", "temperatures must be finite and > 0");
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->st));
    for (int r = 0; r < ctx->nrep; ++r) {
        ctx->desc[r].t_desired = t_desired[r];
        ctx->rh[r].t_desired = t_desired[r];
    }
    // the step graphs read the replica table from device memory: no recapture
    CK(cudaMemcpy(ctx->s.reps, ctx->rh.data(), sizeof(RepDev) * ctx->nrep, cudaMemcpyHostToDevice));
    return P3M_OK;
}
