/*
 * p3m_b200 -- C ABI of the B200 (sm_100a) P3M force step and integrator.
 *
 * A drop-in for the hot path of xgdhar/MD-force-routines: the Python modules
 * yukawa_pp, yukawa_pm_ord6, yukawa_gf_opt, yukawa_p3m_ord6,
 * velocity_verlet_p3m_ord6 and thermostat_p3m_ord6 of this package call these
 * entry points through ctypes. Each entry point names the reference routine it
 * replaces (file:line in the reference tree).
 *
 * Conventions
 *  - Every function returns an int status: P3M_OK (0) or a negative P3M_E*
 *    code; none aborts. p3m_last_error() gives a message for the last failure
 *    on a context (or of a context-free call when ctx is NULL).
 *  - Host arrays are C-contiguous float64 in the reference's layouts: particle
 *    arrays (N,3) row-major, meshes (Mz,My,Mx) with x fastest.
 *  - One context per host thread; calls on a context run in order on its own
 *    CUDA stream. Calls that take host pointers copy in, compute and copy out
 *    before they return ("compat" calls). p3m_run() works on device-resident
 *    state and returns without waiting unless asked to.
 *  - A context holds R replicas (independent systems) with their own N, box,
 *    kappa, alpha, r_c and mesh; every stage advances all of them in one
 *    launch.
 */
#ifndef P3M_B200_H
#define P3M_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define P3M_OK 0
#define P3M_EARG (-1)          /* invalid argument or unsupported size        */
#define P3M_ECUDA (-2)         /* CUDA runtime error                          */
#define P3M_ENODEV (-3)        /* no usable sm_100 device                     */
#define P3M_EBOX (-4)          /* particle outside [-L, 2L) or non-finite     */
#define P3M_ENONFINITE (-5)    /* NaN/Inf in velocities, forces or energies   */
#define P3M_ESTATE (-6)        /* call out of order (e.g. no state uploaded)  */
#define P3M_ENBOVF (-7)        /* neighbour-list capacity exceeded            */

/* arithmetic of the bulk stages (PP pair loop, assignment, FFT, gather) */
#define P3M_FP64 0             /* everything in FP64: the plain method        */
#define P3M_FP32 1             /* FP32 bulk, FP64 reductions and positions    */

/* p3m_run modes */
#define P3M_MODE_NVE 0         /* velocity_verlet_p3m_ord6.update per step    */
#define P3M_MODE_THERMOSTAT 1  /* thermostat_p3m_ord6.vscale per step         */

typedef struct p3m_ctx p3m_ctx;

/* One replica. Mirrors the constants the reference's driver passes down the
 * call stack (yukawa_MD_p3m_ord6.py:26-79). */
typedef struct {
    int32_t n;          /* particles                                         */
    int32_t mesh;       /* M = Mx = My = Mz: power of two, 32..256 (0: no PM) */
    int32_t order;      /* charge-assignment order p: must be 6              */
    int32_t m_alias;    /* mx_max = my_max = mz_max of gf_opt (reference: 3) */
    double box;         /* L = Lx = Ly = Lz                                  */
    double kappa;       /* screening parameter                               */
    double alpha;       /* Ewald splitting parameter (G / G_ew)              */
    double rc;          /* PP cutoff; floor(L/rc) must be >= 3               */
    double dt;          /* time step                                         */
    double t_desired;   /* thermostat target temperature (1/Gamma)           */
    double af, uf, kf;  /* acceleration, energy and kinetic-energy factors    */
    double skin;        /* Verlet-list skin (< 0: default 0.5; <= rc/2)       */
} p3m_replica_desc;

/* ---- context ---------------------------------------------------------- */
int p3m_create(const p3m_replica_desc *reps, int n_reps, int precision, int device,
               p3m_ctx **out);
int p3m_destroy(p3m_ctx *ctx);
const char *p3m_last_error(const p3m_ctx *ctx);
int p3m_version(void);
/* Kernels launched on the context's stream so far (monotone counter). */
int64_t p3m_launch_count(const p3m_ctx *ctx);

/* ---- compat calls: host pointers in and out, one replica ---------------- */

/* yukawa_pp.py:6 particle_particle(kappa,G,rc,Lv,pos,acc_s_r) -> (U, acc).
 * pos (n,3) in; acc (n,3) out; *U out. */
int p3m_pp(p3m_ctx *ctx, int replica, const double *pos, double *acc, double *U);

/* yukawa_pm_ord6.py:6 charge_assgn_6_numba(rho_r,pos,Z,N,...) -> rho_r.
 * rho (M,M,M) out. Z may be NULL (unit charges). */
int p3m_assign(p3m_ctx *ctx, int replica, const double *pos, const double *Z, double *rho);

/* yukawa_pm_ord6.py:213 field_assgn_6_numba(acc,E_x_p,..,E_x_r,..,pos,Z,..)
 * Ex,Ey,Ez (M,M,M) in; acc (n,3) out; Ep (3,n) out (may be NULL). */
int p3m_gather(p3m_ctx *ctx, int replica, const double *pos, const double *Z,
               const double *Ex, const double *Ey, const double *Ez, double *acc,
               double *Ep);

/* yukawa_gf_opt.py:5 gf_opt(kappa,Gew,p,mx_max,my_max,mz_max,Mx,..,Lz):
 * the optimal influence function on an M^3 mesh in the reference's fftshifted
 * layout, computed in FP64 on the device. G_k (M,M,M) out; *A_pm out.
 * Context-free: runs on `device`. */
int p3m_gf_opt(int device, double kappa, double alpha, int p, int m_alias, int M,
               double box, double *G_k, double *A_pm);

/* gf_opt for callers that cannot allocate device memory (no counterpart in
 * the reference). Same kernel and result as p3m_gf_opt, but the caller
 * passes device pointers for the outputs -- G_k_dev (M*M*M doubles,
 * fftshifted layout) and A_pm_dev (one double) -- and the stream to launch
 * on; the call returns without waiting. The only scratch (one FP64 partial
 * per 256-point block) lives in a fixed file-scope device array of 8192
 * doubles (64 KiB, held on every GPU that loads the library until exit), so
 * M is limited to 128; larger M is rejected with P3M_EARG. The call
 * allocates nothing. Every call made outside stream capture looks up that
 * array's device address (cudaGetSymbolAddress); a call under capture reuses
 * the address the last uncaptured call found on that device, so make the
 * first call on a device -- and the first one after a cudaDeviceReset, which
 * unloads the library's device code -- before any stream capture (otherwise
 * P3M_ECUDA). All calls on a device share the array: calls that
 * overlap on the GPU race and must be ordered by the caller. Runs on the
 * current device. Message of the last failure: p3m_gf_opt_static_error(). */
int p3m_gf_opt_static(double kappa, double alpha, int p, int m_alias, int M, double box,
                      double *G_k_dev, double *A_pm_dev, void *stream);
const char *p3m_gf_opt_static_error(void);

/* Install the influence function the PM stage uses for `replica`, given in the
 * reference's fftshifted (M,M,M) layout (as returned by gf_opt). With
 * G_k == NULL the context computes it on the device itself. */
int p3m_set_green(p3m_ctx *ctx, int replica, const double *G_k);

/* yukawa_pm_ord6.py:440 particle_mesh_fft_r(...) -> (U_f, acc_f).
 * acc (n,3) out; *U out; Ep (3,n) out (may be NULL); rho (M,M,M) out (may be
 * NULL). */
int p3m_pm(p3m_ctx *ctx, int replica, const double *pos, const double *Z, double *acc,
           double *U, double *Ep, double *rho);

/* yukawa_p3m_ord6.py:6 force_pot(...) -> (U, acc), with acc = af*(pp+pm) and
 * U = uf*(U_pp + U_pm + U_self). parts (3) out: U_short, U_fft, U_self (may
 * be NULL). */
int p3m_force(p3m_ctx *ctx, int replica, const double *pos, const double *Z, double *acc,
              double *U, double *parts);

/* velocity_verlet_p3m_ord6.py:5 update(pos,vel,acc,dt,...) -> (pos,vel,acc,U)
 * in place on host arrays (n,3); *U out. */
int p3m_update(p3m_ctx *ctx, int replica, double *pos, double *vel, double *acc, double *U);

/* thermostat_p3m_ord6.py:5 vscale(pos,vel,acc,T_desired,PBC,it,...) in place;
 * *U and *T (temperature before the rescale) out. */
int p3m_vscale(p3m_ctx *ctx, int replica, int it, double *pos, double *vel, double *acc,
               double *U, double *T);

/* One row of n(q,t), yukawa_MD_p3m_ord6.py:215-219: out (nq,3) complex128 as
 * interleaved (re,im) doubles, for the wave numbers qv (nq). */
int p3m_nqt(p3m_ctx *ctx, int replica, const double *pos, const double *qv, int nq,
            double *out);

/* s_of_q_w.py:3 n_of_q_w(n_q_t, N, dt, T): S(q,w) of one run, per axis.
 * nqt (nt,3) complex128 as interleaved (re,im) in; out (nt,3) =
 * |dt FFT_t n|^2 / (N T). nt: a power of two <= 2^21, or any length <= 2^20
 * (Bluestein). Context-free: runs on `device`. */
int p3m_sqw_series(int device, const double *nqt, int nt, double N, double dt, double T,
                   double *out);

/* s_of_q_w_avg.py:5 s_of_q_w_avg_mat(n_q_t_array, Nq, sqw_mat, N_avg, N, dt, T):
 * nqt (nrun, nt, nq, 3) complex128 (the stacked n_q_t_<id>.npy files); out
 * (nrun, ncols, nt) = the mean over axes of n_of_q_w on q columns
 * col0 + i*col_stride (the reference: col0 0, col_stride 3, ncols Nq). */
int p3m_sqw_runs(int device, const double *nqt, int nrun, int nt, int nq, int col0, int col_stride,
                 int ncols, double N, double dt, double T, double *out);

/* ---- PPPM accuracy estimates. No counterpart in the reference, which sets
 * alpha, r_c and M by hand (yukawa_MD_p3m_ord6.py:52-68) and whose only
 * error measure is A_pm (yukawa_gf_opt.py:96). RMS per-particle force errors
 * for n unit charges at random positions in a box of side `box`, in the
 * reference's reduced units. */

/* PP truncation at r_c: dF^2 = 4 pi (n/box^3) int_rc^inf F_sr(r)^2 r^2 dr,
 * F_sr the Yukawa-Ewald short-range force of yukawa_pp.py:115-124 (host). */
int p3m_pp_error(double n, double box, double kappa, double alpha, double rc, double *dF);

/* Smallest r_c <= rc_max with p3m_pp_error <= tol; *rc = -1 when rc_max
 * misses tol (host). */
int p3m_pp_cutoff(double n, double box, double kappa, double alpha, double tol, double rc_max,
                  double *rc);

/* PM error of `count` parameter sets (device, FP64): the Q functional at the
 * optimal influence function, dF^2 = n/V^2 sum_k [sum_m k_m^2 G_m^2 - A(k)]
 * with the alias sum of yukawa_gf_opt.py:24-94; a_pm (may be NULL) receives
 * sum_k A(k), the reference's A_pm for the same parameters. */
int p3m_pm_error(int device, int count, const double *n, const double *box, const double *kappa,
                 const double *alpha, const int *M, int p, int m_alias, double *dF, double *a_pm);

/* ---- device-resident ("fast") path over all replicas ----------------------- */

/* Copy state in/out. Any of the pointers may be NULL. Arrays are (n,3). */
int p3m_set_state(p3m_ctx *ctx, int replica, const double *pos, const double *vel,
                  const double *acc);
int p3m_get_state(p3m_ctx *ctx, int replica, double *pos, double *vel, double *acc);

/* New thermostat targets T_desired (one per replica, > 0) for the following
 * p3m_run calls in thermostat mode (thermostat_p3m_ord6.py:5 T_desired). */
int p3m_set_t_desired(p3m_ctx *ctx, const double *t_desired);

/* The same for every replica at once: (sum of n, 3) arrays, replicas
 * concatenated in order, one copy per array (host buffers may be pinned).
 * p3m_set_state marks the replica's neighbour lists for a rebuild; with
 * keep_lists != 0 p3m_set_state_all keeps them, and the next step rebuilds a
 * replica's lists only if one of its particles has moved more than skin/2
 * since they were built (what p3m_run does between its own steps) -- for a
 * caller that continues a trajectory it read back. */
int p3m_set_state_all(p3m_ctx *ctx, const double *pos, const double *vel, const double *acc,
                      int keep_lists);
int p3m_get_state_all(p3m_ctx *ctx, double *pos, double *vel, double *acc);

/* The same copies queued on the context's stream without waiting for them
 * (with p3m_run(..., sync = 0) they let a caller keep one context's copies
 * in flight while another context computes). The host arrays must stay
 * valid, and unread or unchanged, until p3m_sync(ctx) returns; the copy
 * engines reach full speed only from pinned host memory. Errors surface at
 * p3m_sync / p3m_check. */
int p3m_set_state_all_async(p3m_ctx *ctx, const double *pos, const double *vel, const double *acc,
                            int keep_lists);
int p3m_get_state_all_async(p3m_ctx *ctx, double *pos, double *vel, double *acc);

/* What velocity_verlet_p3m_ord6.update (velocity_verlet_p3m_ord6.py:8-30)
 * hands back after a step -- the updated pos, vel, acc and the energies --
 * queued on the context's stream like p3m_get_state_all_async, for a caller
 * that keeps its state in host arrays: energies (may be NULL) receives
 * (U, K, T, thermostat factor) of every replica after the last step, (R, 4).
 * The device status word is staged with the copies, so the next p3m_sync
 * waits for the stream and reads no more device memory (unless more work
 * was queued after this call); energies is written when p3m_sync returns. */
int p3m_get_step_async(p3m_ctx *ctx, double *pos, double *vel, double *acc, double *energies);

/* Compute acc for the uploaded positions of all replicas (the driver's
 * initial force call, yukawa_MD_p3m_ord6.py:171). */
int p3m_init_forces(p3m_ctx *ctx);

/* Configure the per-step n(q,t) record: nq wave numbers per replica given as
 * multiples of 2*pi/L (qmult, nq), a ring of `capacity` steps. nq == 0
 * disables it. */
int p3m_set_nqt(p3m_ctx *ctx, const double *qmult, int nq, int capacity);

/* Advance all replicas n_steps. mode: P3M_MODE_NVE or P3M_MODE_THERMOSTAT
 * (it0 = step index of the first step, for the thermostat's it<=1999 switch).
 * record_nqt: accumulate n(q,t) rows each step. use_graph: capture the step
 * (and, on the FP32 path, a group of 8 steps) in CUDA graphs on first use
 * and replay them -- whole groups of 8 as one graph, the rest one step at a
 * time. sync: wait for completion. */
int p3m_run(p3m_ctx *ctx, int n_steps, int mode, int it0, int record_nqt, int use_graph,
            int sync);

/* S(q,w) of the last nt recorded n(q,t) rows (s_of_q_w.py:3-20,
 * s_of_q_w_avg.py:5-20, and the mean over runs of s_of_q_w_script.py:37):
 * for the q columns col0 + i*col_stride (i < ncols) -- the reference uses
 * every third column, its integer multiples of 2 pi/L -- the time FFT of each
 * axis, |dt X|^2 / (N_r T) with T = nt dt, averaged over the three axes.
 * out (ncols, nt): the mean over replicas (may be NULL); out_rep (R, ncols,
 * nt): per replica (may be NULL). nt as for p3m_sqw_series and at most the
 * ring capacity. */
int p3m_sqw(p3m_ctx *ctx, double dt, int col0, int col_stride, int ncols, int nt, double *out,
            double *out_rep);

/* Per-step energies recorded by p3m_run, (steps, R, 4) doubles:
 * U, K, T (before any rescale), and the thermostat factor applied. Returns
 * the number of steps copied in *n_out. */
int p3m_get_energies(p3m_ctx *ctx, double *out, int max_steps, int *n_out);

/* n(q,t) rows recorded by p3m_run for `replica`: (steps, nq, 3) complex as
 * interleaved (re,im) doubles. */
int p3m_get_nqt(p3m_ctx *ctx, int replica, double *out, int max_steps, int *n_out);

/* State snapshots for the output files of yukawa_MD_p3m_ord6.py:189-231
 * (pos_vel_acc.out, .xyz): with interval > 0, every step `it` of p3m_run
 * with (it + 1) % interval == 0 copies [pos | vel | acc] (n rows of 9) of
 * every replica into a device ring of `capacity` snapshots, inside the step
 * (no host round trip). interval 0 turns them off. Resets the ring. */
int p3m_set_snapshots(p3m_ctx *ctx, int interval, int capacity);

/* The snapshots taken since the last call, oldest first, at most max_snaps:
 * out (n_out, sum of n, 9), replicas concatenated; steps (may be NULL)
 * receives each one's step index. P3M_ESTATE if more than `capacity` were
 * taken since the last call (the oldest were overwritten). */
int p3m_get_snapshots(p3m_ctx *ctx, double *out, int *steps, int max_snaps, int *n_out);

/* Last values of one replica (8 doubles): U_short, U_fft, U_self, U, K, T,
 * thermostat factor, and the number of neighbour-list rebuilds so far. */
int p3m_get_replica_stats(p3m_ctx *ctx, int replica, double *out);

/* Device status word accumulated since the last call (P3M_OK or the first
 * error seen by a kernel), then cleared. Synchronises the stream. */
int p3m_check(p3m_ctx *ctx);

/* Scheduling priority of the context's streams (no counterpart in the
 * reference): level 0 is the highest priority the device offers, larger
 * levels are lower ones (clamped to the lowest). When several contexts share
 * a GPU -- an ensemble split so that one part's host copies overlap another
 * part's steps -- descending levels let the first part finish its step (and
 * start its copies back) while the others still compute. Waits for the
 * context's work, recreates its streams (p3m_stream then returns the new
 * one) and drops its captured step graphs, which the next p3m_run captures
 * again. */
int p3m_set_priority(p3m_ctx *ctx, int level);

/* Wait for all work on the context's stream; then, like p3m_check, report
 * a device status (out-of-box particle, non-finite force, list overflow)
 * raised by that work. */
int p3m_sync(p3m_ctx *ctx);

/* PP configuration: threads per particle in the force kernel (1, 2, 4, 8)
 * and the Verlet-list skin for every replica (< 0: each replica's own /
 * default). p3m_create picks tpi from the particle count; the autotuner of
 * the Python package times candidates and installs the fastest. Forces a
 * list rebuild. get returns tpi, replica 0's skin and the list capacity. */
int p3m_set_pp_config(p3m_ctx *ctx, int tpi, double skin);
int p3m_get_pp_config(p3m_ctx *ctx, int *tpi, double *skin, int *maxnb);

/* Kernel shapes of a context (no counterpart in the reference, whose PP and
 * PM stages have no GPU path): what the autotuner of the Python package
 * searches. p3m_create picks pp_tpi from the particle count, cell_div 2,
 * plane_max 64, gather_mode 1 and prune_buf 0. Setting waits
 * for the context's work, drops its captured step graphs and forces a list
 * rebuild. Every setting computes the same sums; they differ only in the
 * order of additions (pair order in the lists, lanes per particle, FFT
 * passes, entries beyond rc left out of the inner lists), so results agree
 * to rounding. */
typedef struct {
    int32_t pp_tpi;       /* threads per particle in the pair kernel: 1, 2, 4 or 8       */
    int32_t cell_div;     /* list cells are >= (rc + skin)/cell_div wide: 1 or 2          */
    int32_t plane_max;    /* meshes with sides up to this (0, 32 or 64) take the fused
                             y/z plane FFT kernel, larger ones the y and z pencil passes */
    int32_t gather_mode;  /* force gather: 0 = a CTA per mesh brick and field component,
                             1 = a CTA per brick (one tile buffer), 2 = a CTA per brick
                             with two buffers (FP32; FP64 takes 1 for 2)              */
    double skin;          /* Verlet skin for every replica (< 0: each replica's own /
                             the default); get returns the last value set              */
    double prune_buf;     /* FP32 path: 0 = the pair kernel reads the Verlet lists
                             (rc + skin); > 0 (below every skin) = it reads inner lists,
                             the Verlet-list entries closer than rc + prune_buf, which
                             it rebuilds itself whenever a particle of the replica has
                             moved prune_buf/2 since their last build (dynamic pruning)  */
} p3m_tuning;
int p3m_set_tuning(p3m_ctx *ctx, const p3m_tuning *t);
int p3m_get_tuning(p3m_ctx *ctx, p3m_tuning *t);

/* Number of inner-list builds of one replica that came without a Verlet-list
 * rebuild (steps with prune_buf > 0), as a double. */
int p3m_get_inner_builds(p3m_ctx *ctx, int replica, double *out);

/* Measurement: average device time (ms) of each step stage over `iters`
 * back-to-back launches, timed with CUDA events on the context's stream.
 * Stage i is named by p3m_stage_name(i); *n_out stages are written. The
 * drift stage moves the particles: call it after the run being measured. */
int p3m_profile_stages(p3m_ctx *ctx, int iters, double *ms, int max_stages, int *n_out);
const char *p3m_stage_name(int i);

/* Measurement: FP32 FMA throughput of `device` in TFLOP/s (8 independent FMA
 * chains per thread, 8 CTAs of 256 threads per SM) -- the denominator of the
 * FP32-pipe-bound PP kernel's roofline. */
int p3m_fp32_peak(int device, double *tflops);

/* Stream the context launches on (a cudaStream_t), for callers that time it
 * with their own events. */
void *p3m_stream(p3m_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* P3M_B200_H */
