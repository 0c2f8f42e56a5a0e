// Host-side launchers of the p3m_b200 kernels (internal to the library).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "p3m_common.cuh"

namespace p3m {

// Device arrays of one context, shared by all launchers. Particle arrays are
// concatenated over replicas in replica order; cell, brick and mesh arrays
// likewise. `T` selects the precision of the bulk buffers (void* here).
struct DevState {
    int nrep = 0, ntot = 0, ncell = 0, nbrick = 0;
    long long nmesh = 0, nspec = 0, ntile = 0;
    int wa = 0, wb = 0, wc = 0;  // total work items of the mesh passes
    int wp = 0;                  // plane items (fused y/z passes)
    int max_plane = 0;           // largest M among plane replicas
    int pp_tpi = 1;              // threads per particle in the PP force kernel
    int cell_div = CELL_DIV_MAX; // PP cells are >= (rc + skin) / cell_div wide (1 or 2)
    int plane_max = 64;          // meshes up to this side take the fused y/z plane kernel
    int gather_mode = 1;         // gather: 0 a CTA per brick and component, 1 / 2 a CTA per
                                 // brick with one / two tile buffers (2: FP32 only)
    int pp_nblk = 0;             // blocks of the PP force kernel (replica-aligned)
    int maxnb = 0;               // list capacity per particle
    double prune_buf = 0.0;      // inner-list buffer beyond rc (FP32; 0: no inner lists)
    int maxnb_in = 0;            // inner-list capacity per particle
    int has_mesh = 0;
    int max_mesh = 0;            // largest M over replicas
    int nblk = 0;                // replica-aligned particle blocks (PBLK each)
    int nq_nblk = 0;             // replica-aligned blocks of the n(q,t) kernel
    RepDev *reps = nullptr;      // [nrep]
    // particle state, FP64 (ntot,3) row-major in original order
    double *pos = nullptr, *vel = nullptr, *acc = nullptr, *charge = nullptr;
    int *prep = nullptr;         // particle -> replica
    // cell sort
    int *cell_key = nullptr, *cell_count = nullptr, *cell_start = nullptr;
    int *cell_cursor = nullptr, *cell_tmp = nullptr, *cell_perm = nullptr, *cell_slot = nullptr;
    void *xq = nullptr;          // integer coordinates in sorted order (uint4 / ulonglong4)
    int *nnb = nullptr;          // list length per sorted particle
    int *cell_sub = nullptr;     // [particle] sub-cell Morton code (rebuild steps)
    int *nlist = nullptr;        // neighbour lists (sorted indices), in 16-entry group blocks (list_index)
    int *rebuild = nullptr;      // per-replica flags: rebuild cells and lists this step
    // the replicas rebuilding this step (written by k_scan): [0] = count k,
    // [1 .. k] replica indices, [nrep + 1 + j] = cells of the first j of them
    int *rb_list = nullptr;
    double *pos_ref = nullptr;   // positions at the last rebuild (ntot,3)
    // inner lists (prune_buf > 0): the outer entries closer than rc + prune_buf,
    // in outer-list order and the same layout, rebuilt by the pair kernel on the
    // steps a replica's flag is set
    int *nnb_in = nullptr, *nlist_in = nullptr;
    int *prune = nullptr;        // per-replica flags: rebuild the inner lists this step
    double *pos_pref = nullptr;  // positions at the last inner-list build (ntot,3)
    double *prune_count = nullptr;  // per replica: inner-list builds between outer rebuilds
    float4 *pp_tables = nullptr; // FP32 pair tables: cubic of psi = phi r, [nrep][PP_TABLE_N]
    void *acc_pp = nullptr;      // V4<T> PP acceleration, cell-sorted order
    // brick sort
    int *brick_key = nullptr, *brick_count = nullptr, *brick_start = nullptr;
    int *brick_cursor = nullptr, *brick_perm = nullptr, *brick_slot = nullptr;
    int *brick_hist = nullptr;   // [replica][chunk][brick] counts, then chunk offsets
    int nchunk = 0, max_bricks = 0, sort_ch = 2048;  // chunks, bricks of the largest mesh, chunk size
    // mesh
    void *tiles = nullptr;       // T assignment tiles [brick][TILE^3]
    void *spec = nullptr;        // C2<T> half spectrum rho_k / phi_k, [kx][z][y]
    void *ek = nullptr;          // C2<T> 3 field spectra, [3][kx][z][y]
    void *green = nullptr;       // T influence function / V, [kx][z][y]
    void *efield = nullptr;      // T 3 real field meshes [3][z][y][x]
    void *acc_pm = nullptr;      // V4<T> PM acceleration, brick-sorted order
    void *twiddle = nullptr;     // C2<T> exp(-2 pi i k / 256), k < 128
    // reductions
    double *u_pp_part = nullptr;  // [pp_nblk]
    double *u_pm_part = nullptr;  // [wc + wp]
    double *kin_part = nullptr;   // per particle block
    double *rep_out = nullptr;    // [nrep * 8] per-replica scalars of the last step
    int *status = nullptr;
};

enum RepOut { RO_UPP = 0, RO_UPM = 1, RO_USELF = 2, RO_U = 3, RO_K = 4, RO_T = 5, RO_FACT = 6,
              RO_REBUILDS = 7 };


template <typename T> void configure_pp_kernels();
template <typename T> void configure_mesh_kernels();
template <typename T> void launch_keys(const DevState &s, cudaStream_t st);
void launch_cell_keys(const DevState &s, cudaStream_t st);
void launch_scan(const DevState &s, cudaStream_t st, int part = -1);  // -1 both, 0 cells, 1 bricks
void launch_scatter(const DevState &s, cudaStream_t st);
template <typename T> void launch_fix_cells(const DevState &s, cudaStream_t st);
void launch_sort_bricks(const DevState &s, cudaStream_t st);  // 3 kernels
template <typename T> void launch_quantize(const DevState &s, cudaStream_t st);
template <typename T> void launch_build_lists(const DevState &s, cudaStream_t st);
template <typename T> void launch_pp(const DevState &s, cudaStream_t st);
int pp_particles_per_block(int tpi);
void launch_reduce_pp(const DevState &s, cudaStream_t st);

template <typename T> void launch_assign(const DevState &s, cudaStream_t st);
template <typename T> void launch_fft_forward(const DevState &s, cudaStream_t st);
template <typename T> void launch_fft_inverse(const DevState &s, cudaStream_t st);
template <typename T> void launch_gather(const DevState &s, cudaStream_t st);
void launch_reduce_pm(const DevState &s, cudaStream_t st);
int fft_kernel_count(const DevState &s);
int plane_max_mesh();

template <typename T> void launch_green_from_host_layout(const DevState &s, int rep,
                                                         const double *gk_dev,
                                                         cudaStream_t st);
template <typename T> void launch_tiles_to_mesh(const DevState &s, int rep, double *rho,
                                                cudaStream_t st);
template <typename T> void launch_efield_from_mesh(const DevState &s, int rep,
                                                   const double *ex, const double *ey,
                                                   const double *ez, cudaStream_t st);
void launch_gf_opt(double kappa, double alpha, int p, int m_alias, int M, double L,
                   double *G_k, double *a_part, cudaStream_t st);

void launch_kick_drift(const DevState &s, cudaStream_t st);
template <typename T> void launch_kick_finish(const DevState &s, int do_kick, double *ep_out,
                                              cudaStream_t st);
// Sums that k_step_reduce can take over from k_reduce_pp, k_reduce_pm and
// k_nqt_reduce inside a step (NULL pointers: not this time).
struct StepSums {
    const double *u_pp_part = nullptr;  // PP block partials (with u_pm_part)
    int pp_nblk = 0;
    const double *u_pm_part = nullptr;
    int wc_total = 0, wp_total = 0;
};
void launch_step_reduce(const DevState &s, int mode, int *counters, double *ring, int ring_cap,
                        cudaStream_t st, int recorded = 0, int snap_interval = 0,
                        int snap_cap = 0, const StepSums &sums = StepSums());
void launch_snapshot(const DevState &s, const int *counters, double *snap, int *steps,
                     cudaStream_t st);
void launch_set_counters(int *counters, int run_step, int ring_pos, int it0, cudaStream_t st);
void launch_set_flags(int *flag, int n, int value, cudaStream_t st);
void launch_scale_vel(const DevState &s, cudaStream_t st);
template <typename T> void launch_combine(const DevState &s, int use_pp, int use_pm, int scale_af,
                                          double *out, double *ep_out, cudaStream_t st);
template <typename T> void launch_nqt(const DevState &s, const double *pos, const double *qmult,
                                      int nq, int consecutive, double *part, double *out,
                                      const int *counters, int ring_cap, cudaStream_t st);
int nqt_particles_per_block();
template <typename T> void configure_integrate_kernels(int max_nq);
int gf_opt_blocks(int M);
double fp32_fma_tflops(int device);
// S(q, omega) of recorded n(q,t) series (p3m_sqw.cu)
struct SqwArgs {
    const double2 *src;       // series element (row, r, col, ax) at row*row_stride + r*rep_stride + col*3 + ax
    long long row_stride, rep_stride;
    int cap, row0;            // row(t) = (row0 + t) % cap
    int r0, nrep_launch;      // replicas r0 .. r0 + nrep_launch - 1
    int col0, col_stride, ncols, nt, logP, bluestein;
    const double2 *chirp_fft_br;  // Bluestein chirp spectrum, 2^logP points, bit-reversed
    const double *nrep_n;     // particles per replica
    double dt;
    int per_axis;
    double *out_rep;
};
int sqw_max_points();   // largest transform length
int sqw_smem_points();  // largest transform length held in shared memory
void launch_sqw(const SqwArgs &a, double2 *gscratch, cudaStream_t st);
void launch_sqw_mean(const double *out_rep, int nrep, long long n, double *out, cudaStream_t st);
// PPPM error estimates (p3m_tune.cu)
double pp_error_estimate(double n_particles, double box, double kappa, double alpha, double rc);
double pp_cutoff_for(double n_particles, double box, double kappa, double alpha, double tol,
                     double rc_max);
int pm_error_blocks(int M);
void launch_pm_error(double kappa, double alpha, int p, int m_alias, int M, double L,
                     double *q_part, double *a_part, cudaStream_t st);


}  // namespace p3m
