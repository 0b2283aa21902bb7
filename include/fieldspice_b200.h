/*
 * fieldspice_b200 -- C ABI of the B200 elliptic-solve library.
 *
 * The library solves the finite-integration system  G^T M G phi = f  on a
 * rectilinear node grid, matrix-free, with the Dirichlet rows eliminated
 * symmetrically.  Every pointer below is DEVICE memory unless the comment says
 * "host"; every function returns an FS_* status code and never throws.
 *
 * Node layout.  A grid has nx*ny*nz nodes stored in C order, z fastest:
 *     n = (i*ny + j)*nz + k.
 * A field with `nrhs` right-hand sides is stored RHS-interleaved, so value
 * (n, r) sits at  n*nrhs + r.
 *
 * Edge masses.  The reference keeps one concatenated edge vector
 * [x-edges (nx-1,ny,nz) | y-edges (nx,ny-1,nz) | z-edges (nx,ny,nz-1)]
 * (fieldspice/grid.py:322-327).  Here each direction is padded to the node
 * shape: mx[n] is the mass of the x-edge from node (i,j,k) to (i+1,j,k) and is
 * 0 on the last x-plane; my and mz likewise.  This keeps all arrays in the
 * node index space, so a kernel addresses masses and potentials alike.
 *
 * Labels.  One byte per node: FS_LABEL_FREE (unknown) or FS_LABEL_FIXED
 * (Dirichlet, its value held in phi).  The solver further classifies free
 * nodes that are coupled to no other free node as "solo" (solved directly,
 * poisson.py:336-362) and free nodes with no incident mass as "pinned" to 0
 * (poisson.py:282-295).
 */
#ifndef FIELDSPICE_B200_H
#define FIELDSPICE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define FS_OK 0
#define FS_NOT_CONVERGED 1   /* iteration cap reached above tolerance        */
#define FS_TIMEOUT 2         /* the device did not report completion          */
#define FS_BAD_ARG 3         /* invalid size, pointer or option              */
#define FS_NAN 4             /* a residual norm became NaN or Inf             */
#define FS_CUDA_ERROR 5      /* a CUDA runtime call failed                    */
#define FS_STALLED 6         /* mixed precision: FP32 iterations stopped
                                reducing the FP64 residual (solve again in
                                FS_PRECISION_FP64, warm-started)               */

/* ---- enumerations ------------------------------------------------------ */
#define FS_LABEL_FREE 0
#define FS_LABEL_FIXED 1
#define FS_LABEL_SOLO 2
#define FS_LABEL_PINNED 3

#define FS_DTYPE_F64 0
#define FS_DTYPE_F32 1

#define FS_PRECISION_FP64 0  /* every vector and mass in FP64                 */
#define FS_PRECISION_MIXED 1 /* FP32 inner CG, FP64 reliable updates          */

#define FS_AVERAGE_PARALLEL 0 /* dual-area weighted arithmetic mean           */
#define FS_AVERAGE_HARMONIC 1 /* dual-area weighted harmonic mean             */

#define FS_PRECOND_JACOBI 0  /* CG on the Jacobi-equilibrated system          */
#define FS_PRECOND_MG 1      /* geometric multigrid V-cycle preconditioner    */
#define FS_PRECOND_MG_AGG 2  /* multigrid V-cycle on 2x2x2 aggregates with
                                Galerkin coarse operators (P^T A P): for
                                strongly discontinuous coefficients        */

typedef struct fs_rhs_stats {
  int32_t iterations;       /* CG iterations taken                            */
  int32_t status;           /* FS_OK, FS_NOT_CONVERGED, FS_STALLED, FS_NAN    */
  double relres;            /* final FP64 true relative residual              */
  double bnorm;             /* ||D^-1/2 b_free||_2 of the eliminated system   */
  int32_t reliable_updates; /* FP64 residual replacements performed           */
  int32_t reserved;
} fs_rhs_stats;

typedef struct fs_pcg_plan fs_pcg_plan;

/* ---- library ----------------------------------------------------------- */
const char* fs_version(void);
const char* fs_status_string(int status);
/* Last CUDA error text recorded by a failing call on this thread (host).    */
const char* fs_last_error(void);

/* ---- a1-a3: material averaging and edge masses ----------------------------
 * Replaces fieldspice/operators.py:144-237 (cell_to_edge) followed by
 * operators.py:302-315 (edge_mass): for every edge the dual-area weighted
 * mean of the (up to) four cells around it, times dual area over length.
 * prop_cell: (nx-1)*(ny-1)*(nz-1) FP64 per-cell property, C order.
 * h*, hd*: primal widths (n-1) and dual widths (n) per axis, FP64 device
 * arrays, computed on the host exactly as fieldspice/grid.py:196-207.
 * Writes padded node-shaped mx, my, mz (FP64).  The arithmetic order follows
 * the reference so that the result is bit-identical to it.                  */
int fs_build_masses(const double* prop_cell, const double* hx, const double* hy,
                    const double* hz, const double* hxd, const double* hyd,
                    const double* hzd, int nx, int ny, int nz, int mode,
                    double* mx, double* my, double* mz, void* stream);

/* Edge masses of the wrap-around grid of periodic axes `periodic` (bit 0 x,
 * 1 y, 2 z; fieldspice/boundaries.py periodic_pairs and the node merge of
 * poisson.py:665-719): m_full is the 3 x N output of fs_build_masses on the
 * nx x ny x nz grid, m_reduced (3 x N', FP64) receives the masses of the grid
 * with the last plane of every periodic axis merged into the first (each
 * reduced node sums its merged nodes' masses; the last reduced plane's
 * own-direction mass is the wrap edge).  Reduced axes need >= 2 nodes.       */
int fs_periodic_masses(const double* m_full, int nx, int ny, int nz, int periodic,
                       double* m_reduced, void* stream);

/* out = a*m1 + b*m2 elementwise over n values (FP64).  Builds the EQS masses
 * M_eps/dt + theta*M_sigma (fieldspice/solvers/eqs.py:279-280).            */
int fs_combine_masses(const double* m1, const double* m2, double a, double b,
                      double* out, long long n, void* stream);

/* ---- a5: stencil apply ----------------------------------------------------
 * y = (G^T M G) x, the operator of fieldspice/operators.py:340-351 applied
 * matrix-free.  With `label` non-NULL the apply is the eliminated operator of
 * operators.py:362-407: x is read as 0 on non-free nodes and y is written 0
 * there.  dtype selects FP64 or FP32 for x, y and the masses.               */
int fs_stencil_apply(const void* x, void* y, const void* mx, const void* my,
                     const void* mz, const uint8_t* label, int nx, int ny,
                     int nz, int nrhs, int dtype, void* stream);

/* ---- a6/a10: Dirichlet excitation -------------------------------------------
 * phi[n*nrhs + r] = (group[n] == r) ? 1 : 0 for every node whose label is
 * fixed, and 0 on free nodes: the unit excitation of capacitance column r
 * (fieldspice/solvers/poisson.py:1212-1217).  group: int16 per node, -1 for
 * nodes in no terminal.                                                       */
int fs_fill_unit_excitation(const int16_t* group, const uint8_t* label,
                            double* phi, int nx, int ny, int nz, int nrhs,
                            void* stream);

/* phi[n] = values[group[n]] on fixed nodes with group[n] >= 0 (one RHS):
 * the per-step Dirichlet values of fieldspice/solvers/eqs.py:108-129.        */
int fs_set_dirichlet(const int16_t* group, const uint8_t* label,
                     const double* values, double* phi, int nx, int ny, int nz,
                     void* stream);

/* ---- a7-a9: the eliminated CG solve ----------------------------------------
 * Replaces LinearSystem (fieldspice/solvers/poisson.py:260-589) for the
 * symmetric positive definite Dirichlet-eliminated system, with the
 * reference's stopping rule: ||D^-1/2 (b - A x)||_2 < tol*||D^-1/2 b||_2 on
 * the free nodes (SciPy CG on the equilibrated matrix, poisson.py:364-377,
 * 533-552).  The plan is bound to one operator, one label array and one phi
 * buffer (N*nrhs FP64, fixed values in place, the initial guess on free
 * nodes) and an optional source f (N*nrhs FP64, may be NULL).
 * nrhs must be 1, 2, 4, 8 or 16.  precond: FS_PRECOND_JACOBI (CG on the
 * equilibrated system, the reference's method), FS_PRECOND_MG (a
 * geometric-multigrid V-cycle with Chebyshev smoothing as the
 * preconditioner; same stopping rule) or FS_PRECOND_MG_AGG (the same V-cycle
 * on a hierarchy of 2x2x2 node aggregates whose coarse operators are the
 * Galerkin products P^T A P, robust to coefficient jumps of many orders of
 * magnitude, e.g. copper against oxide).  workspace must hold
 * fs_pcg_workspace_bytes() bytes and stay alive until destroy.              */
int fs_pcg_workspace_bytes(int nx, int ny, int nz, int nrhs, int precision,
                           int precond, size_t* bytes);
int fs_pcg_plan_create(int nx, int ny, int nz, int nrhs, int precision,
                       int precond, const double* mx, const double* my,
                       const double* mz, const uint8_t* label_in, double* phi,
                       const double* f, void* workspace, size_t workspace_bytes,
                       fs_pcg_plan** plan, void* stream);
/* The same system plus a node-diagonal term: A = G^T M G + diag(d), d >= 0
 * (FP64, one value per node; the heat capacity / dt and convective wall
 * terms of ThermalSolver, thermal.py:140-160,200-290).  The array must stay
 * valid for the plan's lifetime.                                           */
int fs_pcg_plan_create_diag(int nx, int ny, int nz, int nrhs, int precision,
                            int precond, const double* mx, const double* my,
                            const double* mz, const double* diag,
                            const uint8_t* label_in, double* phi,
                            const double* f, void* workspace, size_t workspace_bytes,
                            fs_pcg_plan** plan, void* stream);
/* The same with periodic axes (bit 0 x, bit 1 y, bit 2 z): the grid is the
 * reduced node set of fieldspice's wrap-around identification (the last node
 * plane of a periodic axis merged into the first, poisson.py:665-719, 942-955),
 * and the first and last planes of each periodic axis are joined by a wrap
 * edge whose mass is stored on the last plane (mx at i = nx-1, and so on).
 * precond = FS_PRECOND_JACOBI or FS_PRECOND_MG_AGG (the node aggregates wrap
 * with the grid); FS_PRECOND_MG is refused with FS_BAD_ARG.                 */
int fs_pcg_plan_create_ex(int nx, int ny, int nz, int nrhs, int precision, int precond,
                          const double* mx, const double* my, const double* mz,
                          const double* diag, int periodic, const uint8_t* label_in,
                          double* phi, const double* f, void* workspace,
                          size_t workspace_bytes, fs_pcg_plan** plan, void* stream);
/* The solve of fs_pcg_plan_solve without blocking the host: begin enqueues
 * the initialisation and the first graph chunk on stream and returns; each
 * poll returns at once.  While the plan runs, poll sets *done = 0 and, when
 * the last enqueued step has completed, enqueues the next one (a chunk, or
 * the finalisation once every RHS is done or the chunk cap is reached).
 * When the finalisation has landed it sets *done = 1, fills stats (nrhs
 * entries, or NULL) and returns what fs_pcg_plan_solve would.  Other
 * returns with *done = 0 are errors (the plan is idle again).  A plan runs
 * one solve at a time; it must not be destroyed or solved otherwise until
 * poll has reported *done = 1.  Drives many plans from one host thread
 * while it builds more of them (batched extraction).                       */
int fs_pcg_plan_solve_begin(fs_pcg_plan* plan, int warm_start, double tol, int maxiter,
                            void* stream);
int fs_pcg_plan_solve_poll(fs_pcg_plan* plan, fs_rhs_stats* stats, int* done);
/* Multigrid and stencil options of one plan.  The plan copies them when it is
 * created; the library keeps no process-wide setting (the stencil autotuner's
 * table is a cache of measured choices per shape class, nothing else).
 * smooth_deg, smooth_lo: Chebyshev smoothing degree (pre and post, 1..16)
 * and the lower end of its interval [smooth_lo, 2] on the unit-diagonal level
 * operators; coarse_deg, coarse_lo: the same on the coarsest level (1..64);
 * coarsest_nodes: coarsening stops at or below this node count (>= 8);
 * stencil_kind: the CG stencil (0..7, see fs_pcg_plan_stencil_kind) or -1
 * (the FS_STENCIL environment variable, else autotuned); agg_alpha: the
 * factor (0 < agg_alpha < 2) on every coarse correction of the aggregation
 * hierarchy (FS_PRECOND_MG_AGG; over-correction for its piecewise-constant
 * prolongation).  fs_mg_params_default fills 2, 0.3, 32, 0.06, 4096, -1, 1.7. */
typedef struct fs_mg_params {
  int smooth_deg;
  double smooth_lo;
  int coarse_deg;
  double coarse_lo;
  long long coarsest_nodes;
  int stencil_kind;
  double agg_alpha;
} fs_mg_params;
void fs_mg_params_default(fs_mg_params* params);
/* fs_pcg_workspace_bytes and fs_pcg_plan_create_ex with options (NULL: the
 * defaults); FS_BAD_ARG if an option is out of range.  The workspace size
 * depends on coarsest_nodes (the number of levels).                        */
int fs_pcg_workspace_bytes_opt(int nx, int ny, int nz, int nrhs, int precision,
                               int precond, const fs_mg_params* opt, size_t* bytes);
int fs_pcg_plan_create_opt(int nx, int ny, int nz, int nrhs, int precision, int precond,
                           const double* mx, const double* my, const double* mz,
                           const double* diag, int periodic, const fs_mg_params* opt,
                           const uint8_t* label_in, double* phi, const double* f,
                           void* workspace, size_t workspace_bytes, fs_pcg_plan** plan,
                           void* stream);
/* Solve in place into phi.  warm_start != 0 keeps the free-node values of
 * phi as the initial guess (the tolerance stays relative to ||b||, as in
 * SciPy); otherwise the guess is 0.  maxiter <= 0 caps the iterations at the
 * reference's max(500, 10 sqrt(n_free)) (poisson.py:535-536) from the plan's
 * own classification, on the device.  stats: host array of nrhs entries.
 * Returns FS_OK when every RHS converged, FS_NOT_CONVERGED if one hit
 * maxiter, FS_STALLED if a mixed-precision RHS stopped making progress,
 * FS_NAN on breakdown, FS_TIMEOUT if a staged load never arrived.           */
int fs_pcg_plan_solve(fs_pcg_plan* plan, int warm_start, double tol,
                      int maxiter, fs_rhs_stats* stats, void* stream);
/* Solve several independent plans (a batch of geometries) together: plan i
 * runs on streams[i], one graph chunk per unfinished plan per round, so the
 * iterations of small systems overlap those of large ones.  stats[i]: host
 * array of plan i's nrhs entries (or NULL); status[i]: plan i's result as
 * fs_pcg_plan_solve would return it.  Returns FS_OK when every plan is.    */
int fs_pcg_plans_solve(fs_pcg_plan* const* plans, int nplans,
                       void* const* streams, int warm_start, double tol,
                       int maxiter, fs_rhs_stats* const* stats, int* status);
/* Label array after classification (free / fixed / solo / pinned), device. */
const uint8_t* fs_pcg_plan_labels(const fs_pcg_plan* plan);
/* Number of kernel launches issued by the last solve (host count).          */
long long fs_pcg_plan_launches(const fs_pcg_plan* plan);
/* Device time of the CG kernels -- p update (p = r + beta p), stencil
 * (A~p, p.q), update (x, r, r.r), reliable update, the preconditioner
 * (V-cycle and r.z; 0 without one) and one fine-level multigrid smoothing
 * step (average over the post-smoothing launches) -- summed over the samples
 * taken during the last solve: the first CG iteration of every graph launch
 * is bracketed by CUDA events.  ms: host array of 6.                        */
int fs_pcg_plan_kernel_times(const fs_pcg_plan* plan, double* ms,
                             long long* samples);
int fs_pcg_plan_destroy(fs_pcg_plan* plan);

/* ---- a10/a13: charge and current integration (FP64) -----------------------
 * out[g*nrhs + r] = sum over nodes n of group g of
 *                   (L_A u)[n, r] - (L_B w)[n, r]
 * where L_A = G^T diag(mA) G and, when mBx is non-NULL, L_B likewise.  The
 * groups are given as a concatenated node list `nodes` (int64) with
 * offsets[0..ngroups].  With B absent this is the terminal charge
 * C[i,j] = sum_{n in T_i} (L phi_j)_n of poisson.py:1219-1221; with
 * A = K, B = Kexp it is the terminal current of eqs.py:328-340.
 * workspace: fs_group_apply_workspace_bytes() bytes.                         */
int fs_group_apply_workspace_bytes(int ngroups, int nrhs, size_t* bytes);
int fs_group_apply(const double* mAx, const double* mAy, const double* mAz,
                   const double* u, const double* mBx, const double* mBy,
                   const double* mBz, const double* w, const long long* nodes,
                   const long long* offsets, int ngroups, int nx, int ny,
                   int nz, int nrhs, double* out, void* workspace,
                   size_t workspace_bytes, void* stream);

/* Allocation-free variant of fs_group_apply, for callers that cannot let a
 * library allocate device memory: hosts that hand the library only their
 * own input and output buffers from a pre-reserved pool (a Go or JVM
 * application binding through cgo or JNI, a real-time time-stepping loop
 * that must not stall on cudaMalloc), so there is no workspace argument.
 * No counterpart in the reference (it allocates freely in NumPy); same
 * arguments and result as fs_group_apply minus the workspace.
 * Scratch is a static device array inside the library: 512 KiB + 256 B per
 * GPU that loads the library, held until the process exits, so
 * ngroups * nrhs must not exceed 2048 (larger sizes return FS_BAD_ARG with
 * the reason in fs_last_error()).  The first call on each device looks up
 * the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  That address
 * is kept for the life of the process, so a cudaDeviceReset between calls
 * is not supported.  nrhs must be 1, 2, 4, 8 or 16; every argument is
 * checked before the array is touched.  Every call
 * shares the one array and it keeps the previous call's contents: calls
 * that overlap on the GPU (two streams, two host threads) race on it and
 * must be serialised by the caller.  Never allocates or frees memory.     */
int fs_group_apply_noalloc(const double* mAx, const double* mAy,
                           const double* mAz, const double* u,
                           const double* mBx, const double* mBy,
                           const double* mBz, const double* w,
                           const long long* nodes, const long long* offsets,
                           int ngroups, int nx, int ny, int nz, int nrhs,
                           double* out, void* stream);

/* out[r] = sum over edges of m_e (u_head - u_tail)^2 = u^T L u per RHS: the
 * stored energy 2*W of poisson.py:905-913 and eqs.py:342-348.               */
int fs_quadform_workspace_bytes(int nrhs, size_t* bytes);
int fs_quadform(const double* mx, const double* my, const double* mz,
                const double* u, int nx, int ny, int nz, int nrhs,
                double* out, void* workspace, size_t workspace_bytes,
                void* stream);

/* out = L u + add (add may be NULL), FP64, every node: the explicit part
 * Kexp @ phi + inject of eqs.py:293.                                         */
int fs_apply_laplacian(const double* mx, const double* my, const double* mz,
                       const double* u, const double* add, double* out, int nx,
                       int ny, int nz, int nrhs, void* stream);


/* ---- Learned preconditioner: BF16 3-D convolution on tensor cores ------ *
 * Activations: BF16, channels-last on a one-voxel zero halo,
 * [batch][X+2][Y+2][Z+2][ctot] (a 16-byte aligned base, ctot a multiple of
 * 8).  Weights: FP32 w[27][cout][cin], taps ordered (dx, dy, dz) with z
 * fastest, offsets -1..1 (the cross-correlation of a padded conv3d).
 * fs_conv3d_pack_weights writes their BF16 tensor-core image (27*cin*cout
 * elements); flip != 0 packs the data-gradient operator (taps reversed,
 * channel roles swapped) for a convolution from cout to cin channels.
 * fs_conv3d_bf16: y[.., cout_off + co] = act(bias + sum W x[.., cin_off + ci]),
 * act = ReLU when relu != 0, times (mask > 0) channel-wise when mask is not
 * NULL, added to y when accumulate != 0; halo rows of y are written as 0
 * (left untouched when accumulating).  cin, cout: multiples of 16, cout
 * <= 128.  error: optional device int set to 1 if a staged load timed out. */
int fs_conv3d_pack_weights(const float* w, int cin, int cout, int flip, void* wpack,
                           void* stream);
int fs_conv3d_bf16(const void* x, int ctot_in, int cin_off, int cin, const void* wpack,
                   const float* bias, void* y, int ctot_out, int cout_off, int cout,
                   const void* mask, int ctot_mask, int mask_off, int batch, int X, int Y,
                   int Z, int relu, int accumulate, int* error, void* stream);
/* Weight and bias gradient of the convolution above from its input x and the
 * gradient dy of its output (same layouts, channel slices as above):
 * dw[t][co][ci] = sum over voxels of dy[v][co] x[v + off_t][ci] (FP32,
 * written), db[co] = sum of dy[v][co] (FP32, written; may be NULL).  The
 * reduction over voxels runs on tcgen05 tensor cores (BF16 operands, FP32
 * accumulation in tensor memory).  cin, cout: multiples of 16, cin <= 160,
 * cout <= 128; dy must be zero on halo rows (as fs_conv3d_bf16 writes it).
 * workspace: fs_conv3d_wgrad_workspace_bytes() bytes, 256-byte aligned.    */
int fs_conv3d_wgrad_workspace_bytes(int cin, int cout, size_t* bytes);
int fs_conv3d_wgrad_bf16(const void* x, int ctot_in, int cin_off, int cin, const void* dy,
                         int ctot_out, int cout_off, int cout, int batch, int X, int Y, int Z,
                         float* dw, float* db, void* workspace, size_t workspace_bytes,
                         int* error, void* stream);


/* ---- Learned preconditioner: the U-Net --------------------------------- *
 * A 4-level BF16 3-D U-Net (channels 16/32/48/64, fourteen 3x3x3
 * convolutions on tensor cores, ReLU, average pooling, nearest upsampling
 * with skip concatenation, a 1x1 FP32 head) mapping a level residual and the
 * level's equilibrated masses and fixed flags to an error estimate.
 * Parameters: one caller-owned FP32 device vector theta of
 * fs_unet_param_count() entries; fs_unet_layer(l) gives layer l's channels
 * and the offsets of its weights [27][cout][cin] and bias (l = 14: the head,
 * 16 weights then 1 bias).  train != 0 adds gradients and Adam state.      */
typedef struct fs_unet fs_unet;
int fs_unet_param_count(long long* n);
int fs_unet_layer(int l, int* cin, int* cout, long long* woff, long long* boff);
int fs_unet_workspace_bytes(int X, int Y, int Z, int batch, int train, size_t* bytes);
int fs_unet_create(int X, int Y, int Z, int batch, int train, float* theta, void* workspace,
                   size_t workspace_bytes, fs_unet** net, void* stream);
/* Re-pack the tensor-core weight images after theta changed on the host side. */
int fs_unet_sync(fs_unet* net, void* stream);
/* out[b*out_sb + n*out_sn] = network(rhs_b, em_b, label_b) in rhs units, 0 on
 * fixed nodes.  rhs[b*rhs_sb + n*rhs_sn]; em: sample b's +x, +y, +z masses at
 * em + b*em_sb + {0, N, 2N} (FP32); label[b*label_sb + n] (FS_LABEL_*).      */
int fs_unet_forward(fs_unet* net, const float* rhs, long long rhs_sn, long long rhs_sb,
                    const float* em, long long em_sb, const uint8_t* label, long long label_sb,
                    float* out, long long out_sn, long long out_sb, void* stream);
/* One Adam step on the relative squared error of the network's output
 * against target (planar [batch][N] inputs, em [batch][3][N]); loss: device
 * float receiving the batch loss before the step (or NULL).                */
int fs_unet_train_step(fs_unet* net, const float* rhs, const float* em, const uint8_t* label,
                       const float* target, float lr, float* loss, void* stream);
/* The same loss and its gradient dL/dtheta (device, theta-sized), no update. */
int fs_unet_gradient(fs_unet* net, const float* rhs, const float* em, const uint8_t* label,
                     const float* target, float* grad, float* loss, void* stream);
/* One Adam step of theta on a caller's gradient (device, theta-sized), e.g.
 * the gradients of fs_unet_gradient averaged over data-parallel ranks by an
 * all-reduce; then the weight images are re-packed.  fs_unet_gradient
 * followed by this step equals fs_unet_train_step on the same batch.       */
int fs_unet_adam_step(fs_unet* net, const float* grad, float lr, void* stream);
/* Host int: 1 if a staged load of a network convolution timed out.        */
int fs_unet_error(const fs_unet* net, int* flag, void* stream);
int fs_unet_destroy(fs_unet* net);


/* ---- Learned preconditioner inside a CG plan --------------------------- *
 * A mixed-precision multigrid plan can stop its V-cycle at `level` and ask
 * the U-Net (parameters theta, caller-owned, read at every application) for
 * that level's correction instead of recursing: smoothing on the levels
 * above, the network below.  The preconditioner is then nonlinear, so the
 * plan switches to flexible CG (beta = -z.Ap / p.Ap).  mode 0: the network's
 * output is the level's correction; mode 1: the network's output plus a
 * V-cycle from that level on its residual.  level = -1 restores plain
 * multigrid.  fs_pcg_plan_levels: the level count and dims (3 ints
 * per level); fs_pcg_plan_level_data: a level's equilibrated masses (FP32 in
 * a mixed plan), labels and diag^-1/2 (NULL on level 0).                   */
int fs_pcg_plan_levels(const fs_pcg_plan* plan, int* nlev, int* dims);
/* y = A~ x for an equilibrated level operator (FP32, nrhs-interleaved,
 * unit diagonal, masses ex/ey/ez of fs_pcg_plan_level_data); 0 on nodes
 * whose label is not FS_LABEL_FREE.                                         */
int fs_eq_apply(const float* x, float* y, const float* ex, const float* ey, const float* ez,
                const uint8_t* label, int nx, int ny, int nz, int nrhs, void* stream);
int fs_pcg_plan_level_data(const fs_pcg_plan* plan, int level, const void** em,
                           const uint8_t** label, const void** scale);
int fs_pcg_plan_unet_workspace_bytes(const fs_pcg_plan* plan, int level, size_t* bytes);
int fs_pcg_plan_set_unet(fs_pcg_plan* plan, int level, int mode, float* theta, void* workspace,
                         size_t workspace_bytes, void* stream);
/* Re-pack the plan's network weights after theta changed.                  */
int fs_pcg_plan_sync_unet(fs_pcg_plan* plan, void* stream);


/* Failure-detection self test: one device thread waits, with a budget of
 * budget_cycles SM clocks, on an mbarrier nothing completes -- the path
 * every staged-load wait of the library takes on a timeout.  *status_host
 * receives FS_TIMEOUT when the bounded wait gave up (and the context stays
 * usable).                                                                   */
int fs_selftest_wait_timeout(long long budget_cycles, int* status_host, void* stream);


/* min, max and the number of non-finite entries of an FP64 device array
 * (stats_host[3], host); the eager input checks of a cell property.
 * workspace: FS_PROP_STATS_WORKSPACE_BYTES of device memory, 16-byte
 * aligned, free for the call (it returns after its stream is synchronised).  */
#define FS_PROP_STATS_WORKSPACE_BYTES 16384
int fs_prop_stats(const double* p, long long n, double* stats_host, void* workspace,
                  size_t workspace_bytes, void* stream);

/* The same reduction, only enqueued on `stream` (no copy, no synchronisation):
 * min, max and the non-finite count land as three doubles at byte offset
 * FS_PROP_STATS_RESULT_OFFSET of the workspace, which must stay allocated
 * until the caller has read them (stream-ordered).  Lets a host overlap the
 * upload and check of a cell property with other work.                      */
#define FS_PROP_STATS_RESULT_OFFSET 14208
int fs_prop_stats_enqueue(const double* p, long long n, void* workspace,
                          size_t workspace_bytes, void* stream);

/* ---- §8f: field region (fieldspice/circuit/coupling.py) ----------------------
 * out[i] = base[i] + sum_{c<ncols} coef_host[c] * phi[i*k + c0 + c] for
 * i < n (FP64; base may be NULL for 0; ncols <= 16, c0 + ncols <= k): the
 * interior back-substitution of FieldRegion.accept_timestep
 * (coupling.py:248-262) as a superposition of the cached unit-excitation
 * solutions (columns of K_ii^-1 K_it) on the history solution.              */
int fs_rhs_superpose(const double* phi, int k, int c0, int ncols,
                     const double* coef_host, const double* base, double* out,
                     long long n, void* stream);

/* ---- a plan's preconditioner on a caller's vectors ---------------------------
 * z = M r for the plan's equilibrated system: one multigrid V-cycle (identity
 * for a Jacobi plan) on N*nrhs values in the plan's precision.  The plan must
 * not carry a learned level.  fs_pcg_plan_scale exposes the plan's FP64
 * scaling s = diag^-1/2 (0 on non-free nodes) and its classified labels
 * (FS_LABEL_*: free, fixed, solo, pinned).                                   */
int fs_pcg_plan_precondition(fs_pcg_plan* plan, const void* r, void* z, void* stream);
int fs_pcg_plan_scale(const fs_pcg_plan* plan, const double** s64, const uint8_t** label);
/* counts[4] (host): the plan's free, fixed, solo and pinned node counts, as
 * classified at creation (LinearSystem's split, poisson.py:282-362).       */
int fs_pcg_plan_label_counts(const fs_pcg_plan* plan, long long* counts, void* stream);
/* The CG stencil kernel the plan runs: 0 cached loads, 1 TMA-staged p,
 * 2 TMA-staged p and masses, 3 as 2 with TMA stores of q, 4 as 2 with each
 * 32-byte node split over two threads, 5 as 2 with the direction update
 * p = z + beta p_old formed inside the stencil from staged z and p_old tiles
 * (no separate p-update kernel) on 32x8 tiles, 6 and 7 as 5 on 32x4 and
 * 32x16 tiles (nodes of at most 32 bytes).  Unless the plan's options or the
 * FS_STENCIL environment variable name one, the first plan of each shape
 * class (RHS block, element size, log2 of the node count, nz a multiple of
 * 32) with vectors of at least 32 MB times kinds 2, 3, 0, 5, 6, 7 (and 4 for
 * 32-byte nodes), each with the direction update it needs, on its own
 * buffers at creation, and later plans of that class reuse the fastest.     */
int fs_pcg_plan_stencil_kind(const fs_pcg_plan* plan);
/* ms[8] (host): the mean time per iteration of the direction update and the
 * stencil for each kind (index = kind) measured by this plan's autotuner;
 * -1 for kinds it did not time (every entry is -1 when the plan reused an
 * earlier choice or FS_STENCIL chose).                                      */
int fs_pcg_plan_stencil_times(const fs_pcg_plan* plan, float* ms);

/* ---- §8f-4: harmonic EQS, the complex-symmetric solve -------------------------
 * Replaces the per-frequency sparse LU of fieldspice/solvers/ac.py:95-145
 * (ACSolver.solve / admittance_matrix): K phi = 0 with K = A + jB, A and B
 * node-padded edge masses (3N FP64 each, x | y | z like fs_build_masses'
 * output: A = sigma - w eps'' masses, B = w eps' masses), phi fixed on the
 * nodes labelled FIXED.  phi: N x K FP64, K = the power of two >= 2*ncplx,
 * column c < K/2 the real and K/2 + c the imaginary part of right-hand side
 * c (ncplx <= 8); Dirichlet values in, solution out.  COCG on the system
 * equilibrated by diag(|A| + |B|)^-1/2, preconditioned by the multigrid
 * V-cycle (precond = FS_PRECOND_MG) of |A| + |B| or by nothing
 * (FS_PRECOND_JACOBI); stopping rule ||S r|| <= tol ||S b|| on the true FP64
 * residual.  stats: ncplx entries.                                          */
int fs_ac_workspace_bytes(int nx, int ny, int nz, int ncplx, int precond, size_t* bytes);
int fs_ac_solve(int nx, int ny, int nz, int ncplx, int precond, const double* mA,
                const double* mB, const uint8_t* label_in, double* phi, double tol,
                int maxiter, void* workspace, size_t workspace_bytes, fs_rhs_stats* stats,
                void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FIELDSPICE_B200_H */
