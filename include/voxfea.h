/*
 * voxfea.h -- C-ABI of libvoxfea.so, the B200 (sm_100a) matrix-free voxel
 * elasticity solve: hex8 element-by-element K*u inside PCG preconditioned by a
 * geometric-multigrid V-cycle.
 *
 * This is the boundary the Python solver layer binds with ctypes
 * (voxelsim_fea_b200/_lib.py).  Each entry point names the reference
 * interface it replaces (VoxelSim-FEA, paths relative to that project).
 *
 * Conventions (identical to the reference, so host arrays pass through):
 *   - grid of nx*ny*nz hex8 voxels of unit edge (stiffness scales with the
 *     modulus the caller passes, E*vsize -- core/solve_worker.py:342-354);
 *   - node id  ix + (nx+1)*(iy + (ny+1)*iz)       (core/fea.py:129-130);
 *   - DOF id   3*node + c, c = x,y,z              (core/fea.py:17);
 *   - element order iz fastest: e = (ix*ny + iy)*nz + iz (core/fea.py:133-148).
 * All host arrays are caller-owned and only read/written during the call.
 * Every function returns an int status (VF_OK == 0); nothing aborts the
 * process.  vf_last_error() gives a message for the last failure on a handle,
 * vf_global_last_error() for failures before a handle exists.
 */
#ifndef VOXFEA_H
#define VOXFEA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VF_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
  VF_OK = 0,
  VF_ERR_ARG = 1,           /* invalid argument                      -> ValueError */
  VF_ERR_STATE = 2,         /* wrong call order ("call set_fixed() before solve()",
                               core/fea.py:427-428)                  -> RuntimeError */
  VF_ERR_CUDA = 3,          /* CUDA runtime failure                  -> RuntimeError */
  VF_ERR_NOMEM = 4,         /* device allocation failed              -> MemoryError */
  VF_ERR_NO_DEVICE = 5,     /* no usable sm_100 device               -> RuntimeError */
  VF_ERR_STALLED = 6,       /* MG-PCG stall/divergence guard fired
                               (core/multigrid.py:523-531)           -> RuntimeError */
  VF_ERR_NONFINITE = 7,     /* NaN/Inf in an input or an iterate     -> FloatingPointError */
  VF_ERR_UNSUPPORTED = 8,   /* option combination not implemented   -> NotImplementedError */
  VF_ERR_BREAKDOWN = 9      /* Krylov breakdown / singular coarse factor */
};

/* ---- options ------------------------------------------------------------ */
enum { VF_PREC_FP64 = 0,    /* every vector, operator and transfer in FP64 */
       VF_PREC_MIXED = 1,   /* FP32 PCG + V-cycle inside an FP64 iterative-
                               refinement loop (FP64 dots, outer residual,
                               coarsest solve) */
       VF_PREC_FP32 = 2 };  /* FP32 vectors/operators, FP64 dots (no refinement) */

enum { VF_METHOD_MG = 0,        /* GMG-preconditioned CG on the full grid
                                   (core/multigrid.py MGSolver.solve) */
       VF_METHOD_JACOBI = 1 };  /* Jacobi-PCG on the active elements only
                                   (core/fea.py VoxelFEA._solve_jacobi) */

enum { VF_COARSE_REDISCRETIZE = 0,  /* reference: coarse E = 2x2x2 mean, x 2^level,
                                       injected Dirichlet mask
                                       (core/multigrid.py:255-315) */
       VF_COARSE_GALERKIN = 1 };    /* R A P with the masked trilinear P; robust
                                       under void/solid contrast */

enum { VF_COARSEST_JACOBI = 0,      /* reference: 30 damped-Jacobi sweeps
                                       (core/multigrid.py:428-429) */
       VF_COARSEST_CHOLESKY = 1 };  /* FP64 dense Cholesky direct solve */

typedef struct vf_options {
  int32_t struct_size;     /* sizeof(vf_options), set by vf_options_default */
  int32_t method;          /* VF_METHOD_*                                   */
  int32_t precision;       /* VF_PREC_*                                     */
  int32_t n_smooth;        /* pre/post sweeps (multigrid.py:86, default 2)  */
  int32_t min_elems;       /* hierarchy guard (multigrid.py:86, default 4)  */
  int32_t max_levels;      /* (multigrid.py:86, default 6)                  */
  int32_t coarse_op;       /* VF_COARSE_*                                   */
  int32_t coarsest;        /* VF_COARSEST_*                                 */
  int32_t coarse_sweeps;   /* sweeps of the Jacobi coarsest solve (30)      */
  int32_t stall_guard;     /* 1: raise VF_ERR_STALLED like multigrid.py:523 */
  int32_t check_every;     /* PCG iterations per device graph launch        */
  int32_t use_graphs;      /* capture iteration chunks as CUDA graphs       */
  int32_t device;          /* CUDA device ordinal                           */
  int32_t max_outer;       /* VF_PREC_MIXED: refinement steps cap           */
  double  omega;           /* Jacobi damping (multigrid.py:86, default 0.6) */
  double  inner_tol;       /* VF_PREC_MIXED: residual reduction between FP64 corrections
                              (1e-2; the FP32 recurrence residual runs ahead of the
                              true one by up to 100x below ~1e-4 of its start)   */
  int32_t omega_mode;      /* VF_OMEGA_FIXED: omega on every level (reference);
                              VF_OMEGA_AUTO: omega_l = omega_rel * 2 / lambda_l with
                              lambda_l a power-iteration estimate of
                              lambda_max(D^-1 A_l) taken at set_material */
  int32_t power_iters;     /* VF_OMEGA_AUTO: power iterations per level (20) */
  double  omega_rel;       /* VF_OMEGA_AUTO: fraction of the stability limit (0.8) */
  int32_t fine_kernel;     /* VF_FINE_MODAL (default) | VF_FINE_GATHER: kernel of the
                              element-operator levels (same operator, different form) */
  int32_t modal_zchunk;    /* z-planes per CTA of the modal kernel; 0 = automatic;
                              -1 = one resident wave of CTAs sharing the (tile, plane)
                              units evenly (TMA form) */
  int32_t coarse_storage;  /* Galerkin stencils as applied in the V-cycle:
                              VF_STENCIL_SYM_HALF (default): symmetric, diagonally
                              scaled, FP16 values for the FP32 V-cycle and FP64 for FP64;
                              VF_STENCIL_SYM: symmetric scaled FP32 / FP64;
                              VF_STENCIL_FULL: all 27 blocks, unscaled */
  int32_t mixed_mode;      /* VF_PREC_MIXED: VF_MIXED_RELIABLE: one FP32 CG whose
                              residual is replaced by the FP64 true residual (and the FP32
                              increment folded into the FP64 solution) each time it has
                              dropped by inner_tol; VF_MIXED_RESTART: iterative refinement,
                              a fresh FP32 PCG per outer step; VF_MIXED_OUTER64 (default): FP64 PCG
                              (x, r, p, A p, dots and the fine operator of A p in FP64)
                              preconditioned by the FP32 V-cycle -- the FP64 Krylov space,
                              so the iteration count of the FP64 solve on hard problems */
  int32_t flexible;        /* 1: flexible CG (Notay's FCG(1): beta = -z.Ap / p.Ap), which
                              stays correct for a preconditioner that varies between
                              iterations; always on while a learned stage is enabled */
  int32_t autotune;        /* 1 (default): at the first vf_set_material, time candidate
                              z-chunk sizes of the marching kernels on every level and keep
                              the fastest (cached per grid shape for the process) */
  int32_t smoother;        /* VF_SMOOTH_JACOBI (default): damped Jacobi sweeps;
                              VF_SMOOTH_CHEBYSHEV: Chebyshev polynomial smoothing of the same
                              degree (n_smooth <= 2 sweeps) on [lambda / cheb_ratio, lambda],
                              lambda the VF_OMEGA_AUTO estimate of lambda_max(D^-1 A_l); needs
                              VF_OMEGA_AUTO, a modal fine kernel and symmetric coarse storage */
  int32_t cheb_ratio;      /* VF_SMOOTH_CHEBYSHEV: lambda_max / lower end of the interval (30) */
  int32_t smoothed_transfers; /* bit l set: the transfer from Galerkin level l to l+1 uses the
                              smoothed prolongation P_s = D (I - (4/3) D^-1 A_l / lambda_l) P
                              (P the reference's trilinear P, multigrid.py:42-73; lambda_l the
                              VF_OMEGA_AUTO estimate), and A_{l+1} = P_s^T A_l P_s couples nodes
                              two coarse spacings apart (125 blocks).  Bit 1 only (level 1 -> 2):
                              needs VF_COARSE_GALERKIN, VF_OMEGA_AUTO and symmetric storage; 0 =
                              trilinear everywhere (default) */
  int32_t learned_watch;   /* learned stage on (vf_learned_configure): when the residual has not
                              halved over this many iterations, the stage is switched off and the
                              solve continues as plain PCG from its current iterate, within the
                              same iteration budget (vf_solve_info.outer_iters = the iteration of
                              the switch); 0 = never (default 64) */
  int32_t smoothed_level_sweeps; /* sweeps before and after the coarse correction on a level whose
                              transfer to the next level is smoothed (its smoothed restriction and
                              prolongation already smooth it once each); 0 = n_smooth (default) */
} vf_options;

enum { VF_OMEGA_FIXED = 0, VF_OMEGA_AUTO = 1 };
enum { VF_FINE_MODAL = 0,     /* modal z-marching kernel, TMA-staged (vf_modal_tma.cu) */
       VF_FINE_GATHER = 1,    /* node-centric 27-neighbour gather (vf_matvec.cu) */
       VF_FINE_MODAL_CPASYNC = 2 };  /* modal z-marching kernel, cp.async-staged (vf_modal.cu) */
enum { VF_STENCIL_SYM_HALF = 0, VF_STENCIL_SYM = 1, VF_STENCIL_FULL = 2 };
enum { VF_MIXED_RELIABLE = 0, VF_MIXED_RESTART = 1, VF_MIXED_OUTER64 = 2 };
enum { VF_SMOOTH_JACOBI = 0, VF_SMOOTH_CHEBYSHEV = 1 };

typedef struct vf_solve_info {
  int32_t iters;           /* PCG iterations (all inner iterations for MIXED);
                              MGSolver.last_iters (multigrid.py:515)        */
  int32_t outer_iters;     /* MIXED: residual replacements (RELIABLE) or
                              refinement steps (RESTART); with a learned stage
                              (FP64 or OUTER64): the iteration after which it
                              was switched off for stagnating (0: stayed on) */
  int32_t converged;       /* MGSolver.last_converged                       */
  int32_t status;          /* VF_OK, VF_ERR_STALLED, VF_ERR_BREAKDOWN, ...   */
  double  resid_ratio;     /* MGSolver.last_resid_ratio (recurrence, or the
                              FP64 true residual for MIXED)                 */
  double  true_resid;      /* ||mask(f - K u)|| / ||mask f|| in FP64 at exit */
  double  device_ms;       /* solve time on the solver's stream (events)    */
  double  setup_ms;        /* of which: density / coarse-operator set-up    */
} vf_solve_info;

typedef struct vf_solver vf_solver;

/* ---- library / device --------------------------------------------------- */
int         vf_abi_version(void);
const char* vf_status_string(int status);
const char* vf_global_last_error(void);
/* backend.gpu_device_count (core/backend_gpu.py:110-122) */
int         vf_device_count(int32_t* count);
/* backend._self_test (core/backend_gpu.py:40-60): runs the hex8 operator on a
 * small grid on the device and compares with a host evaluation.  VF_OK if
 * the device result agrees to 1e-12 (FP64) and 1e-5 (FP32). */
int         vf_self_test(int32_t device);

/* _hex8_KE / _hex8_B_C (core/fea.py:31-122): KE(E=1, nu) (576), the
 * nu-independent split KE = lam*K_lam + mu*K_mu (576 each) and the centroid
 * B0 (6x24).  Host-only; any output pointer may be NULL. */
int         vf_hex8_tables(double nu, double* KE, double* K_lam, double* K_mu, double* B0);

/* ---- solver lifetime ------------------------------------------------------ */
void        vf_options_default(vf_options* opts);
/* MGSolver.__init__ (core/multigrid.py:85-174) / VoxelFEA.__init__
 * (core/fea.py:244-305): builds the level hierarchy (multigrid.py:141-148)
 * and the Ke tables.  nu is the Poisson ratio used when vf_set_material gets
 * no per-voxel ratio. */
int         vf_create(int32_t nx, int32_t ny, int32_t nz, double nu,
                      const vf_options* opts, vf_solver** out);
/* MGSolver.close (core/multigrid.py:245-252) / VoxelFEA.close (fea.py:342-355) */
int         vf_destroy(vf_solver* s);
const char* vf_last_error(const vf_solver* s);
int         vf_num_levels(const vf_solver* s, int32_t* n);
int         vf_level_dims(const vf_solver* s, int32_t level, int32_t* dims3);
/* Damping used on a level and, with VF_OMEGA_AUTO, the lambda_max(D^-1 A)
 * estimate behind it (valid after vf_set_material). */
int         vf_level_omega(const vf_solver* s, int32_t level, double* omega, double* lambda);

/* ---- problem definition --------------------------------------------------- */
/* MGSolver._build_free (multigrid.py:255-278) / VoxelFEA.set_fixed
 * (fea.py:357-369): original (full-grid) DOF ids, any order, duplicates ok. */
int vf_set_fixed(vf_solver* s, const int64_t* fixed_dofs, int64_t n);
/* VoxelFEA active_elems (fea.py:266-279): uint8 per element (NULL = all).
 * Used by VF_METHOD_JACOBI to restrict the system to the active elements'
 * DOFs; the MG method takes e_min voids through the modulus instead. */
int vf_set_active(vf_solver* s, const uint8_t* active);
/* MGSolver.set_density (multigrid.py:281-315): per-element modulus (nelem,
 * float64, iz-fastest); nu_elem (nelem) is an optional per-voxel Poisson
 * ratio (NULL = the ratio given to vf_create).  Builds every level's operator,
 * diagonal and, for VF_COARSEST_CHOLESKY, the coarsest factor.  flags may be
 * VF_SOLVE_DEVICE_PTRS (E, nu_elem already in device memory). */
int vf_set_material(vf_solver* s, const double* E, const double* nu_elem, uint32_t flags);

/* ---- solve ---------------------------------------------------------------- */
#define VF_SOLVE_DEVICE_PTRS 1u   /* array arguments are device pointers      */

/* MGSolver.solve (multigrid.py:439-583) / VoxelFEA._solve_jacobi
 * (fea.py:497-593): f and u_out are full-grid float64 (3*(nx+1)(ny+1)(nz+1));
 * x0 may be NULL.  max_it <= 0 selects the reference default (1000 for MG,
 * 4*n_free for Jacobi).  Returns VF_ERR_STALLED when the stall guard fires
 * (u_out then holds the last iterate). */
int vf_solve(vf_solver* s, const double* f, const double* x0, double tol,
             int32_t max_it, uint32_t flags, double* u_out, vf_solve_info* info);
/* Same as vf_solve, invoking progress(it, resid_ratio, tol, user) once per
 * completed iteration, in order, from the calling thread -- the reference's
 * progress_cb(it, resid, tol) contract (multigrid.py:518-519).  Iterations run
 * on the device in chunks of vf_options.check_every, so callbacks arrive in
 * bursts at chunk boundaries.  With a zero (masked) load the solve returns
 * u = 0 immediately and info->iters = -1 (multigrid.py:471-473). */
typedef void (*vf_progress_fn)(int32_t it, double resid_ratio, double tol, void* user);
int vf_solve_cb(vf_solver* s, const double* f, const double* x0, double tol,
                int32_t max_it, uint32_t flags, double* u_out, vf_solve_info* info,
                vf_progress_fn progress, void* user);
/* MGSolver.resid_history (multigrid.py:452, 517): copies up to cap entries. */
int vf_resid_history(const vf_solver* s, double* out, int32_t cap, int32_t* n_out);

/* ---- post-processing ------------------------------------------------------ */
/* VoxelFEA.element_von_mises_stress (fea.py:604-626): centroid stress of every
 * element with active[e] != 0 (active NULL = all), zeros elsewhere.  E_stress
 * is per element (nelem); nu_elem optional per-voxel ratio. */
int vf_von_mises(vf_solver* s, const double* u, const double* E_stress,
                 const double* nu_elem, const uint8_t* active, double* vm_out);
/* VoxelFEA.element_strain_energy (fea.py:595-602): u_e^T KE u_e, KE at E = 1. */
int vf_strain_energy(vf_solver* s, const double* u, const uint8_t* active,
                     double* se_out);
/* fea.drop_unsupported_islands (fea.py:207-227): 6-connected flood fill of the
 * active elements from those touching a fixed node (device kernels).
 * kept_out may alias active.  *n_removed = active - kept (0 and kept = active
 * when no active element touches a fixed node). */
int vf_drop_unsupported_islands(int32_t nx, int32_t ny, int32_t nz,
                                const uint8_t* active, const int64_t* fixed_dofs,
                                int64_t n_fixed, uint8_t* kept_out,
                                int64_t* n_removed);

/* ---- level operators (parity tests and tools) ------------------------------
 * Host float64 arrays in the reference layout of that level.  precision is
 * VF_PREC_FP64 or VF_PREC_FP32 (the kernel variant that runs).              */
/* MGSolver._apply (multigrid.py:318-341): y = mask(K_l u) */
int vf_apply(vf_solver* s, int32_t level, int32_t precision, const double* u, double* y);
/* MGSolver._smooth (multigrid.py:367-402): `sweeps` damped-Jacobi sweeps */
int vf_smooth(vf_solver* s, int32_t level, int32_t precision, const double* u0,
              const double* b, int32_t sweeps, double* out);
/* MGSolver._restrict (multigrid.py:404-416): fine level -> level+1 */
int vf_restrict(vf_solver* s, int32_t level, int32_t precision, const double* r_fine,
                double* r_coarse);
/* MGSolver._prolongate (multigrid.py:418-424): level+1 -> fine level */
int vf_prolongate(vf_solver* s, int32_t level, int32_t precision, const double* e_coarse,
                  double* e_fine);
/* MGSolver._vcycle(0, r) (multigrid.py:426-436) */
int vf_vcycle(vf_solver* s, int32_t precision, const double* r, double* z);
/* MGSolver levels[l]['Minv'] (multigrid.py:300-304): 3 values per node */
int vf_inv_diagonal(vf_solver* s, int32_t level, double* minv);

/* ---- measurement ------------------------------------------------------------
 * The solver's CUDA stream (cudaStream_t), for event timing by the caller. */
int vf_get_stream(const vf_solver* s, void** stream);
/* Kernels launched by this library since load (graph replays count every
 * kernel node they contain). */
int vf_launch_count(uint64_t* count);

/* Times `iters` back-to-back launches of one kernel on the solver's stream with
 * CUDA events (operands already resident; set_material must have run).
 * kernel: 0 = fine operator y = K p (+ p.y), 1 = fused Jacobi sweep,
 *         2 = residual, 3 = restriction, 4 = prolongation+add, 5 = V-cycle.
 * *ms_per_launch receives the mean duration. */
int vf_time_kernel(vf_solver* s, int32_t kernel, int32_t precision, int32_t iters,
                   double* ms_per_launch);

/* ---- no-allocation operator ---------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- programs that own all device memory through their own allocator or
 * a fixed arena, and code that must avoid the implicit device synchronisation of
 * cudaMalloc/cudaFree.  Computes y = mask(K u) -- the level-0 operator of
 * vf_apply, the fine hex8 operator with Ke(nu) -- and *u_dot_y = u . y on
 * `stream` (cudaStream_t, NULL = default stream), without a solver handle and
 * without allocating: its only scratch is a fixed static device array of
 * 256 KiB + 256 B, shared by every call on a device.
 * All pointers are device pointers in the reference layout: E (nelem, iz-fastest),
 * free_mask (one byte per node, bit c set <=> DOF c free), u and y (3 per node),
 * u_dot_y (one double).  u, y and u_dot_y must not overlap (an overlapping y or
 * u_dot_y returns VF_ERR_ARG).  Limits: (nx+1)(ny+1)(nz+1) <= 8,388,608 nodes,
 * else VF_ERR_ARG.  The first call on each device looks up the scratch address
 * and keeps it; make it before any stream capture, and make no call on a device
 * after cudaDeviceReset there.  Calls that overlap on the GPU race on the shared
 * scratch: order them on one stream.  Asynchronous: returns after enqueueing. */
int vf_apply_noalloc(int32_t nx, int32_t ny, int32_t nz, double nu, const double* E,
                     const uint8_t* free_mask, const double* u, double* y, double* u_dot_y,
                     void* stream);

/* ---- block right-hand sides ----------------------------------------------------
 * k load cases on one geometry (the reference solves them one call at a time:
 * MGSolver.solve, core/multigrid.py:439-583, once per case).  F and U hold k
 * vectors of 3*(nx+1)*(ny+1)*(nz+1) values back to back (host, or device with
 * VF_SOLVE_DEVICE_PTRS); infos receives k records.  The k solves share this
 * solver's operator data (set up once by vf_set_material) and run concurrently,
 * each on its own stream with its own vectors, Krylov state and CUDA graphs
 * (created on first use and kept for later calls).  Not with the learned stage
 * enabled (VF_ERR_UNSUPPORTED). */
int vf_solve_block(vf_solver* s, const double* F, int32_t k, double tol, int32_t max_it,
                   uint32_t flags, double* U, vf_solve_info* infos);

/* Many independent parts (each its own solver: own grid, geometry, stream) set
 * up and solved concurrently in one call -- the reference solves one part per
 * job.  For part i: E[i] / nu_elem[i] (optional, as vf_set_material; E == NULL
 * or E[i] == NULL keeps the material already set), F[i] -> U[i] (host, or
 * device with VF_SOLVE_DEVICE_PTRS), infos[i].  Returns the first failing
 * part's status (vf_global_last_error names it). */
int vf_solve_batch(vf_solver* const* solvers, int32_t n, const double* const* E,
                   const double* const* nu_elem, const double* const* F, double tol,
                   int32_t max_it, uint32_t flags, double* const* U, vf_solve_info* infos);

/* ---- grid assembly of a solve job (core/solve_worker.py:242-287) --------------
 * Role masks -> active voxels (uint8 per element, iz-fastest), fixed-DOF bits
 * (uint8 per node: bit c set <=> DOF c fixed) and the nodal force vector
 * (3 per node, N), on the device.  roles[i] / masks[i] / meta[3i..3i+2]:
 *   VF_ROLE_BUILD    per-element mask; the last one is the active set
 *   VF_ROLE_EXCLUDE  per-element mask removed from it
 *   VF_ROLE_BEARING  per-node mask; meta = axes (0/1) whose DOFs are fixed
 *   VF_ROLE_LOAD     per-node mask; meta = force spread evenly over its nodes,
 *                    added role by role in order (the reference's sums)
 * flags VF_SOLVE_DEVICE_PTRS: masks and outputs are device pointers.
 * *n_active_out / *n_fixed_out (optional): active voxels, fixed DOFs. */
enum { VF_ROLE_BUILD = 0, VF_ROLE_EXCLUDE = 1, VF_ROLE_BEARING = 2, VF_ROLE_LOAD = 3 };
int vf_assemble_grid(int32_t nx, int32_t ny, int32_t nz, int32_t n_roles, const int32_t* roles,
                     const uint8_t* const* masks, const double* meta, uint32_t flags, uint8_t* active_out,
                     uint8_t* fixed_bits_out, double* force_out, int64_t* n_active_out, int64_t* n_fixed_out);
/* fea.drop_unsupported_islands (fea.py:207-227) with the supports given as the
 * per-node fixed-DOF bits of vf_assemble_grid (flags as there). */
int vf_drop_unsupported_islands_mask(int32_t nx, int32_t ny, int32_t nz, const uint8_t* active,
                                     const uint8_t* fixed_bits, uint32_t flags, uint8_t* kept_out,
                                     int64_t* n_removed);
/* VoxelFEA.set_fixed (fea.py:357-369) from per-node fixed-DOF bits (bit c set
 * <=> DOF c fixed; host, or device with VF_SOLVE_DEVICE_PTRS) instead of a DOF
 * list. */
int vf_set_fixed_mask(vf_solver* s, const uint8_t* fixed_bits, uint32_t flags);

/* Per-element displacement field of the result views (core/solve_worker.py:374-388):
 * disp_out[e] = mean over the 8 corners of |u_node| (FP32, element order
 * iz-fastest); u: 3 values per node, reference node order (host arrays). */
int vf_element_displacement(int32_t nx, int32_t ny, int32_t nz, const double* u, float* disp_out);

/* ---- voxelization: point-in-mesh inside test ------------------------------------
 * The reference's parity ray cast (core/inside_worker.py:_inside_mask_numpy,
 * lines 105-147) on the device with its FP64 arithmetic in its evaluation order:
 * the masks are the reference's bit for bit.  verts (nv x 3), faces (nf x 3,
 * indices checked), dir3 = the ray direction (the reference's default is
 * (1, 0.0073301, 0.0031337) normalised).  Host arrays; out: one byte per point. */
int vf_inside_points(const double* verts, int64_t nv, const int64_t* faces, int64_t nf,
                     const double* points, int64_t npts, const double* dir3, uint8_t* out);
/* The same for the voxel centers (target 0, element order iz-fastest) or the
 * grid nodes (target 1, node order x-fastest) of a dims3 grid at origin3 with
 * voxel size vsize (inside_worker.py:voxel_centers / node_coords), the points
 * generated on the device. */
int vf_inside_grid(const double* verts, int64_t nv, const int64_t* faces, int64_t nf,
                   const int32_t* dims3, const double* origin3, double vsize, int32_t target,
                   const double* dir3, uint8_t* out);

/* ---- learned preconditioner stage: BF16 tensor-core 3x3x3 convolutions --------
 * No counterpart in the reference (its solver has no learned part).  Building
 * blocks of the U-Net trained by voxelsim_fea_b200.learned and run inside the
 * flexible-CG preconditioner.  All pointers are device pointers; tensors are
 * channels-last BF16 boxes [Z][Y][X][C], zero-padded ("same" convolution);
 * weights [27][cout][cin] BF16 with tap = (dz+1)*9 + (dy+1)*3 + (dx+1)
 * (cross-correlation, the torch conv3d convention).  FP32 accumulation on the
 * tensor cores.  (cin, cout) in {(16,16) (16,32) (32,16) (32,32) (32,64)
 * (64,32) (64,64)}; other pairs return VF_ERR_ARG.  `stream`: cudaStream_t. */
/* out = relu?(conv(in, w) + bias + skip); bias (FP32, cout), skip (BF16, cout
 * channels) optional; out_f32 non-NULL writes FP32 instead of BF16 `out`. */
int vf_nn_conv3d_forward(const void* in, const void* w, const float* bias, const void* skip,
                         int32_t relu, void* out, float* out_f32, int32_t X, int32_t Y, int32_t Z,
                         int32_t cin, int32_t cout, void* stream);
/* dx = conv^T(dy) * (gate > 0 if gate): the data gradient of a layer with cin
 * inputs and cout outputs; w_t [27][cin][cout] is w with its taps mirrored and
 * its channel axes swapped; gate (BF16, cin channels) is the layer input saved
 * in the forward pass when that input came out of a ReLU. */
int vf_nn_conv3d_backward_data(const void* dy, const void* w_t, const void* gate, void* dx,
                               int32_t X, int32_t Y, int32_t Z, int32_t cin, int32_t cout,
                               void* stream);
/* dw[27][cout][cin] (FP32) (+)= sum_v dy[v][co] x[v + off(tap)][ci]; work is a
 * caller-provided scratch of vf_nn_wgrad_workspace() bytes (deterministic
 * per-CTA partial sums, reduced in a fixed order). */
int vf_nn_conv3d_backward_weight(const void* x, const void* dy, float* dw, int32_t accumulate,
                                 float* work, size_t work_bytes, int32_t X, int32_t Y, int32_t Z,
                                 int32_t cin, int32_t cout, void* stream);
size_t vf_nn_wgrad_workspace(int32_t cin, int32_t cout, int32_t X, int32_t Y, int32_t Z);

/* The learned stage inside the solver's preconditioner: after the V-cycle,
 *   z += P^L NN(R^L (r - A z))
 * with NN the 3-level U-Net (10 convolutions, see vf_learned.cu) run on the
 * node grid of hierarchy level L (>= 1) padded to multiples of 4; its input is
 * the restricted residual scaled by its RMS, the occupancy and the normalised
 * log-modulus of the voxels around each node; its output (x RMS / Eref, Eref
 * the largest voxel modulus) is the level-L correction.  Enabling it switches
 * the iteration to flexible CG.  Parameters: per layer W[27][cout][cin] then
 * b[cout], FP32, vf_learned_param_count() values. */
int64_t vf_learned_param_count(void);
/* Create the stage on `level` (re-created if the level changes), upload
 * `params` when non-NULL, and enable (enable = 1) or disable it. */
int vf_learned_configure(vf_solver* s, int32_t level, const float* params, int64_t n_params,
                         int32_t enable);
/* dims3: the U-Net grid (X, Y, Z); level: the hierarchy level it runs on. */
int vf_learned_info(const vf_solver* s, int32_t* dims3, int32_t* level);
/* The U-Net input for a level-L residual given on the host in the reference
 * node layout of level L: written to in_dev (device, BF16 [Z][Y][X][16]);
 * *scale_out = the residual RMS, *eref_out = Eref.  For training. */
int vf_learned_input(vf_solver* s, const double* r_level, void* in_dev, float* scale_out,
                     double* eref_out);
/* The whole stage on host arrays: e_fine = P^L NN(R^L r_fine) (FP64 transfers,
 * the inference kernels of the solver).  For tests. */
int vf_learned_apply(vf_solver* s, const double* r_fine, double* e_fine);
/* e_out = (I - M A)^n e_in: n stationary iterations of the FP32 V-cycle M of
 * the mixed solver on an error vector (host arrays, reference layout); the
 * training data of the learned stage. */
int vf_mg_propagate(vf_solver* s, const double* e_in, int32_t n, double* e_out);
/* Free-DOF bits of hierarchy level `level` (one byte per node, reference node
 * order of that level). */
int vf_level_mask(vf_solver* s, int32_t level, uint8_t* out);

#ifdef __cplusplus
}
#endif
#endif /* VOXFEA_H */
