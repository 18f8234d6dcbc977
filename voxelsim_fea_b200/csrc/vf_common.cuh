// Shared definitions of libvoxfea: padded grid layout, status plumbing and
// the host-side launcher declarations of every kernel.
//
// HBM layout of one multigrid level (lx*ly*lz voxels):
//   nodes are stored on a padded box with ONE ghost shell on every side,
//   node (x, y, z), x in [-1, lx+1], at  ((z+1)*py + (y+1))*px + (x+1)
//   px = round_up(lx+3, 4) (16-byte aligned rows for float3/double3 AoS),
//   py = ly+3, pz = lz+3.  Ghost and pad nodes hold zeros in every vector and
//   a zero free-mask, so stencils need no bounds checks.
//   Element (ex, ey, ez), ex in [-1, lx], is stored at the slot of its lower
//   corner node; ghost elements have modulus 0.
//   Vectors are AoS: v[3*p + c] (the reference's 3n+c DOF order).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <type_traits>
#include <utility>

namespace vf {

// Every kernel of the library is launched through launch_k so launches can be
// counted (vf_launch_count): launches recorded into a CUDA graph during
// capture are counted when the graph is replayed instead.
void count_launch(cudaStream_t st);
unsigned long long direct_launches();

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args&&... args) {
  count_launch(st);
  kern<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
}

// One-time set-up of a kernel that takes more than 48 KiB of dynamic shared
// memory.  The runtime applies cudaFuncSetAttribute per device, and a process
// may drive solvers on several devices, so the attribute is set -- and the
// resident CTAs per SM measured -- the first time each device launches the
// kernel; `cache` holds one slot per device ordinal.  Returns CTAs per SM (>= 1).
constexpr int kMaxDevices = 64;
template <typename Kern>
inline int kernel_prepare(std::atomic<int> (&cache)[kMaxDevices], Kern kern, size_t smem, int threads) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  std::atomic<int>* slot = (dev >= 0 && dev < kMaxDevices) ? &cache[dev] : nullptr;
  const int have = slot ? slot->load() : 0;
  if (have > 0) return have;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int o = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, threads, smem) != cudaSuccess || o < 1) o = 1;
  if (slot) slot->store(o);
  return o;
}

struct Grid {
  int lx, ly, lz;   // voxels
  int px, py, pz;   // padded node box
  int n;            // px*py*pz (checked < 2^29 at creation)
  __host__ __device__ __forceinline__ int idx(int x, int y, int z) const {
    return ((z + 1) * py + (y + 1)) * px + (x + 1);
  }
  __host__ __device__ __forceinline__ int nodes_ref() const {
    return (lx + 1) * (ly + 1) * (lz + 1);
  }
  __host__ __device__ __forceinline__ int elems_ref() const { return lx * ly * lz; }
};

inline Grid make_grid(int lx, int ly, int lz) {
  Grid g;
  g.lx = lx; g.ly = ly; g.lz = lz;
  g.px = ((lx + 3 + 3) / 4) * 4;
  g.py = ly + 3;
  g.pz = lz + 3;
  g.n = g.px * g.py * g.pz;
  return g;
}

// Free-mask bits per node: bit c set <=> DOF c is free.
constexpr uint8_t kFreeAll = 7;

// Reference local corner order (core/fea.py:33-36, 140-141): offset -> index.
__host__ __device__ constexpr int corner_k(int ox, int oy, int oz) {
  return oz * 4 + (oy ? (ox ? 2 : 3) : (ox ? 1 : 0));
}

struct Status {
  int code = 0;
  std::string msg;
};

// ---- device-side Krylov state (one per solver, lives in device memory) ----
struct KrylovState {
  double rz;        // r.z of the current iterate
  double rz_new;
  double pAp;
  double alpha;
  double beta;
  double rr;        // ||r||^2
  double fnorm;     // ||mask f||
  double tol;
  double resid;     // last ||r||/fnorm
  double best;      // stall guard: best ratio seen
  double scale;     // mixed: the residual scale of the current inner solve
  double hist_scale;
  double rr_trigger;  // > 0: stop the chunk (KS_RELIABLE) once rr drops below it
  double zap;         // flexible CG: z.Ap of the last iteration
  double gnum, gden;  // learned stage: step gamma = gnum / gden
  int it;           // iterations completed (this solve)
  int it_base;      // history offset (mixed: inner iterations before this solve)
  int max_it;
  int done;         // 1 => every later kernel of the chunk is a no-op
  int status;       // 0 running/ok, 1 converged, 2 max_it, 3 stalled, 4 breakdown, 5 nonfinite
  int stall_guard;
  int restart;      // beta := 0 (rz == 0, multigrid.py:534-545)
  int it_trigger;   // > 0: stop the chunk (KS_RELIABLE) once it reaches it
  int x_it;         // split-precision PCG: iterations whose alpha p is already in x
  unsigned int counter[12];  // last-block-done counters (reductions; [11]: x_it)
};

enum KState { KS_RUNNING = 0, KS_CONVERGED = 1, KS_MAXIT = 2, KS_STALLED = 3,
              KS_BREAKDOWN = 4, KS_NONFINITE = 5, KS_RELIABLE = 6 };

// ----------------------------------------------------------------------------
// Launchers (defined in the .cu files; all asynchronous on `st`).
// ----------------------------------------------------------------------------

// vf_ops.cu -- layout conversion and per-level set-up
template <typename T> void launch_pack_vec(const Grid& g, const double* ref, T* pad, const uint8_t* mask, cudaStream_t st);
template <typename T> void launch_unpack_vec(const Grid& g, const T* pad, double* ref, cudaStream_t st);
template <typename T> void launch_pack_elem(const Grid& g, const double* ref, T* pad, const uint8_t* active, double scale, cudaStream_t st);
template <typename T> void launch_pack_lame(const Grid& g, const double* E, const double* nu_elem, double nu, const uint8_t* active, double scale, T* lam, T* mu, cudaStream_t st);
void launch_pack_mask(const Grid& g, const uint8_t* ref_mask, uint8_t* pad_mask, cudaStream_t st);
void launch_inject_mask(const Grid& f, const uint8_t* fmask, const Grid& c, uint8_t* cmask, cudaStream_t st);
template <typename T> void launch_coarsen_E(const Grid& f, const T* Ef, const Grid& c, T* Ec, cudaStream_t st);
template <typename T> void launch_scale(T* v, long long n, double s, cudaStream_t st);
template <typename T> void launch_inv_diag_fine(const Grid& g, const T* E, const T* mu, double dL, double dM, T* minv3, cudaStream_t st);
template <typename Ts, typename Td> void launch_convert(const Ts* src, Td* dst, long long n, cudaStream_t st);
void launch_used_mask(const Grid& g, const uint8_t* active_pad, uint8_t* mask, cudaStream_t st);
void launch_pack_active(const Grid& g, const uint8_t* ref, uint8_t* pad, cudaStream_t st);

// vf_matvec.cu -- the fine-level (matrix-free hex8) operator family
enum OpEpilogue { EPI_APPLY = 0, EPI_SMOOTH = 1, EPI_RESID = 2 };
struct OpArgs {
  const void* u;      // input vector
  void* out;          // output vector
  const void* b;      // rhs (SMOOTH, RESID)
  const void* minv;   // inverse diagonal, 3 per node (SMOOTH)
  const void* E;      // per-element modulus (or lambda with LAME)
  const void* mu;     // per-element mu (LAME) or nullptr
  const uint8_t* mask;
  double omega;
  double* dot_partials;   // APPLY: optional per-CTA partial of u.out
  KrylovState* ks;        // optional: skip when ks->done; finalize the dot
  int dot_slot;           // which reduction finalizes (see vf_reduce.cuh)
  const double* ke_tab;   // HOST pointer: [KE(nu) | K_lam | K_mu], 3 x 576 doubles
  const double* omega_dev;  // device: damping of this level (overrides omega when set)
  int* err;                 // device error flag (bounded waits that expired), or nullptr
  // SMOOTH as a Chebyshev step: out = u + w Minv (b - A u) + c1 dprev, and
  // dout = out - u (the step's update, the next step's dprev); unused if null
  const void* dprev;
  void* dout;
  const double* c1_dev;
};
template <typename T> void launch_fine_op(const Grid& g, int epi, const OpArgs& a, cudaStream_t st);

// vf_modal.cu -- the same operator in modal z-marching form (default).
// Per-mode material factors: L_k = Elam * cL[k], M_k = Emu * cM[k].
struct ModalConst { float cLf[3], cMf[3]; double cLd[3], cMd[3]; };
ModalConst modal_constants(double nu, bool lame);
template <typename T> void launch_modal_op(const Grid& g, int epi, const OpArgs& a, const ModalConst& mc, int ty,
                                           int zchunk, cudaStream_t st);
template <typename T> int fine_op_grid_blocks(const Grid& g);
// vf_modal_tma.cu -- the modal operator with TMA staging (default form);
// returns false without launching when a tensor map cannot be built
template <typename T> bool launch_modal_tma(const Grid& g, int epi, const OpArgs& a, const ModalConst& mc, int zchunk,
                                            cudaStream_t st);
bool modal_tma_supported();

// vf_stencil.cu -- assembled 27-point block stencils (Galerkin levels)
template <typename T> void launch_stencil_op(const Grid& g, int epi, const OpArgs& a, const T* stencil, cudaStream_t st);
template <typename T> int stencil_op_grid_blocks(const Grid& g);
// Warp-chunked storage of the symmetric scaled stencil (128 values per node,
// 123 used): value k of node p at off(p, k) in units of S.  Chunk j (16 bytes)
// of 32 consecutive nodes is contiguous.  Q: type of the D^1/2 scale vector.
template <typename S> struct SymLayout {
  static constexpr int VPC = 16 / (int)sizeof(S);
  static constexpr int NCH = 128 / VPC;
  using Q = typename std::conditional<sizeof(S) == 8, double, float>::type;
  __host__ __device__ static constexpr long long off(long long p, int k) {
    return ((p >> 5) * NCH + k / VPC) * (32LL * VPC) + (p & 31) * VPC + (k % VPC);
  }
  static size_t count(long long n) { return (size_t)((n + 31) / 32) * 32 * 128; }
};
template <typename S> void launch_stencil_compress(const Grid& g, const double* st, const uint8_t* mask, S* stc,
                                                   typename SymLayout<S>::Q* sqrtd, cudaStream_t st_);
template <typename T, typename S> void launch_stencil_sym_op(const Grid& g, int epi, const OpArgs& a, const S* stc,
                                                             const T* sqrtd, int zchunk, cudaStream_t st);
int sym_zchunk(const Grid& g);
void launch_galerkin_from_fine(const Grid& f, const double* E, const double* mu, const uint8_t* fmask,
                               const Grid& c, double* stencil_c, const double* Gtab, int lame, cudaStream_t st);

// vf_wide.cu -- reach-R Galerkin levels (coarse space with a smoothed prolongation).
// Scaled symmetric storage of a reach-R stencil, split over G = 8 lanes per
// node: block u of a node -- the upper blocks s = center + 1 + u (u < NU)
// and the diagonal block (u = NU), 9 values each -- belongs to lane u % G,
// slot u / G; a lane holds NJ blocks (9 NJ values, zero padded).  Storage is
// warp-chunked over virtual nodes v = p * G + lane: 16-byte chunk j of 32
// consecutive virtual nodes is contiguous, so the 32 lanes of a warp (4
// nodes) load one chunk each in one 512-byte transaction.
template <typename S, int R> struct WideLayout {
  static constexpr int W = 2 * R + 1, NB = W * W * W, NU = NB / 2;
  static constexpr int G = 8;
  static constexpr int NBLK = NU + 1;
  static constexpr int NJ = (NBLK + G - 1) / G;
  static constexpr int NVL = (NJ * 9 + 7) / 8 * 8;
  static constexpr int VPC = 16 / (int)sizeof(S);
  static constexpr int NCH = NVL / VPC;
  using Q = typename std::conditional<sizeof(S) == 8, double, float>::type;
  __host__ __device__ static constexpr long long off(long long v, int k) {
    return ((v >> 5) * NCH + k / VPC) * (32LL * VPC) + (v & 31) * VPC + (k % VPC);
  }
  static size_t count(long long n) { return (size_t)((n * G + 31) / 32) * 32 * NVL; }
};
size_t wide_prolong_count(const Grid& f, int Pr);
size_t wide_rapb_count(const Grid& f, int Pr, int Rf);
// A_c (reach Rc = (2 Pr + Rf) / 2, full FP64 stencil) = P_s^T A_f P_s with
// P_s = D_f (I - c D_f^-1 A_f) P (c = *cdev; cdev null or *cdev == 0: the
// trilinear P, Pr = 1); psb / bsb: scratch of wide_prolong_count /
// wide_rapb_count doubles.
void launch_wide_galerkin(const Grid& f, const double* stf, int Rf, const uint8_t* fmask, const double* minvf,
                          const double* cdev, int Pr, const Grid& c, double* stc, int Rc, double* psb, double* bsb,
                          cudaStream_t st);
void launch_wide_mask(const Grid& c, int R, double* stc, uint8_t* cmask, double* minv3, cudaStream_t st);
// coef = (4/3) / lambda (0 when lambda <= 0), on the device
void launch_smoothing_coef(const double* lambda, double* coef, cudaStream_t st);
template <typename S, int R>
void launch_wide_compress(const Grid& g, const double* st, const uint8_t* mask, S* stc,
                          typename WideLayout<S, R>::Q* sqrtd, cudaStream_t st_);
template <typename T, typename S, int R>
void launch_wide_op(const Grid& g, int epi, const OpArgs& a, const S* stc, const T* sqrtd, cudaStream_t st);
int wide_op_grid_blocks(const Grid& g);
int wide_dense_assemble(const Grid& c, int R, const double* stencil, const uint8_t* cmask, double* A, int n,
                        cudaStream_t st);
void launch_galerkin_from_stencil(const Grid& f, const double* stencil_f, const Grid& c, double* stencil_c, cudaStream_t st);
void launch_stencil_mask_and_diag(const Grid& c, double* stencil, uint8_t* cmask, double* minv3, cudaStream_t st);

// vf_transfer.cu -- restriction / prolongation / first sweep
template <typename T> void launch_restrict(const Grid& f, const T* rf, const Grid& c, const uint8_t* cmask, T* rc, const KrylovState* ks, cudaStream_t st);
template <typename T> void launch_prolong_add(const Grid& c, const T* ec, const Grid& f, const uint8_t* fmask, T* uf, const KrylovState* ks, cudaStream_t st);
// restriction + the coarse level's first smoothing step from zero: uc = w (Minv rc), w = *wdev
template <typename T> void launch_restrict_first(const Grid& f, const T* rf, const Grid& c, const uint8_t* cmask, T* rc, const T* minvc, const double* wdev, T* uc, const KrylovState* ks, cudaStream_t st);
template <typename T> void launch_jacobi_from_zero(const Grid& g, const T* b, const T* minv3, const uint8_t* mask, double omega, const double* omega_dev, T* u, const KrylovState* ks, cudaStream_t st);

// vf_dense.cu -- coarsest-level dense FP64 direct solve
int dense_assemble(const Grid& c, const double* stencil, const uint8_t* cmask, double* A, int n, cudaStream_t st);
int dense_cholesky_inverse(double* A, double* work, int n, int bw, int* d_info, cudaStream_t st);
size_t dense_work_count(int n);
int dense_ld32(int n);   // row stride (floats) of the padded FP32 inverse
void launch_dense_perm(const Grid& c, int* perm, int n, cudaStream_t st);
void launch_dense_convert_pad(const double* A, float* B, int n, cudaStream_t st);
template <typename T> void launch_dense_solve(const double* Ainv, int n, const int* perm, const T* b, T* x, const KrylovState* ks, cudaStream_t st);
void launch_dense_solve_f32(const float* Ainv32, int n, const int* perm, const float* b, float* x, const KrylovState* ks, cudaStream_t st);

// vf_krylov.cu -- fused PCG vector kernels with deterministic FP64 reductions
constexpr int kVecBlocks = 148 * 8;     // grid of the vector kernels (fixed => deterministic)
constexpr int kVecThreads = 256;
template <typename T> void launch_dot(const Grid& g, const T* a, const T* b, double* partials, KrylovState* ks, int slot, cudaStream_t st);
template <typename T> void launch_cg_update(const Grid& g, T* x, const T* p, T* r, const T* Ap, double* partials, KrylovState* ks, double* hist, cudaStream_t st);
template <typename T> void launch_p_update(const Grid& g, T* p, const T* z, KrylovState* ks, cudaStream_t st);
template <typename T> void launch_dot_fcg(const Grid& g, const T* r, const T* z, const T* Ap, double* partials,
                                          KrylovState* ks, cudaStream_t st);
template <typename T> void launch_jacobi_precond(const Grid& g, const T* r, const T* minv3, const uint8_t* mask, T* z, const KrylovState* ks, cudaStream_t st);
template <typename T> void launch_copy_vec(const Grid& g, const T* src, T* dst, const KrylovState* ks, cudaStream_t st);
void launch_norm2_f64(const Grid& g, const double* v, double* partials, KrylovState* ks, int slot, cudaStream_t st);
void launch_ir_prepare(const Grid& g, const double* r64, float* r32, KrylovState* ks, cudaStream_t st);
void launch_ir_accumulate(const Grid& g, double* x64, const float* d32, const KrylovState* ks, cudaStream_t st);
void launch_ir_replace(const Grid& g, const double* r64, float* r32, const KrylovState* ks, cudaStream_t st);
void launch_cg_update_split(const Grid& g, double* r, const double* Ap, float* r32, double* partials,
                            KrylovState* ks, double* hist, cudaStream_t st);
void launch_p_update_split(const Grid& g, double* x, double* p, const float* z, KrylovState* ks, cudaStream_t st);
void launch_dot_fcg_split(const Grid& g, const float* r, const float* z, const double* Ap, double* partials,
                          KrylovState* ks, cudaStream_t st);
void launch_scale64(const Grid& g, const double* x, double* y, double sc, cudaStream_t st);
void launch_sub_from(const Grid& g, const double* f, double* r, cudaStream_t st);
template <typename T> void launch_sub_inplace(const Grid& g, T* y, const T* x, cudaStream_t st);
template <typename T> void launch_axpy_gamma(const Grid& g, T* z, const T* c, const KrylovState* ks, const int* skip,
                                             cudaStream_t st);
// power iteration on D^-1 A (per-level damping)
template <typename T> void launch_power_init(const Grid& g, T* x, const uint8_t* mask, cudaStream_t st);
template <typename T>
void launch_power_scale(const Grid& g, T* y, const T* minv3, double* partials, KrylovState* ks, cudaStream_t st);
template <typename T>
void launch_power_normalize(const Grid& g, const T* y, T* x, const KrylovState* ks, cudaStream_t st);
void launch_cheb_coefs(const double* lambda, int nl, int ratio, double* coef, cudaStream_t st);
void launch_power_omega(const KrylovState* ks, double omega_rel, double safety, double* omega_out, double* lambda_out, cudaStream_t st);

// vf_post.cu -- post-processing and the island pre-step
void launch_von_mises(const Grid& g, const double* u_pad, const double* Es_ref, const double* nu_ref, double nu,
                      const uint8_t* active_ref, const double* B0, double* vm_ref, cudaStream_t st);
void launch_strain_energy(const Grid& g, const double* u_pad, const uint8_t* active_ref, double* se_ref, cudaStream_t st);
int flood_fill_islands(int nx, int ny, int nz, const uint8_t* d_active, const uint8_t* d_fixed_node,
                       uint8_t* d_kept, int* d_changed, cudaStream_t st);

}  // namespace vf
