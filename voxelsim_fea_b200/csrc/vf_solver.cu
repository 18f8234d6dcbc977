// libvoxfea: solver object and C-ABI (include/voxfea.h).
//
// One vf_solver = one device, one non-blocking stream, the level hierarchy of
// core/multigrid.py:141-171 laid out in HBM (vf_common.cuh), and the PCG
// state.  The iteration loop of core/multigrid.py:497-546 runs entirely on the
// device: dots finalize into device scalars (vf_reduce.cuh) and every kernel
// of an iteration turns into a no-op once the device-side `done` flag is set,
// so CHUNKS of iterations are captured once as a CUDA graph and replayed; the
// host only reads the state between chunks (progress callbacks, history).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/voxfea.h"
#include "vf_common.cuh"
#include "vf_hex8.h"
#include "vf_reduce.cuh"
#include "vf_nn.cuh"
#include <cuda_fp16.h>

namespace vf {
unsigned long long direct_launches();
// launchers defined in other translation units without a header entry
void launch_elem_allfree(const Grid& f, const uint8_t* fmask, uint8_t* allfree, cudaStream_t st);
void launch_galerkin_from_fine(const Grid& f, const double* E, const double* mu, const uint8_t* fmask,
                               const uint8_t* allfree, const Grid& c, double* stencil_c, const double* Gtab,
                               const double* Ktab, int lame, cudaStream_t st);
void launch_stencil_from_elements(const Grid& g, const double* E, const double* mu, const uint8_t* mask,
                                  double* stencil, const double* Ktab, int lame, cudaStream_t st);
void launch_galerkin_mask(const Grid& c, double* stencil, uint8_t* cmask, double* minv3, cudaStream_t st);
void launch_stencil_diag(const Grid& c, double* stencil, const uint8_t* cmask, double* minv3, cudaStream_t st);
void dense_prepare_smem(int n);
void launch_strain_energy_tab(const Grid& g, const double* u_pad, const uint8_t* active_ref, const double* KE,
                              double* se_ref, cudaStream_t st);
}  // namespace vf

using namespace vf;

namespace vf {
thread_local std::string g_last_error;   // vf_global_last_error (shared with vf_noalloc.cu)
}

namespace {

using vf::g_last_error;
std::atomic<unsigned long long> g_launches{0};

// Kernel nodes of an instantiated chunk graph.
unsigned long long graph_kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
  unsigned long long k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

struct Level {
  Grid g{};
  int zchunk = 0;          // modal kernel: z-planes per CTA (< 0: one even wave)
  int szchunk = 0;         // marching stencil kernel: z-planes per CTA
  uint8_t* mask = nullptr;
  bool galerkin = false;   // operator is the assembled stencil
  double* E64 = nullptr; double* mu64 = nullptr; double* minv64 = nullptr; double* st64 = nullptr;
  float* E32 = nullptr; float* mu32 = nullptr; float* minv32 = nullptr; float* st32 = nullptr;
  // symmetric scaled stencils (Galerkin levels): 123 values per node + sqrt(diag)
  // (reach 2: WideLayout, 568 values per node)
  double* sym64 = nullptr; double* sq64 = nullptr;
  float* sym32 = nullptr; __half* sym16 = nullptr; float* sq32 = nullptr;
  // sym64 / sq64 hold the current stencil: built at set-up for an FP64
  // solver, on the first FP64 use otherwise (a mixed or FP32 solve never
  // applies an FP64 coarse operator)
  bool sym64_ok = false;
  int reach = 1;             // Galerkin stencil reach: 1 (27 blocks) or 2 (125 blocks, vf_wide.cu)
  bool smooth_down = false;  // the transfer to the next level uses the smoothed prolongation
  // x, tmp, resid, rhs, and a second temporary for the smoothed restriction
  double* w64[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float* w32[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

template <typename T> struct Sel;
template <> struct Sel<double> {
  static double* E(Level& l) { return l.E64; }
  static double* mu(Level& l) { return l.mu64; }
  static double* minv(Level& l) { return l.minv64; }
  static double* st(Level& l) { return l.st64; }
  static double* w(Level& l, int i) { return l.w64[i]; }
};
template <> struct Sel<float> {
  static float* E(Level& l) { return l.E32; }
  static float* mu(Level& l) { return l.mu32; }
  static float* minv(Level& l) { return l.minv32; }
  static float* st(Level& l) { return l.st32; }
  static float* w(Level& l, int i) { return l.w32[i]; }
};

}  // namespace

struct vf_solver {
  int device = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;   // set-up work that overlaps the main stream (coarsest factorization)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  vf_options o{};
  double nu = 0.3;
  int nx = 0, ny = 0, nz = 0;
  std::vector<Level> L;
  double tab[1728];    // KE(nu) | K_lam | K_mu
  vf::ModalConst mc{}, mc_lame{};
  double B0[144];
  double* d_Gtab = nullptr;   // Galerkin child tables (8 or 16 x 576)
  double* d_Ktab = nullptr;   // KE or K_lam|K_mu (576 or 1152)
  double* d_Gtab_lame = nullptr;
  double* d_Ktab_lame = nullptr;
  bool have_fixed = false, have_material = false, lame = false;
  std::vector<uint8_t> h_mask_ref;     // level-0 free bits, reference node order
  uint8_t* d_active_ref = nullptr;     // per element (reference order)
  std::vector<uint8_t> h_active;        // host copy (Jacobi default max_it)
  uint8_t* d_active_pad = nullptr;
  bool have_active = false;
  uint8_t* d_allfree = nullptr;
  // coarsest dense factor
  double* d_Ainv = nullptr;
  float* d_Ainv32 = nullptr;    // FP32 copy of the coarsest inverse for the FP32 V-cycle (rows of dense_ld32(n))
  int* d_dense_perm = nullptr;  // padded-vector index of each coarsest DOF
  double* d_dense_work = nullptr;
  int dense_n = 0;
  int* d_info = nullptr;
  // Krylov vectors on level 0: x, r, z, p, Ap
  double* k64[5] = {};
  float* k32[5] = {};
  double* f64 = nullptr;      // padded masked rhs
  double* r64 = nullptr;      // outer residual (mixed)
  KrylovState* ks = nullptr;
  KrylovState* h_ks = nullptr;   // pinned
  double* d_partials = nullptr;
  double* d_hist = nullptr;
  int hist_cap = 0;
  std::vector<double> history;
  std::string err;
  double* d_ref_a = nullptr;   // staging, reference layout (max(ndof, nelem) doubles)
  double* d_ref_b = nullptr;
  double* d_ref_c = nullptr;
  uint8_t* d_ref_u8 = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  // FP64 MG / FP32 MG / Jacobi / FP64 PCG with the FP32 V-cycle
  cudaGraphExec_t chunk[4] = {nullptr, nullptr, nullptr, nullptr};
  unsigned long long chunk_kernels[4] = {0, 0, 0, 0};
  std::vector<void*> allocs;
  double last_setup_ms = 0.0;
  double last_best = 0.0;       // stall guard: best ratio of the last solve
  // learned preconditioner stage (vf_learned.cu)
  vf::NnStage* nn = nullptr;
  int nn_level = 1;
  bool nn_on = false;
  bool nn_stagnated = false;    // run_chunks stopped a learned-stage solve that stopped progressing
  double* d_nn_eref = nullptr;  // [0] max voxel modulus, [1..] reduction scratch
  int* d_err = nullptr;         // kernels' error flag (expired bounded waits)
  double* d_omega = nullptr;    // damping per level (read by the smoothers)
  double* d_lambda = nullptr;   // lambda_max(D^-1 A_l) estimates (VF_OMEGA_AUTO)
  double* d_cheb = nullptr;     // Chebyshev steps per level: [level][step][c1, c2]
  double* d_spc = nullptr;      // smoothed transfers: c_l = (4/3) / lambda_l per level
  double* d_one = nullptr;      // the constant 1 (step field of the smoothed prolongation)
  double* d_psb = nullptr;      // set-up scratch of the wide Galerkin products (vf_wide.cu)
  double* d_bsb = nullptr;
  std::vector<char> lam_done;   // lambda_l already estimated during this set-up
  std::vector<double> h_omega, h_lambda;
  // block right-hand sides: solvers that share this one's operator data and
  // own their vectors, Krylov state, stream and graphs (vf_solve_block)
  std::vector<vf_solver*> children;
  bool is_child = false;
  bool tuned = false;
};

namespace {

#define VF_TRY(expr)                                                                  \
  do {                                                                                \
    cudaError_t _e = (expr);                                                          \
    if (_e != cudaSuccess) {                                                          \
      s->err = std::string(#expr) + ": " + cudaGetErrorString(_e);                    \
      return (_e == cudaErrorMemoryAllocation) ? VF_ERR_NOMEM : VF_ERR_CUDA;          \
    }                                                                                 \
  } while (0)

#define VF_CHECK_LAUNCH()                                                             \
  do {                                                                                \
    cudaError_t _e = cudaGetLastError();                                              \
    if (_e != cudaSuccess) {                                                          \
      s->err = std::string("kernel launch: ") + cudaGetErrorString(_e);               \
      return VF_ERR_CUDA;                                                             \
    }                                                                                 \
  } while (0)

template <typename T>
int dalloc(vf_solver* s, T** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    s->err = std::string("cudaMalloc(") + std::to_string(count * sizeof(T)) + " B): " + cudaGetErrorString(e);
    return VF_ERR_NOMEM;
  }
  // zeroed on the solver's own (non-blocking) stream: a legacy-stream memset
  // is not ordered before the solver's kernels and could land after them
  e = cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(T), s->st);
  if (e != cudaSuccess) { s->err = cudaGetErrorString(e); return VF_ERR_CUDA; }
  s->allocs.push_back(q);
  *p = (T*)q;
  return VF_OK;
}

#define VF_ALLOC(ptr, count)                              \
  do {                                                    \
    int _rc = dalloc(s, &(ptr), (size_t)(count));         \
    if (_rc) return _rc;                                  \
  } while (0)

std::vector<std::array<int, 3>> level_dims(int nx, int ny, int nz, int min_elems, int max_levels) {
  std::vector<std::array<int, 3>> d{{nx, ny, nz}};
  while ((int)d.size() < max_levels && d.back()[0] % 2 == 0 && d.back()[1] % 2 == 0 && d.back()[2] % 2 == 0 &&
         std::min({d.back()[0], d.back()[1], d.back()[2]}) / 2 >= min_elems / 2 &&
         std::min({d.back()[0], d.back()[1], d.back()[2]}) >= 2) {
    auto b = d.back();
    d.push_back({b[0] / 2, b[1] / 2, b[2] / 2});
  }
  return d;
}

bool use_mg(const vf_solver* s) { return s->o.method == VF_METHOD_MG; }
int nlev(const vf_solver* s) { return use_mg(s) ? (int)s->L.size() : 1; }

// ---------------------------------------------------------------------------
// operator dispatch on one level
// ---------------------------------------------------------------------------
template <typename T> void level_sym_op(vf_solver* s, Level& l, int epi, const OpArgs& a);
void compress_sym64(vf_solver* s, Level& l) {
  if (l.reach == 2) launch_wide_compress<double, 2>(l.g, l.st64, l.mask, l.sym64, l.sq64, s->st);
  else launch_stencil_compress<double>(l.g, l.st64, l.mask, l.sym64, l.sq64, s->st);
  l.sym64_ok = true;
}
template <> void level_sym_op<double>(vf_solver* s, Level& l, int epi, const OpArgs& a) {
  if (!l.sym64_ok) compress_sym64(s, l);
  if (l.reach == 2) launch_wide_op<double, double, 2>(l.g, epi, a, l.sym64, l.sq64, s->st);
  else launch_stencil_sym_op<double, double>(l.g, epi, a, l.sym64, l.sq64, l.szchunk, s->st);
}
template <> void level_sym_op<float>(vf_solver* s, Level& l, int epi, const OpArgs& a) {
  if (l.reach == 2) {
    if (s->o.coarse_storage == VF_STENCIL_SYM_HALF) launch_wide_op<float, __half, 2>(l.g, epi, a, l.sym16, l.sq32, s->st);
    else launch_wide_op<float, float, 2>(l.g, epi, a, l.sym32, l.sq32, s->st);
  } else if (s->o.coarse_storage == VF_STENCIL_SYM_HALF) {
    launch_stencil_sym_op<float, __half>(l.g, epi, a, l.sym16, l.sq32, l.szchunk, s->st);
  } else {
    launch_stencil_sym_op<float, float>(l.g, epi, a, l.sym32, l.sq32, l.szchunk, s->st);
  }
}

int auto_zchunk(const Grid& g, int requested);

// A sweep as a Chebyshev step (omega_dev: the step's Minv weight; c1_dev and
// dprev: the previous step's update; dout: this step's update).
struct SweepStep {
  const double* omega_dev = nullptr;
  const double* c1_dev = nullptr;
  const void* dprev = nullptr;
  void* dout = nullptr;
};

template <typename T>
void level_op(vf_solver* s, int li, int epi, const T* u, T* out, const T* b, KrylovState* ks, double* partials,
              int slot, const SweepStep* step = nullptr) {
  Level& l = s->L[li];
  OpArgs a{};
  a.u = u; a.out = out; a.b = b;
  a.minv = Sel<T>::minv(l);
  a.E = Sel<T>::E(l);
  a.mu = s->lame ? Sel<T>::mu(l) : nullptr;
  a.mask = l.mask;
  a.omega = s->o.omega;
  a.omega_dev = (step && step->omega_dev) ? step->omega_dev : s->d_omega + li;
  if (step) {
    a.c1_dev = step->c1_dev;
    a.dprev = step->dprev;
    a.dout = step->dout;
  }
  a.dot_partials = partials;
  a.ks = ks;
  a.dot_slot = slot;
  a.ke_tab = s->tab;
  a.err = s->d_err;
  if (l.galerkin) {
    if (s->o.coarse_storage == VF_STENCIL_FULL) launch_stencil_op<T>(l.g, epi, a, Sel<T>::st(l), s->st);
    else level_sym_op<T>(s, l, epi, a);
  } else if (s->o.fine_kernel == VF_FINE_GATHER) {
    launch_fine_op<T>(l.g, epi, a, s->st);
  } else {
    const ModalConst& mc = s->lame ? s->mc_lame : s->mc;
    if (s->o.fine_kernel == VF_FINE_MODAL_CPASYNC || !launch_modal_tma<T>(l.g, epi, a, mc, l.zchunk, s->st))
      launch_modal_op<T>(l.g, epi, a, mc, 8, l.zchunk > 0 ? l.zchunk : auto_zchunk(l.g, 0), s->st);
  }
}

// Chebyshev smoothing of degree `sweeps` (<= 2) on x (through tmp; dbuf
// holds the first step's update when the second step needs it): step 0 is a
// Jacobi sweep weighted 1/theta (from zero: x = Minv b / theta, whose update
// is x itself), step 1 adds c1 times that update (k_cheb_coefs).
template <typename T>
void smooth_cheb(vf_solver* s, int li, T* x, T* tmp, T* dbuf, const T* b, int sweeps, bool from_zero,
                 KrylovState* ks, int dot_slot, bool first_ready = false) {
  Level& l = s->L[li];
  const double* c = s->d_cheb + 4 * li;
  T* cur = x;
  SweepStep s0, s1;
  s0.omega_dev = c + 1;
  s1.omega_dev = c + 3;
  s1.c1_dev = c + 2;
  if (from_zero) {
    T* first = (sweeps % 2 == 1) ? x : tmp;   // (cheb_first_target)
    if (!first_ready) launch_jacobi_from_zero<T>(l.g, b, Sel<T>::minv(l), l.mask, 0.0, c + 1, first, ks, s->st);
    cur = first;
    s1.dprev = first;
  } else {
    T* nxt = tmp;
    const bool last = sweeps == 1;
    if (sweeps > 1) s0.dout = dbuf;
    level_op<T>(s, li, EPI_SMOOTH, cur, nxt, b, ks, (last && dot_slot >= 0) ? s->d_partials : nullptr,
                (last && dot_slot >= 0) ? dot_slot : 0, &s0);
    cur = nxt;
    s1.dprev = dbuf;
  }
  if (sweeps > 1) {
    T* nxt = (cur == x) ? tmp : x;
    level_op<T>(s, li, EPI_SMOOTH, cur, nxt, b, ks, dot_slot >= 0 ? s->d_partials : nullptr,
                dot_slot >= 0 ? dot_slot : 0, &s1);
    cur = nxt;
  }
  if (cur != x) launch_copy_vec<T>(l.g, cur, x, ks, s->st);
}

// `sweeps` damped-Jacobi sweeps on x (in place, through tmp); from_zero uses
// the exact first sweep x = w*Minv*b.
// dot_slot >= 0: the last sweep also reduces b.x into that slot (modal kernels)
template <typename T>
void smooth(vf_solver* s, int li, T* x, T* tmp, const T* b, int sweeps, bool from_zero, KrylovState* ks,
            int dot_slot = -1) {
  Level& l = s->L[li];
  if (sweeps <= 0) {
    if (from_zero) cudaMemsetAsync(x, 0, sizeof(T) * 3 * (size_t)l.g.n, s->st);
    return;
  }
  T* cur;
  int rest;
  if (from_zero) {
    T* first = (sweeps % 2 == 1) ? x : tmp;
    launch_jacobi_from_zero<T>(l.g, b, Sel<T>::minv(l), l.mask, s->o.omega, s->d_omega + li, first, ks, s->st);
    cur = first;
    rest = sweeps - 1;
  } else {
    cur = x;
    rest = sweeps;
  }
  for (int k = 0; k < rest; ++k) {
    T* nxt = (cur == x) ? tmp : x;
    const bool last_dot = dot_slot >= 0 && k + 1 == rest;
    level_op<T>(s, li, EPI_SMOOTH, cur, nxt, b, ks, last_dot ? s->d_partials : nullptr, last_dot ? dot_slot : 0);
    cur = nxt;
  }
  if (cur != x) launch_copy_vec<T>(l.g, cur, x, ks, s->st);
}

// Transfers between level li and li + 1.  Trilinear: r_c = P^T r, x += P e.
// Smoothed (l.smooth_down): with P_s = D (I - c Minv A) P,
//   r_c = P_s^T r = P^T (r - c A (Minv r))   (r masked),
//   x  += P_s e   = t - c Minv A t + x,  t = P e,
// i.e. a from-zero sweep, a residual and the trilinear restriction; and the
// trilinear prolongation into a temporary followed by one sweep of the level
// operator with a zero rhs, weight c and the step field (dprev = x, c1 = 1).
// Temporaries: w[1] and w[4] of level li (free outside the smoothing).
// first != nullptr: the restriction also makes the coarse level's first
// smoothing step from zero, first = (*wfirst) Minv_c rc
template <typename T>
void restrict_to(vf_solver* s, const Level& l, const T* r, Level& c, T* rc, KrylovState* ks, T* first,
                 const double* wfirst) {
  if (first) launch_restrict_first<T>(l.g, r, c.g, c.mask, rc, Sel<T>::minv(c), wfirst, first, ks, s->st);
  else launch_restrict<T>(l.g, r, c.g, c.mask, rc, ks, s->st);
}

template <typename T>
void restrict_level(vf_solver* s, int li, const T* r, T* rc, KrylovState* ks, T* first = nullptr,
                    const double* wfirst = nullptr) {
  Level& l = s->L[li];
  Level& c = s->L[li + 1];
  if (!l.smooth_down) {
    restrict_to<T>(s, l, r, c, rc, ks, first, wfirst);
    return;
  }
  T* z = Sel<T>::w(l, 1);
  T* rs = Sel<T>::w(l, 4);
  launch_jacobi_from_zero<T>(l.g, r, Sel<T>::minv(l), l.mask, 0.0, s->d_spc + li, z, ks, s->st);
  level_op<T>(s, li, EPI_RESID, z, rs, r, ks, nullptr, 0);
  restrict_to<T>(s, l, rs, c, rc, ks, first, wfirst);
}

template <typename T>
void prolong_level(vf_solver* s, int li, const T* ec, T* x, KrylovState* ks) {
  Level& l = s->L[li];
  Level& c = s->L[li + 1];
  if (!l.smooth_down) {
    launch_prolong_add<T>(c.g, ec, l.g, l.mask, x, ks, s->st);
    return;
  }
  T* t = Sel<T>::w(l, 1);
  cudaMemsetAsync(t, 0, sizeof(T) * 3 * (size_t)l.g.n, s->st);
  launch_prolong_add<T>(c.g, ec, l.g, l.mask, t, ks, s->st);
  SweepStep st;
  st.omega_dev = s->d_spc + li;
  st.c1_dev = s->d_one;
  st.dprev = x;
  level_op<T>(s, li, EPI_SMOOTH, t, x, nullptr, ks, nullptr, 0, &st);
}

template <typename T>
void coarse_solve(vf_solver* s, int li, const T* b, T* x, KrylovState* ks) {
  Level& l = s->L[li];
  if (s->o.coarsest == VF_COARSEST_CHOLESKY && s->d_Ainv) {
    if constexpr (sizeof(T) == 4) {
      if (s->d_Ainv32) launch_dense_solve_f32(s->d_Ainv32, s->dense_n, s->d_dense_perm, b, x, ks, s->st);
      else launch_dense_solve<T>(s->d_Ainv, s->dense_n, s->d_dense_perm, b, x, ks, s->st);
    } else {
      launch_dense_solve<T>(s->d_Ainv, s->dense_n, s->d_dense_perm, b, x, ks, s->st);
    }
  } else {
    smooth<T>(s, li, x, Sel<T>::w(l, 1), b, s->o.coarse_sweeps, true, ks);
  }
}

// pre/post smoothing steps on level li, and whether they are Chebyshev steps
int level_sweeps(const vf_solver* s, int li) {
  const Level& l = s->L[li];
  // a level whose transfer down is smoothed gets one more smoothing step from
  // each of its smoothed restriction and prolongation
  return (l.smooth_down && s->o.smoothed_level_sweeps > 0) ? s->o.smoothed_level_sweeps : s->o.n_smooth;
}
bool level_cheb(const vf_solver* s, int li) {
  return s->o.smoother == VF_SMOOTH_CHEBYSHEV && level_sweeps(s, li) > 0 && li < (int)s->L.size() - 1;
}

// x = V-cycle(b) on level li (core/multigrid.py:426-436); dot_slot >= 0: the
// last sweep on this level also reduces b.x (r.z of the PCG) into that slot.
// first_ready: the restriction into this level already made the first
// Chebyshev step from zero (level_cheb(li))
template <typename T>
void vcycle(vf_solver* s, int li, const T* b, T* x, KrylovState* ks, int dot_slot = -1, bool first_ready = false) {
  Level& l = s->L[li];
  if (li == (int)s->L.size() - 1) {
    coarse_solve<T>(s, li, b, x, ks);
    return;
  }
  Level& c = s->L[li + 1];
  T* tmp = Sel<T>::w(l, 1);
  T* res = Sel<T>::w(l, 2);
  const int sweeps = level_sweeps(s, li);
  const bool cheb = level_cheb(s, li);
  if (cheb) smooth_cheb<T>(s, li, x, tmp, res, b, sweeps, true, ks, -1, first_ready);
  else smooth<T>(s, li, x, tmp, b, sweeps, true, ks);
  level_op<T>(s, li, EPI_RESID, x, res, b, ks, nullptr, 0);
  // the next level's first Chebyshev step from zero rides on the restriction
  // (its target: the next level's x for an odd step count, else its tmp)
  const bool fuse = level_cheb(s, li + 1);
  T* first = fuse ? ((level_sweeps(s, li + 1) % 2 == 1) ? Sel<T>::w(c, 0) : Sel<T>::w(c, 1)) : nullptr;
  restrict_level<T>(s, li, res, Sel<T>::w(c, 3), ks, first, fuse ? s->d_cheb + 4 * (li + 1) + 1 : nullptr);
  vcycle<T>(s, li + 1, Sel<T>::w(c, 3), Sel<T>::w(c, 0), ks, -1, fuse);
  prolong_level<T>(s, li, Sel<T>::w(c, 0), x, ks);
  // (res is free again: the post-smoothing's first update goes there)
  if (cheb) smooth_cheb<T>(s, li, x, tmp, res, b, sweeps, false, ks, dot_slot);
  else smooth<T>(s, li, x, tmp, b, sweeps, false, ks, dot_slot);
}

template <typename T> T** kvec(vf_solver* s);
template <> double** kvec<double>(vf_solver* s) { return s->k64; }
template <> float** kvec<float>(vf_solver* s) { return s->k32; }

bool flexible(const vf_solver* s) { return s->o.flexible || s->nn_on; }

// Learned stage after the V-cycle: z += gamma c, c = P^L NN(R^L r1),
// r1 = r - A z.  The residual the V-cycle leaves is restricted to hierarchy
// level L, the U-Net maps it (with the occupancy / modulus features) to a
// level-L correction, the V-cycle's own prolongation carries it back to the
// fine grid, and gamma = (c.r1) / (c.A c) is the A-norm-optimal step along it
// -- the network gives a direction, the step never increases the error of z.
template <typename T>
void learned_stage(vf_solver* s, const T* r, T* z, KrylovState* ks) {
  Level& l0 = s->L[0];
  T* r1 = Sel<T>::w(l0, 2);   // level-0 work vectors are free once the V-cycle is done
  T* c = Sel<T>::w(l0, 1);
  T* Ac = Sel<T>::w(l0, 0);
  KrylovState* kk = s->ks;     // the step reductions (also before the loop, where ks == nullptr)
  level_op<T>(s, 0, EPI_RESID, z, r1, r, ks, nullptr, 0);
  const T* cur = r1;
  for (int li = 0; li < s->nn_level; ++li) {
    Level& f = s->L[li];
    Level& c = s->L[li + 1];
    launch_restrict<T>(f.g, cur, c.g, c.mask, Sel<T>::w(c, 3), ks, s->st);
    cur = Sel<T>::w(c, 3);
  }
  Level& lL = s->L[s->nn_level];
  const int* skip = ks ? &ks->done : nullptr;
  nn_make_input<T>(s->nn, lL.g, cur, skip, s->st);
  nn_forward(s->nn, skip, s->st);
  nn_make_output<T>(s->nn, lL.g, lL.mask, Sel<T>::w(lL, 0), skip, s->st);
  for (int li = s->nn_level; li >= 1; --li) {
    Level& cl = s->L[li];
    Level& f = s->L[li - 1];
    T* target = (li == 1) ? c : Sel<T>::w(f, 0);
    cudaMemsetAsync(target, 0, sizeof(T) * 3 * (size_t)f.g.n, s->st);
    launch_prolong_add<T>(cl.g, Sel<T>::w(cl, 0), f.g, f.mask, target, ks, s->st);
  }
  level_op<T>(s, 0, EPI_APPLY, c, Ac, nullptr, kk, s->d_partials, SLOT_GDEN);
  launch_dot<T>(l0.g, c, r1, s->d_partials, kk, SLOT_GNUM, s->st);
  launch_axpy_gamma<T>(l0.g, z, c, kk, skip, s->st);
}

// PCG's r.z can come out of the V-cycle's last fine sweep (its rhs is r, its
// output z): modal fine kernels, a fixed preconditioner, at least one sweep.
bool fused_rz(const vf_solver* s) {
  return use_mg(s) && !flexible(s) && s->o.n_smooth >= 1 && s->L.size() > 1 &&
         (s->o.fine_kernel == VF_FINE_MODAL || s->o.fine_kernel == VF_FINE_MODAL_CPASYNC);
}

template <typename T>
void precondition(vf_solver* s, const T* r, T* z, KrylovState* ks, int dot_slot = -1) {
  if (use_mg(s)) {
    vcycle<T>(s, 0, r, z, ks, dot_slot);
    if (s->nn_on) learned_stage<T>(s, r, z, ks);
  } else {
    launch_jacobi_precond<T>(s->L[0].g, r, Sel<T>::minv(s->L[0]), s->L[0].mask, z, ks, s->st);
  }
}

// After z = M r: the beta reduction (PCG r.z, or flexible (r.z, z.Ap)) and p = z + beta p.
// (with fused_rz the PCG r.z was reduced by the V-cycle's last sweep)
template <typename T>
void update_direction(vf_solver* s, const T* r, const T* z, T* p, const T* Ap) {
  const Grid& g = s->L[0].g;
  if (flexible(s)) launch_dot_fcg<T>(g, r, z, Ap, s->d_partials, s->ks, s->st);
  else if (!fused_rz(s)) launch_dot<T>(g, r, z, s->d_partials, s->ks, SLOT_RZ, s->st);
  launch_p_update<T>(g, p, z, s->ks, s->st);
}

// One PCG iteration (core/multigrid.py:497-546 / core/fea.py:548-580).
template <typename T>
void pcg_iteration(vf_solver* s) {
  T** v = kvec<T>(s);
  T *x = v[0], *r = v[1], *z = v[2], *p = v[3], *Ap = v[4];
  const Grid& g = s->L[0].g;
  // the fine operator (level 0), masked, fused with p.Ap -> alpha
  level_op<T>(s, 0, EPI_APPLY, p, Ap, nullptr, s->ks, s->d_partials, SLOT_PAP);
  launch_cg_update<T>(g, x, p, r, Ap, s->d_partials, s->ks, s->d_hist, s->st);
  precondition<T>(s, r, z, s->ks, fused_rz(s) ? SLOT_RZ : -1);
  update_direction<T>(s, r, z, p, Ap);
}

// One iteration of the FP64 PCG preconditioned by the FP32 V-cycle
// (VF_MIXED_OUTER64): the iteration of pcg_iteration<double>, with the
// residual handed to the V-cycle as an FP32 copy and z widened in p = z + beta p.
void pcg_iteration_outer64(vf_solver* s) {
  double *x = s->k64[0], *r = s->k64[1], *p = s->k64[3], *Ap = s->k64[4];
  float *r32 = s->k32[1], *z32 = s->k32[2];
  const Grid& g = s->L[0].g;
  level_op<double>(s, 0, EPI_APPLY, p, Ap, nullptr, s->ks, s->d_partials, SLOT_PAP);
  launch_cg_update_split(g, r, Ap, r32, s->d_partials, s->ks, s->d_hist, s->st);
  precondition<float>(s, r32, z32, s->ks, fused_rz(s) ? SLOT_RZ : -1);
  if (flexible(s)) launch_dot_fcg_split(g, r32, z32, Ap, s->d_partials, s->ks, s->st);
  else if (!fused_rz(s)) launch_dot<float>(g, r32, z32, s->d_partials, s->ks, SLOT_RZ, s->st);
  launch_p_update_split(g, x, p, z32, s->ks, s->st);
}

int graph_slot(const vf_solver* s, bool fp32) { return use_mg(s) ? (fp32 ? 1 : 0) : 2; }
constexpr int kSlotOuter64 = 3;

void drop_graph(vf_solver* s, int slot) {
  if (s->chunk[slot]) {
    cudaGraphExecDestroy(s->chunk[slot]);
    s->chunk[slot] = nullptr;
  }
}

// A solve with the learned stage that stopped progressing (run_chunks'
// watch) or that the stall guard stopped: it is the fallback the stage
// keeps -- plain PCG, the stage switched off, from the current iterate and
// residual, with the rest of the iteration budget.
bool learned_fallback_due(const vf_solver* s) {
  return s->nn_on && (s->nn_stagnated || s->h_ks->status == KS_STALLED);
}

// Run PCG chunks of `iteration` until the device says done.  Host callbacks
// see each new history entry.
int run_chunks(vf_solver* s, void (*iteration)(vf_solver*), int gslot,
               void (*progress)(int, double, double, void*), void* user, double tol) {
  const int K = std::max(1, s->o.check_every);
  if (s->o.use_graphs && !s->chunk[gslot]) {
    cudaGraph_t graph = nullptr;
    VF_TRY(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < K; ++k) iteration(s);
    cudaError_t e = cudaStreamEndCapture(s->st, &graph);
    if (e != cudaSuccess) { s->err = std::string("graph capture: ") + cudaGetErrorString(e); return VF_ERR_CUDA; }
    e = cudaGraphInstantiate(&s->chunk[gslot], graph, 0);
    s->chunk_kernels[gslot] = graph_kernel_nodes(graph);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { s->err = std::string("graph instantiate: ") + cudaGetErrorString(e); return VF_ERR_CUDA; }
  }
  int seen = s->h_ks->it;
  // Host-side bound: the device stops at max_it by itself; if the state
  // ever fails to advance, report an error instead of polling forever.
  const long long max_chunks = (long long)(s->h_ks->max_it + K - 1) / K + 4;
  long long chunks = 0;
  for (;;) {
    if (++chunks > max_chunks) {
      s->err = "PCG state did not reach max_it/convergence within the expected number of chunks";
      return VF_ERR_CUDA;
    }
    if (s->o.use_graphs) {
      VF_TRY(cudaGraphLaunch(s->chunk[gslot], s->st));
      g_launches += s->chunk_kernels[gslot];
    } else {
      for (int k = 0; k < K; ++k) iteration(s);
      VF_CHECK_LAUNCH();
    }
    VF_TRY(cudaMemcpyAsync(s->h_ks, s->ks, sizeof(KrylovState), cudaMemcpyDeviceToHost, s->st));
    VF_TRY(cudaStreamSynchronize(s->st));
    const int it = s->h_ks->it;
    if (it > seen) {
      const int base = s->h_ks->it_base;
      const size_t old = s->history.size();
      s->history.resize(base + it);
      VF_TRY(cudaMemcpy(s->history.data() + base + seen, s->d_hist + base + seen, sizeof(double) * (it - seen),
                        cudaMemcpyDeviceToHost));
      (void)old;
      if (progress)
        for (int k = seen; k < it; ++k) progress(base + k + 1, s->history[base + k], tol, user);
      seen = it;
    }
    if (s->h_ks->done) break;
    // learned stage on: a residual that has not halved over the last
    // learned_watch iterations hands the solve to plain PCG (the caller
    // switches the stage off and continues from the current iterate)
    const int W = s->o.learned_watch;
    if (s->nn_on && W > 0 && it > W) {
      const int base = s->h_ks->it_base;
      if (!(s->history[base + it - 1] < 0.5 * s->history[base + it - 1 - W])) {
        s->nn_stagnated = true;
        break;
      }
    }
  }
  return VF_OK;
}

void init_ks(KrylovState& h, double tol, int max_it, int stall_guard, int it_base, double hist_scale) {
  memset(&h, 0, sizeof(h));
  h.tol = tol;
  h.max_it = max_it;
  h.stall_guard = stall_guard;
  h.it_base = it_base;
  h.hist_scale = hist_scale;
  h.best = std::numeric_limits<double>::infinity();
  h.resid = std::numeric_limits<double>::quiet_NaN();
  h.fnorm = 1.0;
}

int ensure_hist(vf_solver* s, int need) {
  if (need <= s->hist_cap) return VF_OK;
  int cap = std::max(need, 2 * s->hist_cap);
  double* nh = nullptr;
  VF_ALLOC(nh, cap);
  s->d_hist = nh;   // old buffer stays in allocs until destroy
  s->hist_cap = cap;
  // captured graphs hold the old pointer
  for (auto& gexe : s->chunk)
    if (gexe) { cudaGraphExecDestroy(gexe); gexe = nullptr; }
  return VF_OK;
}

// Inner PCG on the already-prepared r (level-0 vectors of precision T), x = 0.
template <typename T>
int pcg_solve(vf_solver* s, double tol, int max_it, int stall_guard, int it_base, double hist_scale, double fnorm,
              void (*progress)(int, double, double, void*), void* user, double tol_report) {
  T** v = kvec<T>(s);
  const Grid& g = s->L[0].g;
  init_ks(*s->h_ks, tol, max_it, stall_guard, it_base, hist_scale);
  s->h_ks->fnorm = fnorm;
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  precondition<T>(s, v[1], v[2], nullptr);
  launch_dot<T>(g, v[1], v[2], s->d_partials, s->ks, SLOT_RZ_INIT, s->st);
  launch_copy_vec<T>(g, v[2], v[3], nullptr, s->st);
  VF_CHECK_LAUNCH();
  if (max_it <= 0) return VF_OK;
  return run_chunks(s, pcg_iteration<T>, graph_slot(s, sizeof(T) == 4), progress, user, tol_report);
}

int map_status(int ks) {
  switch (ks) {
    case KS_STALLED: return VF_ERR_STALLED;
    case KS_NONFINITE: return VF_ERR_NONFINITE;
    default: return VF_OK;
  }
}

// ---------------------------------------------------------------------------
// set-up
// ---------------------------------------------------------------------------
// Partial sums of the fused reductions: one (or two) doubles per CTA of the
// largest grid any reducing kernel can get -- the marching kernels at the
// smallest z-chunk the autotuner may pick, or the fixed vector grid.
size_t partials_needed(const vf_solver* s) {
  size_t m = 2 * (size_t)kVecBlocks;
  for (const auto& l : s->L) {
    const size_t planes = (size_t)l.g.lz + 1;
    const size_t modal = (size_t)((l.g.lx + 31) / 31) * ((l.g.ly + 7) / 7) * planes;
    const size_t sym = (size_t)((l.g.lx + 32) / 32) * ((l.g.ly + 8) / 8) * planes;
    m = std::max(m, std::max(modal, sym));
  }
  return std::max<size_t>(m, 148 * 64);
}

int build_levels(vf_solver* s) {
  auto dims = level_dims(s->nx, s->ny, s->nz, s->o.min_elems, s->o.max_levels);
  if (s->o.method != VF_METHOD_MG) dims.resize(1);
  s->L.resize(dims.size());
  for (size_t i = 0; i < dims.size(); ++i) {
    Level& l = s->L[i];
    l.g = make_grid(dims[i][0], dims[i][1], dims[i][2]);
    if ((long long)l.g.px * l.g.py * l.g.pz * 3 >= (1LL << 31)) {
      s->err = "grid too large for 32-bit indexing";
      return VF_ERR_ARG;
    }
    l.galerkin = (i > 0 && s->o.coarse_op == VF_COARSE_GALERKIN);
    // stencil reach: level 1 is built from the hex8 level (27 blocks); a
    // level below a smoothed transfer reaches (2 Pr + R_fine) / 2 coarse
    // spacings with Pr = 1 + R_fine (smoothed) or 1 (trilinear)
    if (i >= 2 && l.galerkin) {
      const Level& f = s->L[i - 1];
      const int pr = f.smooth_down ? 1 + f.reach : 1;
      l.reach = (2 * pr + f.reach) / 2;
    }
    l.smooth_down = l.galerkin && i + 1 < dims.size() && ((s->o.smoothed_transfers >> i) & 1);
    if (l.reach > 2) {
      s->err = "smoothed transfers give level " + std::to_string(i) + " a stencil reach of " +
               std::to_string(l.reach) + " (at most 2 supported)";
      return VF_ERR_UNSUPPORTED;
    }
    const size_t n = l.g.n;
    const size_t nblk = (size_t)(2 * l.reach + 1) * (2 * l.reach + 1) * (2 * l.reach + 1);
    VF_ALLOC(l.mask, n);
    VF_ALLOC(l.minv64, 3 * n);
    VF_ALLOC(l.minv32, 3 * n);
    if (!l.galerkin) {
      VF_ALLOC(l.E64, n);
      VF_ALLOC(l.E32, n);
    } else {
      VF_ALLOC(l.st64, 9 * nblk * n);
      if (s->o.coarse_storage == VF_STENCIL_FULL) VF_ALLOC(l.st32, 243 * n);
      else {
        using W64 = WideLayout<double, 2>;
        using W32 = WideLayout<float, 2>;
        using W16 = WideLayout<__half, 2>;
        const bool wide = l.reach == 2;
        const size_t c64 = wide ? W64::count(n) : SymLayout<double>::count(n);
        const size_t c32 = wide ? W32::count(n) : SymLayout<float>::count(n);
        const size_t c16 = wide ? W16::count(n) : SymLayout<__half>::count(n);
        VF_ALLOC(l.sym64, c64);
        VF_ALLOC(l.sq64, 3 * n);
        VF_ALLOC(l.sq32, 3 * n);
        if (s->o.coarse_storage == VF_STENCIL_SYM_HALF) VF_ALLOC(l.sym16, c16);
        else VF_ALLOC(l.sym32, c32);
      }
    }
    for (int k = 0; k < 4; ++k) {
      VF_ALLOC(l.w64[k], 3 * n);
      VF_ALLOC(l.w32[k], 3 * n);
    }
    if (l.smooth_down) {
      VF_ALLOC(l.w64[4], 3 * n);
      VF_ALLOC(l.w32[4], 3 * n);
    }
  }
  // set-up scratch of the wide Galerkin products
  {
    size_t np = 0, nb = 0;
    for (size_t i = 2; i < s->L.size(); ++i) {
      const Level& f = s->L[i - 1];
      if (s->L[i].reach < 2) continue;
      const int pr = f.smooth_down ? 1 + f.reach : 1;
      np = std::max(np, wide_prolong_count(f.g, pr));
      nb = std::max(nb, wide_rapb_count(f.g, pr, f.reach));
    }
    if (np) {
      VF_ALLOC(s->d_psb, np);
      VF_ALLOC(s->d_bsb, nb);
    }
  }
  const Grid& g0 = s->L[0].g;
  for (int k = 0; k < 5; ++k) {
    VF_ALLOC(s->k64[k], 3 * (size_t)g0.n);
    VF_ALLOC(s->k32[k], 3 * (size_t)g0.n);
  }
  VF_ALLOC(s->f64, 3 * (size_t)g0.n);
  VF_ALLOC(s->r64, 3 * (size_t)g0.n);
  const size_t nref = std::max<size_t>(3 * (size_t)g0.nodes_ref(), (size_t)g0.elems_ref());
  VF_ALLOC(s->d_ref_a, nref);
  VF_ALLOC(s->d_ref_b, nref);
  VF_ALLOC(s->d_ref_c, nref);
  VF_ALLOC(s->d_ref_u8, nref);
  VF_ALLOC(s->d_active_ref, (size_t)g0.elems_ref());
  VF_ALLOC(s->d_active_pad, (size_t)g0.n);
  VF_ALLOC(s->d_allfree, (size_t)g0.n);
  VF_ALLOC(s->ks, 1);
  VF_ALLOC(s->d_partials, partials_needed(s));
  VF_ALLOC(s->d_info, 1);
  VF_ALLOC(s->d_omega, 16);
  VF_ALLOC(s->d_nn_eref, 148 * 4 + 1);
  // coarsest dense factor: allocated (and zeroed on st) here, because it is
  // built on the second set-up stream, which does not wait for st's memsets
  if (use_mg(s) && s->o.coarsest == VF_COARSEST_CHOLESKY) {
    Level& lc = s->L.back();
    const int n = 3 * lc.g.nodes_ref();
    if (n <= 16384) {
      VF_ALLOC(s->d_Ainv, (size_t)n * n);
      VF_ALLOC(s->d_Ainv32, (size_t)n * dense_ld32(n));
      VF_ALLOC(s->d_dense_perm, (size_t)n);
      VF_ALLOC(s->d_dense_work, dense_work_count(n));
      s->dense_n = n;
      dense_prepare_smem(n);
      launch_dense_perm(lc.g, s->d_dense_perm, n, s->st);
      if (!lc.galerkin && !lc.st64) VF_ALLOC(lc.st64, 243 * (size_t)lc.g.n);
    }
  }
  VF_ALLOC(s->d_err, 1);
  VF_ALLOC(s->d_lambda, 16);
  VF_ALLOC(s->d_cheb, 16 * 2 * 2);
  VF_ALLOC(s->d_spc, 16);
  VF_ALLOC(s->d_one, 1);
  {
    const double one = 1.0;
    VF_TRY(cudaMemcpyAsync(s->d_one, &one, sizeof(double), cudaMemcpyHostToDevice, s->st));
    VF_TRY(cudaStreamSynchronize(s->st));
  }
  VF_TRY(cudaMallocHost(&s->h_ks, sizeof(KrylovState)));
  memset(s->h_ks, 0, sizeof(KrylovState));
  return ensure_hist(s, 4096);
}

// z-planes per CTA of the modal kernel: about 4 CTAs per SM over the level
// (22 planes measured best on the 256x128x128 fine level).
// occupancy / log-modulus features of the learned stage (shear modulus when
// the Poisson ratio is per voxel, else E), normalised by the largest modulus
void nn_refresh_features(vf_solver* s) {
  Level& l0 = s->L[0];
  const double* mod = s->lame ? l0.mu64 : l0.E64;
  launch_max_f64(mod, (long long)l0.g.n, s->d_nn_eref, s->st);
  nn_set_features(s->nn, l0.g, mod, s->d_nn_eref, s->st);
}

// ---------------------------------------------------------------------------
// autotuner: z-planes per CTA of the marching kernels, per level, timed with
// CUDA events on the FP32 Jacobi sweep (the kernel the V-cycle runs most);
// the choice is cached per (grid, kernel form) for the process.
// ---------------------------------------------------------------------------
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune_cache;
int auto_zchunk(const Grid& g, int requested);

int autotune_levels(vf_solver* s) {
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  VF_TRY(cudaEventCreate(&t0));
  VF_TRY(cudaEventCreate(&t1));
  struct Ev {
    cudaEvent_t a, b;
    ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } ev{t0, t1};
  for (size_t li = 0; li < s->L.size(); ++li) {
    Level& l = s->L[li];
    const bool stencil = l.galerkin && s->o.coarse_storage != VF_STENCIL_FULL && l.reach == 1;
    const bool modal = !l.galerkin && s->o.fine_kernel == VF_FINE_MODAL;
    if (!stencil && !modal) continue;
    if (modal && s->o.modal_zchunk != 0) continue;   // fixed by the caller
    const auto key = std::make_tuple(l.g.lx, l.g.ly, l.g.lz, stencil ? 1 + s->o.coarse_storage : 0);
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        (stencil ? l.szchunk : l.zchunk) = it->second;
        continue;
      }
    }
    const int planes = l.g.lz + 1;
    // CTAs of a candidate; candidates that leave SMs idle while a finer split
    // would fill them are not considered (a short level is latency bound)
    const long long tiles = stencil ? (long long)((l.g.lx + 32) / 32) * ((l.g.ly + 8) / 8)
                                    : (long long)((l.g.lx + 31) / 31) * ((l.g.ly + 7) / 7);
    auto ctas = [&](int c) { return tiles * ((planes + c - 1) / c); };
    const long long floor_ctas = std::min<long long>(148, ctas(modal ? 2 : 1));
    // every distinct z-chunk ceil(planes / n) for n = 1..64 z-ranges: the
    // last wave of CTAs can be anywhere from nearly empty to full, and which
    // split fills it best depends on the tile count and the residency
    std::vector<int> cand;
    const int base = stencil ? sym_zchunk(l.g) : auto_zchunk(l.g, 0);
    cand.push_back(base);
    // (the TMA modal kernel's one-wave split, z-chunk -1, is not a candidate:
    // it is ~3 % faster on the 256x128x128 level but its CTAs march
    // neighbouring tiles at different z, so the tile halos miss L2 and the
    // DRAM traffic grows from 219 to 336 MB per sweep)
    for (int n = 1; n <= 64; ++n) {
      const int c = (planes + n - 1) / n;
      if (c >= 1 && (modal ? c >= 2 : true) && ctas(c) >= floor_ctas &&
          std::find(cand.begin(), cand.end(), c) == cand.end())
        cand.push_back(c);
    }
    // two passes, minimum per candidate: the first pass also brings the
    // clocks up after the set-up, which would otherwise favour late candidates
    std::vector<float> tmin(cand.size(), 1e30f);
    for (int pass = 0; pass < 2; ++pass)
      for (size_t ci = 0; ci < cand.size(); ++ci) {
        (stencil ? l.szchunk : l.zchunk) = cand[ci];
        level_op<float>(s, (int)li, EPI_SMOOTH, l.w32[0], l.w32[1], l.w32[3], nullptr, nullptr, 0);   // warm
        VF_TRY(cudaEventRecord(t0, s->st));
        for (int r = 0; r < 6; ++r)
          level_op<float>(s, (int)li, EPI_SMOOTH, l.w32[0], l.w32[1], l.w32[3], nullptr, nullptr, 0);
        VF_TRY(cudaEventRecord(t1, s->st));
        VF_TRY(cudaEventSynchronize(t1));
        VF_CHECK_LAUNCH();
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        tmin[ci] = std::min(tmin[ci], ms);
      }
    int best = base;
    float best_ms = 1e30f;
    for (size_t ci = 0; ci < cand.size(); ++ci)
      if (tmin[ci] < best_ms) { best_ms = tmin[ci]; best = cand[ci]; }
    (stencil ? l.szchunk : l.zchunk) = best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  return VF_OK;
}

int auto_zchunk(const Grid& g, int requested) {
  if (requested != 0) return requested;
  const long long tiles = (long long)((g.lx + 1 + 30) / 31) * ((g.ly + 1 + 6) / 7);
  long long nz = (4LL * 148 + tiles - 1) / tiles;
  if (nz < 1) nz = 1;
  const int planes = g.lz + 1;
  int zc = (int)((planes + nz - 1) / nz);
  return zc < 2 ? 2 : zc;
}

int upload_tables(vf_solver* s) {
  hex8_tables(s->nu, s->tab, s->B0);
  s->mc = vf::modal_constants(s->nu, false);
  s->mc_lame = vf::modal_constants(s->nu, true);
  for (auto& l : s->L) {
    l.zchunk = auto_zchunk(l.g, s->o.modal_zchunk);
    l.szchunk = sym_zchunk(l.g);
  }
  std::vector<double> G(8 * 576), GL(16 * 576);
  galerkin_child_tables(s->tab, G.data());
  galerkin_child_tables(s->tab + 576, GL.data());
  galerkin_child_tables(s->tab + 1152, GL.data() + 8 * 576);
  VF_ALLOC(s->d_Gtab, 8 * 576);
  VF_ALLOC(s->d_Ktab, 576);
  VF_ALLOC(s->d_Gtab_lame, 16 * 576);
  VF_ALLOC(s->d_Ktab_lame, 1152);
  // stream-ordered with the solver's kernels; the host vectors stay alive
  // until the synchronisation below
  VF_TRY(cudaMemcpyAsync(s->d_Gtab, G.data(), sizeof(double) * 8 * 576, cudaMemcpyHostToDevice, s->st));
  VF_TRY(cudaMemcpyAsync(s->d_Ktab, s->tab, sizeof(double) * 576, cudaMemcpyHostToDevice, s->st));
  VF_TRY(cudaMemcpyAsync(s->d_Gtab_lame, GL.data(), sizeof(double) * 16 * 576, cudaMemcpyHostToDevice, s->st));
  VF_TRY(cudaMemcpyAsync(s->d_Ktab_lame, s->tab + 576, sizeof(double) * 1152, cudaMemcpyHostToDevice, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  return VF_OK;
}

// Level masks: level 0 from the fixed DOFs (and the used-node restriction of
// the Jacobi method); rediscretized levels by injection.
int build_masks(vf_solver* s) {
  Level& l0 = s->L[0];
  const int nref = l0.g.nodes_ref();
  VF_TRY(cudaMemcpyAsync(s->d_ref_u8, s->h_mask_ref.data(), nref, cudaMemcpyHostToDevice, s->st));
  launch_pack_mask(l0.g, s->d_ref_u8, l0.mask, s->st);
  if (!use_mg(s) && s->have_active) launch_used_mask(l0.g, s->d_active_pad, l0.mask, s->st);
  for (size_t i = 1; i < s->L.size(); ++i)
    if (!s->L[i].galerkin) launch_inject_mask(s->L[i - 1].g, s->L[i - 1].mask, s->L[i].g, s->L[i].mask, s->st);
  VF_CHECK_LAUNCH();
  return VF_OK;
}

// Per-level damping.  VF_OMEGA_FIXED: the reference's single omega.
// VF_OMEGA_AUTO: omega_l = omega_rel * 2 / lambda_l, lambda_l from a power
// iteration on D^-1 A_l (x <- D^-1 A x / ||.||), so the damped-Jacobi sweep
// stays contractive on every level whatever the contrast (plain omega = 0.6
// is divergent on high modes when lambda_max(D^-1 A) > 3.3, as on noise
// geometry with void elements).
// lambda_max(D^-1 A_li) by power iteration (x <- D^-1 A x / ||.||) into
// d_lambda[li] (padded by 1.1), omega_li into d_omega[li]; in FP32 on the
// V-cycle's FP32 operators (half-precision scaled stencils on Galerkin
// levels): lambda is needed to a few percent, and the FP32 sweeps cost half
// the FP64 ones.
int power_level(vf_solver* s, int li) {
  init_ks(*s->h_ks, 1.0, 1, 0, 0, 1.0);
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  Level& l = s->L[li];
  launch_power_init<float>(l.g, l.w32[0], l.mask, s->st);
  for (int k = 0; k < std::max(2, s->o.power_iters); ++k) {
    level_op<float>(s, li, EPI_APPLY, l.w32[0], l.w32[1], nullptr, nullptr, nullptr, 0);
    launch_power_scale<float>(l.g, l.w32[1], l.minv32, s->d_partials, s->ks, s->st);
    launch_power_normalize<float>(l.g, l.w32[1], l.w32[0], s->ks, s->st);
  }
  launch_power_omega(s->ks, s->o.omega_rel, 1.1, s->d_omega + li, s->d_lambda + li, s->st);
  VF_CHECK_LAUNCH();
  return VF_OK;
}

int set_level_omegas(vf_solver* s) {
  const int nl = nlev(s);
  s->h_omega.assign(nl, s->o.omega);
  s->h_lambda.assign(nl, 0.0);
  if (s->o.omega_mode != VF_OMEGA_AUTO || !use_mg(s)) {
    VF_TRY(cudaMemcpyAsync(s->d_omega, s->h_omega.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, s->st));
    return VF_OK;
  }
  for (int li = 0; li < nl; ++li) {
    if (li < (int)s->lam_done.size() && s->lam_done[li]) continue;   // estimated while the hierarchy was built
    int rc = power_level(s, li);
    if (rc) return rc;
  }
  if (s->o.smoother == VF_SMOOTH_CHEBYSHEV) launch_cheb_coefs(s->d_lambda, nl, s->o.cheb_ratio, s->d_cheb, s->st);
  VF_CHECK_LAUNCH();
  return VF_OK;   // h_omega / h_lambda are read back by fetch_level_omegas (a blocking copy)
}

int fetch_level_omegas(vf_solver* s) {
  const int nl = (int)s->h_omega.size();
  if (s->o.omega_mode != VF_OMEGA_AUTO || !use_mg(s) || nl == 0) return VF_OK;
  VF_TRY(cudaMemcpyAsync(s->h_omega.data(), s->d_omega, sizeof(double) * nl, cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaMemcpyAsync(s->h_lambda.data(), s->d_lambda, sizeof(double) * nl, cudaMemcpyDeviceToHost, s->st));
  return VF_OK;
}

// Runs on s->st2 (the coarsest stencil is final when it starts; see
// vf_set_material), so the factorization overlaps the damping estimates.
int build_dense_coarsest(vf_solver* s) {
  cudaStream_t sd = s->st2 ? s->st2 : s->st;
  Level& lc = s->L.back();
  const int n = 3 * lc.g.nodes_ref();
  if (n > 16384) {
    s->err = "coarsest level has " + std::to_string(n) + " DOFs; the dense coarsest solve supports <= 16384 "
             "(use more levels or VF_COARSEST_JACOBI)";
    return VF_ERR_UNSUPPORTED;
  }
  if (s->dense_n != n) {
    VF_ALLOC(s->d_Ainv, (size_t)n * n);
    VF_ALLOC(s->d_Ainv32, (size_t)n * dense_ld32(n));
    VF_ALLOC(s->d_dense_perm, (size_t)n);
    VF_ALLOC(s->d_dense_work, dense_work_count(n));
    s->dense_n = n;
    dense_prepare_smem(n);
    launch_dense_perm(lc.g, s->d_dense_perm, n, s->st);   // after its zeroing on st; read on st
  }
  double* st = lc.st64;
  if (!lc.galerkin) {
    // stencil of the rediscretized element operator on the coarsest level
    if (!lc.st64) VF_ALLOC(lc.st64, 243 * (size_t)lc.g.n);
    st = lc.st64;
    launch_stencil_from_elements(lc.g, lc.E64, s->lame ? lc.mu64 : nullptr, lc.mask, st,
                                 s->lame ? s->d_Ktab_lame : s->d_Ktab, s->lame ? 1 : 0, sd);
  }
  if (lc.reach > 1) wide_dense_assemble(lc.g, lc.reach, st, lc.mask, s->d_Ainv, n, sd);
  else dense_assemble(lc.g, st, lc.mask, s->d_Ainv, n, sd);
  // DOF bandwidth of the reach-R stencil in reference node order
  const long long nx1 = lc.g.lx + 1, ny1 = lc.g.ly + 1;
  const long long bw = 3LL * std::max(lc.reach, 1) * (1 + nx1 + nx1 * ny1) + 2;
  dense_cholesky_inverse(s->d_Ainv, s->d_dense_work, n, (int)std::min<long long>(bw, n), s->d_info, sd);
  launch_dense_convert_pad(s->d_Ainv, s->d_Ainv32, n, sd);
  VF_CHECK_LAUNCH();
  int info = 0;
  VF_TRY(cudaMemcpyAsync(&info, s->d_info, sizeof(int), cudaMemcpyDeviceToHost, sd));
  VF_TRY(cudaStreamSynchronize(sd));
  if (info != 0) {
    s->err = "coarsest-level Cholesky: non-positive pivot at row " + std::to_string(info - 1) +
             " (singular coarse operator: is the part supported?)";
    return VF_ERR_BREAKDOWN;
  }
  return VF_OK;
}

}  // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

int vf_abi_version(void) { return VF_ABI_VERSION; }

int vf_get_stream(const vf_solver* s, void** stream) {
  if (!s || !stream) return VF_ERR_ARG;
  *stream = (void*)s->st;
  return VF_OK;
}

int vf_launch_count(uint64_t* count) {
  if (!count) return VF_ERR_ARG;
  *count = (uint64_t)(g_launches.load() + vf::direct_launches());
  return VF_OK;
}

const char* vf_status_string(int status) {
  switch (status) {
    case VF_OK: return "ok";
    case VF_ERR_ARG: return "invalid argument";
    case VF_ERR_STATE: return "invalid call order";
    case VF_ERR_CUDA: return "CUDA error";
    case VF_ERR_NOMEM: return "out of device memory";
    case VF_ERR_NO_DEVICE: return "no usable CUDA device";
    case VF_ERR_STALLED: return "MG-PCG stalled/diverged";
    case VF_ERR_NONFINITE: return "non-finite value";
    case VF_ERR_UNSUPPORTED: return "unsupported option";
    case VF_ERR_BREAKDOWN: return "breakdown";
    default: return "unknown status";
  }
}

const char* vf_global_last_error(void) { return g_last_error.c_str(); }

int vf_hex8_tables(double nu, double* KE, double* KL, double* KM, double* B0) {
  if (!(nu > -1.0 && nu < 0.5)) { g_last_error = "Poisson ratio must lie in (-1, 0.5)"; return VF_ERR_ARG; }
  double tab[1728], b0[144];
  hex8_tables(nu, tab, b0);
  if (KE) memcpy(KE, tab, sizeof(double) * 576);
  if (KL) memcpy(KL, tab + 576, sizeof(double) * 576);
  if (KM) memcpy(KM, tab + 1152, sizeof(double) * 576);
  if (B0) memcpy(B0, b0, sizeof(double) * 144);
  return VF_OK;
}

int vf_device_count(int32_t* count) {
  if (!count) return VF_ERR_ARG;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) { *count = 0; g_last_error = cudaGetErrorString(e); return VF_ERR_NO_DEVICE; }
  *count = n;
  return VF_OK;
}

void vf_options_default(vf_options* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->struct_size = (int32_t)sizeof(vf_options);
  o->method = VF_METHOD_MG;
  o->precision = VF_PREC_FP64;
  o->n_smooth = 2;
  o->min_elems = 4;
  o->max_levels = 6;
  o->coarse_op = VF_COARSE_REDISCRETIZE;
  o->coarsest = VF_COARSEST_JACOBI;
  o->coarse_sweeps = 30;
  o->stall_guard = 1;
  o->check_every = 8;
  o->use_graphs = 1;
  o->device = 0;
  o->max_outer = 20;
  o->omega = 0.6;
  o->inner_tol = 1e-2;
  o->omega_mode = VF_OMEGA_FIXED;
  o->power_iters = 20;
  o->omega_rel = 0.8;
  o->fine_kernel = VF_FINE_MODAL;
  o->modal_zchunk = 0;
  o->coarse_storage = VF_STENCIL_SYM_HALF;
  o->mixed_mode = VF_MIXED_OUTER64;
  o->smoother = VF_SMOOTH_JACOBI;
  o->cheb_ratio = 30;
  o->autotune = 1;
  o->learned_watch = 64;
}

int vf_destroy(vf_solver* s) {
  if (!s) return VF_OK;
  cudaSetDevice(s->device);
  for (vf_solver* c : s->children) vf_destroy(c);
  s->children.clear();
  if (s->st) cudaStreamSynchronize(s->st);
  for (auto& gexe : s->chunk)
    if (gexe) cudaGraphExecDestroy(gexe);
  for (void* p : s->allocs) cudaFree(p);
  if (s->nn) vf::nn_destroy(s->nn);
  if (s->h_ks) cudaFreeHost(s->h_ks);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->ev2) cudaEventDestroy(s->ev2);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  if (s->st2) { cudaStreamSynchronize(s->st2); cudaStreamDestroy(s->st2); }
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
  return VF_OK;
}

int vf_create(int32_t nx, int32_t ny, int32_t nz, double nu, const vf_options* opts, vf_solver** out) {
  if (!out) { g_last_error = "out is NULL"; return VF_ERR_ARG; }
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1) { g_last_error = "grid dimensions must be >= 1"; return VF_ERR_ARG; }
  if (!(nu > -1.0 && nu < 0.5)) { g_last_error = "Poisson ratio must lie in (-1, 0.5)"; return VF_ERR_ARG; }
  vf_options o;
  vf_options_default(&o);
  if (opts) {
    if (opts->struct_size != (int32_t)sizeof(vf_options)) { g_last_error = "vf_options.struct_size mismatch"; return VF_ERR_ARG; }
    o = *opts;
  }
  if (o.precision < 0 || o.precision > 2 || o.method < 0 || o.method > 1 || o.coarse_op < 0 || o.coarse_op > 1 ||
      o.coarsest < 0 || o.coarsest > 1 || o.n_smooth < 0 || o.max_levels < 1 || o.coarse_sweeps < 0 ||
      o.omega_mode < 0 || o.omega_mode > 1 || !(o.omega_rel > 0.0 && o.omega_rel < 1.0) || o.power_iters < 0 ||
      o.fine_kernel < 0 || o.fine_kernel > 2 || o.modal_zchunk < -1 || o.coarse_storage < 0 ||
      o.coarse_storage > 2 || o.mixed_mode < 0 || o.mixed_mode > 2 || o.smoother < 0 || o.smoother > 1 ||
      o.learned_watch < 0 || o.smoothed_level_sweeps < 0) {
    g_last_error = "invalid vf_options field";
    return VF_ERR_ARG;
  }
  if (o.smoother == VF_SMOOTH_CHEBYSHEV &&
      (o.omega_mode != VF_OMEGA_AUTO || o.n_smooth > 2 || o.smoothed_level_sweeps > 2 || o.cheb_ratio < 2 || o.fine_kernel == VF_FINE_GATHER ||
       o.coarse_storage == VF_STENCIL_FULL)) {
    g_last_error = "Chebyshev smoothing needs omega_mode AUTO, n_smooth and smoothed_level_sweeps <= 2, cheb_ratio >= 2, a modal fine kernel "
                   "and symmetric coarse storage";
    return VF_ERR_ARG;
  }
  if (o.smoothed_transfers != 0 &&
      ((o.smoothed_transfers & ~2) != 0 || o.method != VF_METHOD_MG || o.coarse_op != VF_COARSE_GALERKIN ||
       o.omega_mode != VF_OMEGA_AUTO || o.coarse_storage == VF_STENCIL_FULL)) {
    g_last_error = "smoothed transfers: bit 1 (level 1 -> 2) only, with the MG method, Galerkin coarse "
                   "operators, omega_mode AUTO and symmetric coarse storage";
    return VF_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { g_last_error = "no CUDA device"; return VF_ERR_NO_DEVICE; }
  if (o.device < 0 || o.device >= ndev) { g_last_error = "device ordinal out of range"; return VF_ERR_ARG; }
  vf_solver* s = new vf_solver();
  s->o = o;
  s->nu = nu;
  s->nx = nx; s->ny = ny; s->nz = nz;
  s->device = o.device;
  int rc = VF_OK;
  auto fail = [&](int code) {
    g_last_error = s->err;
    vf_destroy(s);
    return code;
  };
  if (cudaSetDevice(s->device) != cudaSuccess) { s->err = "cudaSetDevice failed"; return fail(VF_ERR_CUDA); }
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->st2, cudaStreamNonBlocking) != cudaSuccess) {
    s->err = "stream";
    return fail(VF_ERR_CUDA);
  }
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  cudaEventCreate(&s->ev2);
  cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming);
  if ((rc = build_levels(s))) return fail(rc);
  if ((rc = upload_tables(s))) return fail(rc);
  s->h_mask_ref.assign((size_t)s->L[0].g.nodes_ref(), kFreeAll);
  *out = s;
  return VF_OK;
}

const char* vf_last_error(const vf_solver* s) { return s ? s->err.c_str() : g_last_error.c_str(); }

int vf_num_levels(const vf_solver* s, int32_t* n) {
  if (!s || !n) return VF_ERR_ARG;
  *n = (int32_t)s->L.size();
  return VF_OK;
}

int vf_level_omega(const vf_solver* s, int32_t level, double* omega, double* lambda) {
  if (!s || level < 0 || level >= (int)s->h_omega.size()) return VF_ERR_ARG;
  if (omega) *omega = s->h_omega[level];
  if (lambda) *lambda = s->h_lambda[level];
  return VF_OK;
}

int vf_level_dims(const vf_solver* s, int32_t level, int32_t* dims3) {
  if (!s || !dims3 || level < 0 || level >= (int)s->L.size()) return VF_ERR_ARG;
  dims3[0] = s->L[level].g.lx; dims3[1] = s->L[level].g.ly; dims3[2] = s->L[level].g.lz;
  return VF_OK;
}

int vf_set_fixed(vf_solver* s, const int64_t* fixed, int64_t n) {
  if (!s || (n > 0 && !fixed) || n < 0) return VF_ERR_ARG;
  cudaSetDevice(s->device);
  const long long ndof = 3LL * s->L[0].g.nodes_ref();
  std::fill(s->h_mask_ref.begin(), s->h_mask_ref.end(), kFreeAll);
  for (int64_t i = 0; i < n; ++i) {
    const long long d = fixed[i];
    if (d < 0 || d >= ndof) {
      s->err = "fixed DOF " + std::to_string(d) + " out of range [0, " + std::to_string(ndof) + ")";
      return VF_ERR_ARG;
    }
    s->h_mask_ref[d / 3] &= (uint8_t)~(1u << (d % 3));
  }
  s->have_fixed = true;
  s->have_material = false;   // masks feed the coarse operators
  return build_masks(s);
}

int vf_set_fixed_mask(vf_solver* s, const uint8_t* bits, uint32_t flags) {
  if (!s || !bits) return VF_ERR_ARG;
  cudaSetDevice(s->device);
  const size_t nn = s->h_mask_ref.size();
  std::vector<uint8_t> staged;
  const uint8_t* b = bits;
  if (flags & VF_SOLVE_DEVICE_PTRS) {
    staged.resize(nn);
    VF_TRY(cudaMemcpy(staged.data(), bits, nn, cudaMemcpyDeviceToHost));
    b = staged.data();
  }
  for (size_t i = 0; i < nn; ++i) s->h_mask_ref[i] = (uint8_t)(kFreeAll & ~(b[i] & 7));
  s->have_fixed = true;
  s->have_material = false;   // masks feed the coarse operators
  return build_masks(s);
}

int vf_set_active(vf_solver* s, const uint8_t* active) {
  if (!s) return VF_ERR_ARG;
  cudaSetDevice(s->device);
  const Grid& g0 = s->L[0].g;
  if (active) {
    s->h_active.assign(active, active + (size_t)g0.elems_ref());
    VF_TRY(cudaMemcpyAsync(s->d_active_ref, s->h_active.data(), (size_t)g0.elems_ref(), cudaMemcpyHostToDevice, s->st));
    launch_pack_active(g0, s->d_active_ref, s->d_active_pad, s->st);
    s->have_active = true;
  } else {
    launch_pack_active(g0, nullptr, s->d_active_pad, s->st);
    s->have_active = false;
  }
  VF_CHECK_LAUNCH();
  s->have_material = false;
  return s->have_fixed ? build_masks(s) : VF_OK;
}

int vf_set_material(vf_solver* s, const double* E, const double* nu_elem, uint32_t flags) {
  if (!s || !E) return VF_ERR_ARG;
  const cudaMemcpyKind kind = (flags & VF_SOLVE_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (!s->have_fixed) { s->err = "call set_fixed() before solve()"; return VF_ERR_STATE; }
  cudaSetDevice(s->device);
  VF_TRY(cudaEventRecord(s->ev0, s->st));
  const Grid& g0 = s->L[0].g;
  const size_t ne = (size_t)g0.elems_ref();
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, E, sizeof(double) * ne, kind, s->st));
  const bool lame = nu_elem != nullptr;
  if (lame) VF_TRY(cudaMemcpyAsync(s->d_ref_b, nu_elem, sizeof(double) * ne, kind, s->st));
  if (lame != s->lame) {
    // per-voxel mu arrays on the element-operator levels
    for (auto& l : s->L)
      if (!l.galerkin && !l.mu64) {
        VF_ALLOC(l.mu64, l.g.n);
        VF_ALLOC(l.mu32, l.g.n);
      }
    for (auto& gexe : s->chunk)
      if (gexe) { cudaGraphExecDestroy(gexe); gexe = nullptr; }
    s->lame = lame;
  }
  const uint8_t* act = (!use_mg(s) && s->have_active) ? s->d_active_ref : nullptr;
  Level& l0 = s->L[0];
  if (lame) launch_pack_lame<double>(g0, s->d_ref_a, s->d_ref_b, s->nu, act, 1.0, l0.E64, l0.mu64, s->st);
  else launch_pack_elem<double>(g0, s->d_ref_a, l0.E64, act, 1.0, s->st);
  const double dL = lame ? s->tab[576] : s->tab[0];
  const double dM = lame ? s->tab[1152] : 0.0;
  launch_inv_diag_fine<double>(g0, l0.E64, lame ? l0.mu64 : nullptr, dL, dM, l0.minv64, s->st);
  // A level's FP32 copies / compressed stencils: built as soon as the level is
  // complete when a smoothed transfer needs its lambda, else after the loop.
  std::vector<char> finalized(s->L.size(), 0);
  s->lam_done.assign(s->L.size(), 0);
  auto finalize = [&](size_t i) {
    Level& l = s->L[i];
    const long long n = l.g.n;
    if (!l.galerkin) {
      launch_convert<double, float>(l.E64, l.E32, n, s->st);
      if (lame) launch_convert<double, float>(l.mu64, l.mu32, n, s->st);
    } else if (s->o.coarse_storage == VF_STENCIL_FULL) {
      launch_convert<double, float>(l.st64, l.st32, 243 * n, s->st);
    } else if (l.reach == 2) {
      l.sym64_ok = false;
      if (s->o.precision == VF_PREC_FP64) compress_sym64(s, l);
      if (s->o.coarse_storage == VF_STENCIL_SYM_HALF)
        launch_wide_compress<__half, 2>(l.g, l.st64, l.mask, l.sym16, l.sq32, s->st);
      else
        launch_wide_compress<float, 2>(l.g, l.st64, l.mask, l.sym32, l.sq32, s->st);
    } else {
      l.sym64_ok = false;
      if (s->o.precision == VF_PREC_FP64) compress_sym64(s, l);
      if (s->o.coarse_storage == VF_STENCIL_SYM_HALF)
        launch_stencil_compress<__half>(l.g, l.st64, l.mask, l.sym16, l.sq32, s->st);
      else
        launch_stencil_compress<float>(l.g, l.st64, l.mask, l.sym32, l.sq32, s->st);
    }
    launch_convert<double, float>(l.minv64, l.minv32, 3 * n, s->st);
    finalized[i] = 1;
  };
  if (use_mg(s)) {
    for (size_t i = 1; i < s->L.size(); ++i) {
      Level& f = s->L[i - 1];
      Level& c = s->L[i];
      if (c.galerkin && c.reach == 2) {
        // reach-2 level: from the smoothed (or, below a reach-2 level, the
        // trilinear) prolongation of level i-1
        const int pr = f.smooth_down ? 1 + f.reach : 1;
        if (f.smooth_down) {
          finalize(i - 1);
          int rc = power_level(s, (int)i - 1);
          if (rc) return rc;
          s->lam_done[i - 1] = 1;
          launch_smoothing_coef(s->d_lambda + i - 1, s->d_spc + i - 1, s->st);
        }
        launch_wide_galerkin(f.g, f.st64, f.reach, f.mask, f.minv64, f.smooth_down ? s->d_spc + i - 1 : nullptr, pr,
                             c.g, c.st64, c.reach, s->d_psb, s->d_bsb, s->st);
        launch_wide_mask(c.g, c.reach, c.st64, c.mask, c.minv64, s->st);
      } else if (!c.galerkin) {
        launch_coarsen_E<double>(f.g, f.E64, c.g, c.E64, s->st);
        if (lame) launch_coarsen_E<double>(f.g, f.mu64, c.g, c.mu64, s->st);
        launch_inv_diag_fine<double>(c.g, c.E64, lame ? c.mu64 : nullptr, dL, dM, c.minv64, s->st);
      } else if (i == 1) {
        launch_elem_allfree(f.g, f.mask, s->d_allfree, s->st);
        launch_galerkin_from_fine(f.g, f.E64, lame ? f.mu64 : nullptr, f.mask, s->d_allfree, c.g, c.st64,
                                  lame ? s->d_Gtab_lame : s->d_Gtab, lame ? s->d_Ktab_lame : s->d_Ktab,
                                  lame ? 1 : 0, s->st);
        launch_galerkin_mask(c.g, c.st64, c.mask, c.minv64, s->st);
      } else {
        launch_galerkin_from_stencil(f.g, f.st64, c.g, c.st64, s->st);
        launch_galerkin_mask(c.g, c.st64, c.mask, c.minv64, s->st);
      }
    }
  }
  // FP32 copies and the compressed stencils of the remaining levels
  for (size_t i = 0; i < (size_t)nlev(s); ++i)
    if (!finalized[i]) finalize(i);
  VF_CHECK_LAUNCH();
  // the coarsest factorization (second stream) overlaps the damping estimates
  const bool dense = use_mg(s) && s->o.coarsest == VF_COARSEST_CHOLESKY;
  if (dense) {
    VF_TRY(cudaEventRecord(s->ev_fork, s->st));
    VF_TRY(cudaStreamWaitEvent(s->st2, s->ev_fork, 0));
  }
  {
    int rc = set_level_omegas(s);
    if (rc) return rc;
  }
  if (dense) {
    int rc = build_dense_coarsest(s);   // synchronises st2 (pivot check) while st keeps running
    if (rc) return rc;
    VF_TRY(cudaEventRecord(s->ev_join, s->st2));
    VF_TRY(cudaStreamWaitEvent(s->st, s->ev_join, 0));
  }
  {
    int rc = fetch_level_omegas(s);
    if (rc) return rc;
  }
  if (s->nn) nn_refresh_features(s);
  VF_CHECK_LAUNCH();
  if (s->o.autotune && !s->tuned && use_mg(s)) {
    // the kernels' shapes are baked into the captured graphs: tune before any capture
    int rc = autotune_levels(s);
    if (rc) return rc;
    s->tuned = true;
    for (auto& gexe : s->chunk)
      if (gexe) { cudaGraphExecDestroy(gexe); gexe = nullptr; }
  }
  VF_TRY(cudaEventRecord(s->ev1, s->st));
  VF_TRY(cudaEventSynchronize(s->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  s->last_setup_ms = ms;
  s->have_material = true;
  return VF_OK;
}

int vf_solve(vf_solver* s, const double* f, const double* x0, double tol, int32_t max_it, uint32_t flags,
             double* u_out, vf_solve_info* info) {
  return vf_solve_cb(s, f, x0, tol, max_it, flags, u_out, info, nullptr, nullptr);
}

}  // extern "C"

// Mixed precision with reliable updates (residual replacement).  One FP32
// PCG runs on A d = r / scale (scale = ||f - A x0||, fixed), with FP64 dot
// products.  Whenever its recurrence residual has dropped by inner_tol since
// the last correction -- or the recurrence says converged -- the FP32
// increment is folded into the FP64 solution, the true residual f - A x is
// recomputed in FP64 and replaces the FP32 recurrence residual; the search
// direction and the CG scalars carry on, so the Krylov space is not thrown
// away as a restart would.  Convergence is decided on the FP64 true residual.
int mixed_reliable(vf_solver* s, bool have_x0, double tol, int max_it, double fnorm,
                   void (*progress)(int, double, double, void*), void* user, vf_solve_info& inf, int& status) {
  Level& l0 = s->L[0];
  const Grid& g = l0.g;
  double* x64 = s->k64[0];
  float** v = s->k32;
  if (have_x0) launch_pack_vec<double>(g, s->d_ref_b, x64, l0.mask, s->st);
  else cudaMemsetAsync(x64, 0, sizeof(double) * 3 * (size_t)g.n, s->st);
  auto true_residual = [&](double& ratio, double& rnorm) -> int {
    level_op<double>(s, 0, EPI_APPLY, x64, s->r64, nullptr, nullptr, nullptr, 0);
    launch_sub_from(g, s->f64, s->r64, s->st);
    launch_norm2_f64(g, s->r64, s->d_partials, s->ks, SLOT_PLAIN, s->st);
    VF_CHECK_LAUNCH();
    VF_TRY(cudaMemcpyAsync(s->h_ks, s->ks, sizeof(KrylovState), cudaMemcpyDeviceToHost, s->st));
    VF_TRY(cudaStreamSynchronize(s->st));
    rnorm = std::sqrt(s->h_ks->rr);
    ratio = rnorm / fnorm;
    return VF_OK;
  };
  // the CG state must be idle before the first residual (SLOT_PLAIN writes ks->rr only)
  init_ks(*s->h_ks, tol, max_it, 0, 0, 1.0);
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  double ratio = 0.0, rnorm = 0.0;
  {
    int rc = true_residual(ratio, rnorm);
    if (rc) return rc;
  }
  inf.iters = 0;
  inf.outer_iters = 0;
  inf.resid_ratio = ratio;
  if (!(ratio == ratio)) { status = VF_ERR_NONFINITE; return VF_OK; }
  if (ratio < tol) { inf.converged = 1; return VF_OK; }
  const double scale = rnorm;
  // replacement interval: below ~1e-4 of its starting value the FP32
  // recurrence residual can run ~100x ahead of the true one, and a CG
  // continued from that point on the true residual stalls; 1e-2 keeps the
  // two within a few percent (measured on the 64x16x16 cantilever)
  const double delta = std::min(std::max(s->o.inner_tol, 1e-6), 0.5);
  // CG state: ratio = ||r32|| (fnorm 1), history scaled back to ||r|| / ||f||
  // a replacement cycle that has not gained delta after this many iterations
  // is treated as a stall of the FP32 recurrence: replace AND restart
  const int first_cycle_cap = 400;
  init_ks(*s->h_ks, tol * fnorm / scale, max_it, 0, 0, scale / fnorm);
  s->h_ks->scale = scale;
  s->h_ks->rr_trigger = delta * delta;
  s->h_ks->it_trigger = first_cycle_cap;
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  launch_ir_replace(g, s->r64, v[1], s->ks, s->st);
  cudaMemsetAsync(v[0], 0, sizeof(float) * 3 * (size_t)g.n, s->st);
  precondition<float>(s, v[1], v[2], nullptr);
  launch_dot<float>(g, v[1], v[2], s->d_partials, s->ks, SLOT_RZ_INIT, s->st);
  launch_copy_vec<float>(g, v[2], v[3], nullptr, s->st);
  VF_CHECK_LAUNCH();
  double best = ratio;
  int no_gain = 0;
  const int max_updates = std::max(1, s->o.max_outer) * 8;
  int cycle_start = 0, longest = 0;
  for (;;) {
    int rc = run_chunks(s, pcg_iteration<float>, graph_slot(s, true), progress, user, tol);
    if (rc) return rc;
    const int kst = s->h_ks->status;
    const int it = s->h_ks->it;
    // stopped by the iteration cap, not by a residual drop: the cycle stalled
    const bool stalled = kst == KS_RELIABLE && !(s->h_ks->rr < s->h_ks->rr_trigger);
    if (!stalled) longest = std::max(longest, it - cycle_start);
    cycle_start = it;
    // fold the FP32 increment into x (ks->scale == scale), restart the increment
    launch_ir_accumulate(g, x64, v[0], s->ks, s->st);
    cudaMemsetAsync(v[0], 0, sizeof(float) * 3 * (size_t)g.n, s->st);
    rc = true_residual(ratio, rnorm);
    if (rc) return rc;
    ++inf.outer_iters;
    inf.iters = it;
    inf.resid_ratio = ratio;
    if (!(ratio == ratio) || kst == KS_NONFINITE) { status = VF_ERR_NONFINITE; break; }
    if (ratio < tol) { inf.converged = 1; break; }
    if (kst == KS_MAXIT || kst == KS_BREAKDOWN || it >= max_it || inf.outer_iters >= max_updates) break;
    // FP32 floor: stop when corrections no longer reduce the true residual
    if (ratio < 0.5 * best) { best = ratio; no_gain = 0; }
    else if (++no_gain >= 6) break;
    // replace the recurrence residual by the true one and carry on
    launch_ir_replace(g, s->r64, v[1], s->ks, s->st);
    VF_CHECK_LAUNCH();
    const double rr32 = (rnorm / scale) * (rnorm / scale);
    s->h_ks->done = 0;
    s->h_ks->status = KS_RUNNING;
    s->h_ks->rr = rr32;
    s->h_ks->resid = rnorm / scale;
    s->h_ks->rr_trigger = delta * delta * rr32;
    s->h_ks->it_trigger = it + std::max(100, 3 * std::max(longest, 1));
    VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
    if (stalled) {
      // restart the direction on the replaced residual: z = M r, p = z
      precondition<float>(s, v[1], v[2], s->ks);
      launch_dot<float>(g, v[1], v[2], s->d_partials, s->ks, SLOT_RZ_INIT, s->st);
      launch_copy_vec<float>(g, v[2], v[3], s->ks, s->st);
    } else {
      // the chunk stopped inside an iteration, right after r was updated: finish
      // that iteration on the replaced residual (z = M r, beta, p = z + beta p)
      precondition<float>(s, v[1], v[2], s->ks, fused_rz(s) ? SLOT_RZ : -1);
      update_direction<float>(s, v[1], v[2], v[3], v[4]);
    }
    VF_CHECK_LAUNCH();
  }
  s->history.resize(inf.iters);
  return VF_OK;
}

// FP64 PCG preconditioned by the FP32 V-cycle (VF_MIXED_OUTER64).  The
// system is solved scaled by 1 / ||f|| (A x~ = f / ||f||, x = ||f|| x~), so
// the FP32 residual copies and corrections stay O(1) -> far from FP32's range
// limits whatever the units of E and f; the relative residual, the stall
// guard and the history are those of the FP64 solve.
int mixed_outer64(vf_solver* s, bool have_x0, double tol, int max_it, double fnorm,
                  void (*progress)(int, double, double, void*), void* user, vf_solve_info& inf, int& status) {
  Level& l0 = s->L[0];
  const Grid& g = l0.g;
  double** v = s->k64;
  float** w = s->k32;
  const double inv = 1.0 / fnorm;
  launch_scale64(g, s->f64, v[1], inv, s->st);                       // r~ = f~
  if (have_x0) {
    launch_pack_vec<double>(g, s->d_ref_b, v[0], l0.mask, s->st);
    launch_scale64(g, v[0], v[0], inv, s->st);                       // x~0 = x0 / ||f||
    level_op<double>(s, 0, EPI_APPLY, v[0], s->r64, nullptr, nullptr, nullptr, 0);
    launch_sub_inplace<double>(g, v[1], s->r64, s->st);              // r~ = f~ - A x~0
  } else {
    cudaMemsetAsync(v[0], 0, sizeof(double) * 3 * (size_t)g.n, s->st);
  }
  init_ks(*s->h_ks, tol, max_it, use_mg(s) ? s->o.stall_guard : 0, 0, 1.0);
  s->h_ks->fnorm = 1.0;
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  launch_convert<double, float>(v[1], w[1], 3LL * g.n, s->st);
  precondition<float>(s, w[1], w[2], nullptr);
  launch_dot<float>(g, w[1], w[2], s->d_partials, s->ks, SLOT_RZ_INIT, s->st);
  launch_convert<float, double>(w[2], v[3], 3LL * g.n, s->st);      // p = z
  VF_CHECK_LAUNCH();
  int switched = 0;
  if (max_it > 0) {
    int rc = run_chunks(s, pcg_iteration_outer64, kSlotOuter64, progress, user, tol);
    if (rc) return rc;
    if (learned_fallback_due(s)) {
      s->nn_stagnated = false;
      switched = s->h_ks->it;
      s->nn_on = false;
      drop_graph(s, kSlotOuter64);
      init_ks(*s->h_ks, tol, max_it - switched, use_mg(s) ? s->o.stall_guard : 0, switched, 1.0);
      s->h_ks->fnorm = 1.0;
      VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
      launch_convert<double, float>(v[1], w[1], 3LL * g.n, s->st);   // r (current) -> FP32
      precondition<float>(s, w[1], w[2], nullptr);
      launch_dot<float>(g, w[1], w[2], s->d_partials, s->ks, SLOT_RZ_INIT, s->st);
      launch_convert<float, double>(w[2], v[3], 3LL * g.n, s->st);  // p = z: a restart
      VF_CHECK_LAUNCH();
      rc = max_it > switched ? run_chunks(s, pcg_iteration_outer64, kSlotOuter64, progress, user, tol) : VF_OK;
      s->nn_on = true;
      drop_graph(s, kSlotOuter64);
      if (rc) return rc;
    }
  }
  launch_scale64(g, v[0], v[0], fnorm, s->st);                       // x = ||f|| x~
  VF_CHECK_LAUNCH();
  inf.iters = switched + s->h_ks->it;
  inf.outer_iters = switched;
  inf.converged = s->h_ks->status == KS_CONVERGED;
  inf.resid_ratio = s->h_ks->it > 0 ? s->h_ks->resid : std::numeric_limits<double>::quiet_NaN();
  status = map_status(s->h_ks->status);
  s->last_best = s->h_ks->best;
  return VF_OK;
}

extern "C" int vf_solve_cb(vf_solver* s, const double* f, const double* x0, double tol, int32_t max_it,
                           uint32_t flags, double* u_out, vf_solve_info* info,
                           vf_progress_fn progress, void* user) {
  if (!s || !f || !u_out) return VF_ERR_ARG;
  if (!s->have_fixed) { s->err = "call set_fixed() before solve()"; return VF_ERR_STATE; }
  if (!s->have_material) { s->err = "call set_material() before solve()"; return VF_ERR_STATE; }
  if (!(tol > 0.0)) { s->err = "tol must be > 0"; return VF_ERR_ARG; }
  cudaSetDevice(s->device);
  const bool dev = (flags & VF_SOLVE_DEVICE_PTRS) != 0;
  Level& l0 = s->L[0];
  const Grid& g = l0.g;
  const size_t nref = 3 * (size_t)g.nodes_ref();
  const cudaMemcpyKind h2d = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  VF_TRY(cudaEventRecord(s->ev0, s->st));
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, f, sizeof(double) * nref, h2d, s->st));
  launch_pack_vec<double>(g, s->d_ref_a, s->f64, l0.mask, s->st);   // f = where(free, f, 0)
  if (x0) {
    VF_TRY(cudaMemcpyAsync(s->d_ref_b, x0, sizeof(double) * nref, h2d, s->st));
  }
  VF_CHECK_LAUNCH();
  s->history.clear();
  int n_free = 0;
  if (max_it <= 0) {
    if (use_mg(s)) max_it = 1000;   // multigrid.py:481
    else {
      // fea.py:546: 4 x the free DOFs of the active-restricted system
      const int nx1 = s->nx + 1, ny1 = s->ny + 1;
      std::vector<uint8_t> used(s->h_mask_ref.size(), s->have_active ? 0 : 1);
      if (s->have_active)
        for (int ix = 0; ix < s->nx; ++ix)
          for (int iy = 0; iy < s->ny; ++iy)
            for (int iz = 0; iz < s->nz; ++iz) {
              if (!s->h_active[((size_t)ix * s->ny + iy) * s->nz + iz]) continue;
              for (int k = 0; k < 8; ++k)
                used[(ix + kCorner[k][0]) + (size_t)nx1 * ((iy + kCorner[k][1]) + (size_t)ny1 * (iz + kCorner[k][2]))] = 1;
            }
      for (size_t i = 0; i < s->h_mask_ref.size(); ++i)
        if (used[i]) n_free += __builtin_popcount(s->h_mask_ref[i]);
      max_it = std::max(1, 4 * n_free);
    }
  }
  {
    int rc = ensure_hist(s, max_it + 8);
    if (rc) return rc;
  }
  const bool mixed = s->o.precision == VF_PREC_MIXED;
  const bool fp32 = s->o.precision == VF_PREC_FP32;
  // fnorm = ||mask f|| (multigrid.py:471)
  init_ks(*s->h_ks, tol, max_it, s->o.stall_guard, 0, 1.0);
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  launch_norm2_f64(g, s->f64, s->d_partials, s->ks, SLOT_FNORM, s->st);
  VF_TRY(cudaMemcpyAsync(s->h_ks, s->ks, sizeof(KrylovState), cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  const double fnorm = s->h_ks->fnorm;
  vf_solve_info inf{};
  inf.resid_ratio = std::numeric_limits<double>::quiet_NaN();
  int status = VF_OK;
  double* x64 = s->k64[0];
  if (fnorm == 0.0) {
    // multigrid.py:472-473 / fea.py:543-545: zero load -> zero displacement
    cudaMemsetAsync(x64, 0, sizeof(double) * 3 * (size_t)g.n, s->st);
    inf.converged = use_mg(s) ? 0 : 1;
    inf.iters = -1;
  } else if (!mixed && !fp32) {
    // ---- FP64 PCG (reference algorithm) ----
    double** v = s->k64;
    if (x0) {
      launch_pack_vec<double>(g, s->d_ref_b, v[0], l0.mask, s->st);   // u = where(free, x0, 0)
      level_op<double>(s, 0, EPI_APPLY, v[0], v[1], nullptr, nullptr, nullptr, 0);
      launch_sub_from(g, s->f64, v[1], s->st);                           // r = f - A u
    } else {
      cudaMemsetAsync(v[0], 0, sizeof(double) * 3 * (size_t)g.n, s->st);
      launch_copy_vec<double>(g, s->f64, v[1], nullptr, s->st);
    }
    VF_CHECK_LAUNCH();
    int rc = pcg_solve<double>(s, tol, max_it, use_mg(s) ? s->o.stall_guard : 0, 0, 1.0, fnorm, progress, user, tol);
    if (rc) return rc;
    int switched = 0;
    if (learned_fallback_due(s)) {
      s->nn_stagnated = false;
      switched = s->h_ks->it;
      s->nn_on = false;
      drop_graph(s, graph_slot(s, false));
      rc = pcg_solve<double>(s, tol, max_it - switched, use_mg(s) ? s->o.stall_guard : 0, switched, 1.0, fnorm,
                             progress, user, tol);
      s->nn_on = true;
      drop_graph(s, graph_slot(s, false));
      if (rc) return rc;
    }
    inf.iters = switched + s->h_ks->it;
    inf.outer_iters = switched;
    inf.converged = s->h_ks->status == KS_CONVERGED;
    inf.resid_ratio = s->h_ks->it > 0 ? s->h_ks->resid : std::numeric_limits<double>::quiet_NaN();
    status = map_status(s->h_ks->status);
    s->last_best = s->h_ks->best;
  } else if (fp32) {
    // ---- FP32 vectors/operators, FP64 dots, no refinement ----
    float** v = s->k32;
    launch_convert<double, float>(s->f64, v[1], 3LL * g.n, s->st);
    cudaMemsetAsync(v[0], 0, sizeof(float) * 3 * (size_t)g.n, s->st);
    if (x0) {
      launch_pack_vec<double>(g, s->d_ref_b, s->r64, l0.mask, s->st);
      launch_convert<double, float>(s->r64, v[0], 3LL * g.n, s->st);
      level_op<float>(s, 0, EPI_RESID, v[0], v[2], v[1], nullptr, nullptr, 0);
      launch_copy_vec<float>(g, v[2], v[1], nullptr, s->st);
    }
    VF_CHECK_LAUNCH();
    int rc = pcg_solve<float>(s, tol, max_it, use_mg(s) ? s->o.stall_guard : 0, 0, 1.0, fnorm, progress, user, tol);
    if (rc) return rc;
    launch_convert<float, double>(v[0], x64, 3LL * g.n, s->st);
    inf.iters = s->h_ks->it;
    inf.converged = s->h_ks->status == KS_CONVERGED;
    inf.resid_ratio = s->h_ks->it > 0 ? s->h_ks->resid : std::numeric_limits<double>::quiet_NaN();
    status = map_status(s->h_ks->status);
  } else if (s->o.mixed_mode == VF_MIXED_RELIABLE) {
    int rc = mixed_reliable(s, x0 != nullptr, tol, max_it, fnorm, progress, user, inf, status);
    if (rc) return rc;
  } else if (s->o.mixed_mode == VF_MIXED_OUTER64) {
    int rc = mixed_outer64(s, x0 != nullptr, tol, max_it, fnorm, progress, user, inf, status);
    if (rc) return rc;
  } else {
    // ---- mixed precision iterative refinement ----
    if (x0) launch_pack_vec<double>(g, s->d_ref_b, x64, l0.mask, s->st);
    else cudaMemsetAsync(x64, 0, sizeof(double) * 3 * (size_t)g.n, s->st);
    int total = 0, outer = 0;
    double resid = 0.0;
    for (;;) {
      // r64 = f - A64 x64 (true residual in FP64)
      level_op<double>(s, 0, EPI_APPLY, x64, s->r64, nullptr, nullptr, nullptr, 0);
      launch_sub_from(g, s->f64, s->r64, s->st);
      init_ks(*s->h_ks, tol, max_it, 0, total, 1.0);
      s->h_ks->fnorm = fnorm;
      VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
      launch_norm2_f64(g, s->r64, s->d_partials, s->ks, SLOT_OUTER, s->st);
      VF_CHECK_LAUNCH();
      VF_TRY(cudaMemcpyAsync(s->h_ks, s->ks, sizeof(KrylovState), cudaMemcpyDeviceToHost, s->st));
      VF_TRY(cudaStreamSynchronize(s->st));
      resid = s->h_ks->resid;
      if (!(resid == resid)) { status = VF_ERR_NONFINITE; break; }
      if (resid < tol) { inf.converged = 1; break; }
      if (outer >= s->o.max_outer || total >= max_it) break;
      // inner FP32 solve of A d = r64 / ||r64||
      launch_ir_prepare(g, s->r64, s->k32[1], s->ks, s->st);
      cudaMemsetAsync(s->k32[0], 0, sizeof(float) * 3 * (size_t)g.n, s->st);
      const double itol = std::max(s->o.inner_tol, 0.5 * tol / resid);
      const double scale = std::sqrt(s->h_ks->rr);
      int rc = pcg_solve<float>(s, itol, max_it - total, 0, total, scale / fnorm, 1.0, progress, user, tol);
      if (rc) return rc;
      const int it = s->h_ks->it;
      const int kst = s->h_ks->status;
      // ks->scale was set by ir_prepare before pcg_solve reset the state: restore it
      s->h_ks->scale = scale;
      VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
      launch_ir_accumulate(g, x64, s->k32[0], s->ks, s->st);
      VF_CHECK_LAUNCH();
      total += it;
      ++outer;
      if (kst == KS_NONFINITE) { status = VF_ERR_NONFINITE; break; }
      if (it == 0) break;
    }
    inf.iters = total;
    inf.outer_iters = outer;
    inf.resid_ratio = resid;
    s->history.resize(total);
  }
  // u = where(free, u, 0) and the FP64 true residual
  level_op<double>(s, 0, EPI_APPLY, x64, s->r64, nullptr, nullptr, nullptr, 0);
  launch_sub_from(g, s->f64, s->r64, s->st);
  init_ks(*s->h_ks, tol, 0, 0, 0, 1.0);
  s->h_ks->fnorm = fnorm > 0.0 ? fnorm : 1.0;
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  launch_norm2_f64(g, s->r64, s->d_partials, s->ks, SLOT_OUTER, s->st);
  launch_unpack_vec<double>(g, x64, s->d_ref_c, s->st);
  VF_CHECK_LAUNCH();
  VF_TRY(cudaMemcpyAsync(u_out, s->d_ref_c, sizeof(double) * nref, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                         s->st));
  VF_TRY(cudaMemcpyAsync(s->h_ks, s->ks, sizeof(KrylovState), cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaEventRecord(s->ev1, s->st));
  VF_TRY(cudaEventSynchronize(s->ev1));
  inf.true_resid = fnorm > 0.0 ? s->h_ks->resid : 0.0;
  {
    int kerr = 0;
    VF_TRY(cudaMemcpy(&kerr, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (kerr) {
      s->err = "a kernel's bounded wait on its TMA pipeline expired (results invalid)";
      return VF_ERR_CUDA;
    }
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  inf.device_ms = ms;
  inf.setup_ms = s->last_setup_ms;
  inf.status = status;
  if (info) *info = inf;
  if (status == VF_ERR_STALLED) {
    char buf[320];
    snprintf(buf, sizeof(buf),
             "MG-PCG stalled/diverged at iter %d (resid ratio %.3e, best seen %.3e) -- likely a small/thin "
             "essential-BC patch the coarse grid can't represent well",
             inf.iters, inf.resid_ratio, s->last_best);
    s->err = buf;
  }
  return status;
}

extern "C" {

int vf_resid_history(const vf_solver* s, double* out, int32_t cap, int32_t* n_out) {
  if (!s || !n_out) return VF_ERR_ARG;
  const int n = (int)s->history.size();
  *n_out = n;
  if (out) memcpy(out, s->history.data(), sizeof(double) * std::min(n, (int)cap));
  return VF_OK;
}

int vf_von_mises(vf_solver* s, const double* u, const double* E_stress, const double* nu_elem,
                 const uint8_t* active, double* vm_out) {
  if (!s || !u || !E_stress || !vm_out) return VF_ERR_ARG;
  cudaSetDevice(s->device);
  const Grid& g = s->L[0].g;
  const size_t nref = 3 * (size_t)g.nodes_ref(), ne = (size_t)g.elems_ref();
  double* upad = s->k64[4];
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, u, sizeof(double) * nref, cudaMemcpyHostToDevice, s->st));
  launch_pack_vec<double>(g, s->d_ref_a, upad, nullptr, s->st);
  VF_TRY(cudaMemcpyAsync(s->d_ref_b, E_stress, sizeof(double) * ne, cudaMemcpyHostToDevice, s->st));
  double* nud = nullptr;
  if (nu_elem) {
    VF_TRY(cudaMemcpyAsync(s->d_ref_c, nu_elem, sizeof(double) * ne, cudaMemcpyHostToDevice, s->st));
    nud = s->d_ref_c;
  }
  uint8_t* act = nullptr;
  if (active) {
    VF_TRY(cudaMemcpyAsync(s->d_ref_u8, active, ne, cudaMemcpyHostToDevice, s->st));
    act = s->d_ref_u8;
  }
  launch_von_mises(g, upad, s->d_ref_b, nud, s->nu, act, s->B0, s->d_ref_a, s->st);
  VF_CHECK_LAUNCH();
  VF_TRY(cudaMemcpyAsync(vm_out, s->d_ref_a, sizeof(double) * ne, cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  return VF_OK;
}

int vf_strain_energy(vf_solver* s, const double* u, const uint8_t* active, double* se_out) {
  if (!s || !u || !se_out) return VF_ERR_ARG;
  cudaSetDevice(s->device);
  const Grid& g = s->L[0].g;
  const size_t nref = 3 * (size_t)g.nodes_ref(), ne = (size_t)g.elems_ref();
  double* upad = s->k64[4];
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, u, sizeof(double) * nref, cudaMemcpyHostToDevice, s->st));
  launch_pack_vec<double>(g, s->d_ref_a, upad, nullptr, s->st);
  uint8_t* act = nullptr;
  if (active) {
    VF_TRY(cudaMemcpyAsync(s->d_ref_u8, active, ne, cudaMemcpyHostToDevice, s->st));
    act = s->d_ref_u8;
  }
  launch_strain_energy_tab(g, upad, act, s->tab, s->d_ref_b, s->st);
  VF_CHECK_LAUNCH();
  VF_TRY(cudaMemcpyAsync(se_out, s->d_ref_b, sizeof(double) * ne, cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  return VF_OK;
}

int vf_drop_unsupported_islands(int32_t nx, int32_t ny, int32_t nz, const uint8_t* active, const int64_t* fixed,
                                int64_t n_fixed, uint8_t* kept_out, int64_t* n_removed) {
  if (nx < 1 || ny < 1 || nz < 1 || !active || !kept_out || !n_removed || (n_fixed > 0 && !fixed)) {
    g_last_error = "invalid argument";
    return VF_ERR_ARG;
  }
  const size_t ne = (size_t)nx * ny * nz;
  const size_t nn = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
  std::vector<uint8_t> fixed_node(nn, 0);
  for (int64_t i = 0; i < n_fixed; ++i) {
    if (fixed[i] < 0 || (size_t)fixed[i] >= 3 * nn) { g_last_error = "fixed DOF out of range"; return VF_ERR_ARG; }
    fixed_node[fixed[i] / 3] = 1;
  }
  uint8_t *d_act = nullptr, *d_fix = nullptr, *d_kept = nullptr;
  int* d_changed = nullptr;
  cudaStream_t st = nullptr;
  int rc = VF_OK;
  auto cleanup = [&]() {
    if (d_act) cudaFree(d_act);
    if (d_fix) cudaFree(d_fix);
    if (d_kept) cudaFree(d_kept);
    if (d_changed) cudaFree(d_changed);
    if (st) cudaStreamDestroy(st);
  };
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaMalloc(&d_act, ne) != cudaSuccess ||
      cudaMalloc(&d_fix, nn) != cudaSuccess || cudaMalloc(&d_kept, ne) != cudaSuccess ||
      cudaMalloc(&d_changed, sizeof(int)) != cudaSuccess) {
    g_last_error = "device allocation failed";
    cleanup();
    return VF_ERR_NOMEM;
  }
  std::vector<uint8_t> act01(ne);
  long long n_active = 0;
  for (size_t e = 0; e < ne; ++e) { act01[e] = active[e] ? 1 : 0; n_active += act01[e]; }
  cudaMemcpyAsync(d_act, act01.data(), ne, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_fix, fixed_node.data(), nn, cudaMemcpyHostToDevice, st);
  if (flood_fill_islands(nx, ny, nz, d_act, d_fix, d_kept, d_changed, st) < 0) rc = VF_ERR_CUDA;
  std::vector<uint8_t> kept(ne);
  if (!rc && cudaMemcpyAsync(kept.data(), d_kept, ne, cudaMemcpyDeviceToHost, st) != cudaSuccess) rc = VF_ERR_CUDA;
  if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = VF_ERR_CUDA;
  cleanup();
  if (rc) { g_last_error = "CUDA error in flood fill"; return rc; }
  long long n_kept = 0;
  for (size_t e = 0; e < ne; ++e) n_kept += kept[e];
  if (n_kept == 0) {   // fea.py:220-225: nothing reached -> unchanged
    for (size_t e = 0; e < ne; ++e) kept_out[e] = act01[e];
    *n_removed = 0;
    return VF_OK;
  }
  for (size_t e = 0; e < ne; ++e) kept_out[e] = kept[e];
  *n_removed = n_active - n_kept;
  return VF_OK;
}

}  // extern "C"

// ---- level operators ------------------------------------------------------

static int level_check(vf_solver* s, int level, int precision) {
  if (!s) return VF_ERR_ARG;
  if (level < 0 || level >= nlev(s)) { s->err = "level out of range"; return VF_ERR_ARG; }
  if (precision != VF_PREC_FP64 && precision != VF_PREC_FP32) { s->err = "precision must be FP64 or FP32"; return VF_ERR_ARG; }
  if (!s->have_fixed || !s->have_material) { s->err = "call set_fixed() and set_material() first"; return VF_ERR_STATE; }
  cudaSetDevice(s->device);
  return VF_OK;
}

template <typename T>
static int op_in(vf_solver* s, int level, const double* h, T* pad, const uint8_t* mask) {
  const Grid& g = s->L[level].g;
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, h, sizeof(double) * 3 * (size_t)g.nodes_ref(), cudaMemcpyHostToDevice, s->st));
  launch_pack_vec<T>(g, s->d_ref_a, pad, mask, s->st);
  return VF_OK;
}

template <typename T>
static int op_out(vf_solver* s, int level, const T* pad, double* h) {
  const Grid& g = s->L[level].g;
  launch_unpack_vec<T>(g, pad, s->d_ref_c, s->st);
  VF_CHECK_LAUNCH();
  VF_TRY(cudaMemcpyAsync(h, s->d_ref_c, sizeof(double) * 3 * (size_t)g.nodes_ref(), cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  return VF_OK;
}

template <typename T>
static int apply_t(vf_solver* s, int level, const double* u, double* y) {
  Level& l = s->L[level];
  T* a = Sel<T>::w(l, 0);
  T* b = Sel<T>::w(l, 1);
  int rc = op_in<T>(s, level, u, a, nullptr);
  if (rc) return rc;
  level_op<T>(s, level, EPI_APPLY, a, b, nullptr, nullptr, nullptr, 0);
  return op_out<T>(s, level, b, y);
}

template <typename T>
static int smooth_t(vf_solver* s, int level, const double* u0, const double* b, int sweeps, double* out) {
  Level& l = s->L[level];
  T* x = Sel<T>::w(l, 0);
  T* t = Sel<T>::w(l, 1);
  T* rhs = Sel<T>::w(l, 3);
  int rc = op_in<T>(s, level, u0, x, nullptr);
  if (!rc) rc = op_in<T>(s, level, b, rhs, nullptr);
  if (rc) return rc;
  smooth<T>(s, level, x, t, rhs, sweeps, false, nullptr);
  return op_out<T>(s, level, x, out);
}

template <typename T>
static int restrict_t(vf_solver* s, int level, const double* rf, double* rc_out) {
  Level& l = s->L[level];
  Level& c = s->L[level + 1];
  T* a = Sel<T>::w(l, 2);
  // the smoothed restriction is P_s^T r with P_s = D (...): masked input
  int rc = op_in<T>(s, level, rf, a, l.smooth_down ? l.mask : nullptr);
  if (rc) return rc;
  restrict_level<T>(s, level, a, Sel<T>::w(c, 3), nullptr);
  return op_out<T>(s, level + 1, Sel<T>::w(c, 3), rc_out);
}

template <typename T>
static int prolong_t(vf_solver* s, int level, const double* ec, double* ef) {
  Level& l = s->L[level];
  Level& c = s->L[level + 1];
  int rc = op_in<T>(s, level + 1, ec, Sel<T>::w(c, 0), nullptr);
  if (rc) return rc;
  cudaMemsetAsync(Sel<T>::w(l, 0), 0, sizeof(T) * 3 * (size_t)l.g.n, s->st);
  prolong_level<T>(s, level, Sel<T>::w(c, 0), Sel<T>::w(l, 0), nullptr);
  return op_out<T>(s, level, Sel<T>::w(l, 0), ef);
}

template <typename T>
static int vcycle_t(vf_solver* s, const double* r, double* z) {
  T** v = kvec<T>(s);
  int rc = op_in<T>(s, 0, r, v[1], nullptr);
  if (rc) return rc;
  precondition<T>(s, v[1], v[2], nullptr);
  return op_out<T>(s, 0, v[2], z);
}

extern "C" {

int vf_apply(vf_solver* s, int32_t level, int32_t precision, const double* u, double* y) {
  int rc = level_check(s, level, precision);
  if (rc) return rc;
  if (!u || !y) return VF_ERR_ARG;
  return precision == VF_PREC_FP64 ? apply_t<double>(s, level, u, y) : apply_t<float>(s, level, u, y);
}

int vf_smooth(vf_solver* s, int32_t level, int32_t precision, const double* u0, const double* b, int32_t sweeps,
              double* out) {
  int rc = level_check(s, level, precision);
  if (rc) return rc;
  if (!u0 || !b || !out || sweeps < 0) return VF_ERR_ARG;
  return precision == VF_PREC_FP64 ? smooth_t<double>(s, level, u0, b, sweeps, out)
                                   : smooth_t<float>(s, level, u0, b, sweeps, out);
}

int vf_restrict(vf_solver* s, int32_t level, int32_t precision, const double* rf, double* rc_out) {
  int rc = level_check(s, level, precision);
  if (rc) return rc;
  if (level + 1 >= nlev(s) || !rf || !rc_out) { s->err = "no coarser level"; return VF_ERR_ARG; }
  return precision == VF_PREC_FP64 ? restrict_t<double>(s, level, rf, rc_out) : restrict_t<float>(s, level, rf, rc_out);
}

int vf_prolongate(vf_solver* s, int32_t level, int32_t precision, const double* ec, double* ef) {
  int rc = level_check(s, level, precision);
  if (rc) return rc;
  if (level + 1 >= nlev(s) || !ec || !ef) { s->err = "no coarser level"; return VF_ERR_ARG; }
  return precision == VF_PREC_FP64 ? prolong_t<double>(s, level, ec, ef) : prolong_t<float>(s, level, ec, ef);
}

int vf_vcycle(vf_solver* s, int32_t precision, const double* r, double* z) {
  int rc = level_check(s, 0, precision);
  if (rc) return rc;
  if (!r || !z) return VF_ERR_ARG;
  return precision == VF_PREC_FP64 ? vcycle_t<double>(s, r, z) : vcycle_t<float>(s, r, z);
}

int vf_inv_diagonal(vf_solver* s, int32_t level, double* minv) {
  int rc = level_check(s, level, VF_PREC_FP64);
  if (rc) return rc;
  if (!minv) return VF_ERR_ARG;
  return op_out<double>(s, level, s->L[level].minv64, minv);
}

int vf_time_kernel(vf_solver* s, int32_t kernel, int32_t precision, int32_t iters, double* ms) {
  int rc = level_check(s, 0, precision);
  if (rc) return rc;
  if (!ms || iters < 1 || kernel < 0 || kernel > 5) return VF_ERR_ARG;
  const bool f32 = precision == VF_PREC_FP32;
  Level& l0 = s->L[0];
  init_ks(*s->h_ks, 1.0, 1, 0, 0, 1.0);
  VF_TRY(cudaMemcpyAsync(s->ks, s->h_ks, sizeof(KrylovState), cudaMemcpyHostToDevice, s->st));
  auto one = [&]() {
    if (f32) {
      float** v = s->k32;
      switch (kernel) {
        case 0: level_op<float>(s, 0, EPI_APPLY, v[3], v[4], nullptr, s->ks, s->d_partials, SLOT_PLAIN); break;
        case 1: level_op<float>(s, 0, EPI_SMOOTH, v[3], v[4], v[1], nullptr, nullptr, 0); break;
        case 2: level_op<float>(s, 0, EPI_RESID, v[3], v[4], v[1], nullptr, nullptr, 0); break;
        case 3: if (s->L.size() > 1) launch_restrict<float>(l0.g, v[3], s->L[1].g, s->L[1].mask, s->L[1].w32[3], nullptr, s->st); break;
        case 4: if (s->L.size() > 1) launch_prolong_add<float>(s->L[1].g, s->L[1].w32[0], l0.g, l0.mask, v[4], nullptr, s->st); break;
        default: precondition<float>(s, v[1], v[2], nullptr); break;
      }
    } else {
      double** v = s->k64;
      switch (kernel) {
        case 0: level_op<double>(s, 0, EPI_APPLY, v[3], v[4], nullptr, s->ks, s->d_partials, SLOT_PLAIN); break;
        case 1: level_op<double>(s, 0, EPI_SMOOTH, v[3], v[4], v[1], nullptr, nullptr, 0); break;
        case 2: level_op<double>(s, 0, EPI_RESID, v[3], v[4], v[1], nullptr, nullptr, 0); break;
        case 3: if (s->L.size() > 1) launch_restrict<double>(l0.g, v[3], s->L[1].g, s->L[1].mask, s->L[1].w64[3], nullptr, s->st); break;
        case 4: if (s->L.size() > 1) launch_prolong_add<double>(s->L[1].g, s->L[1].w64[0], l0.g, l0.mask, v[4], nullptr, s->st); break;
        default: precondition<double>(s, v[1], v[2], nullptr); break;
      }
    }
  };
  one();   // warm-up
  VF_TRY(cudaEventRecord(s->ev0, s->st));
  for (int i = 0; i < iters; ++i) one();
  VF_TRY(cudaEventRecord(s->ev1, s->st));
  VF_CHECK_LAUNCH();
  VF_TRY(cudaEventSynchronize(s->ev1));
  float t = 0.f;
  cudaEventElapsedTime(&t, s->ev0, s->ev1);
  *ms = t / iters;
  return VF_OK;
}

// Host evaluation of sum_e E_e Ke u_e on a small grid vs the device (FP64 and
// FP32 element kernels): the library's analogue of backend._self_test.
int vf_self_test(int32_t device) {
  const int nx = 4, ny = 3, nz = 5;
  vf_options o;
  vf_options_default(&o);
  o.device = device;
  vf_solver* s = nullptr;
  int rc = vf_create(nx, ny, nz, 0.3, &o, &s);
  if (rc) return rc;
  const int ne = nx * ny * nz, nn = (nx + 1) * (ny + 1) * (nz + 1);
  std::vector<double> E(ne), u(3 * nn), y(3 * nn), ref(3 * nn, 0.0);
  unsigned long long st = 88172645463325252ULL;
  auto rnd = [&]() { st ^= st << 13; st ^= st >> 7; st ^= st << 17; return (double)(st % 1000003) / 1000003.0; };
  for (auto& e : E) e = 0.5 + rnd();
  for (auto& v : u) v = rnd() - 0.5;
  rc = vf_set_fixed(s, nullptr, 0);
  if (!rc) rc = vf_set_material(s, E.data(), nullptr, 0);
  for (int ix = 0; ix < nx; ++ix)
    for (int iy = 0; iy < ny; ++iy)
      for (int iz = 0; iz < nz; ++iz) {
        const int e = (ix * ny + iy) * nz + iz;
        int dofs[24];
        for (int k = 0; k < 8; ++k) {
          const int nid = (ix + kCorner[k][0]) + (nx + 1) * ((iy + kCorner[k][1]) + (ny + 1) * (iz + kCorner[k][2]));
          for (int c = 0; c < 3; ++c) dofs[3 * k + c] = 3 * nid + c;
        }
        for (int i = 0; i < 24; ++i) {
          double acc = 0.0;
          for (int j = 0; j < 24; ++j) acc += s->tab[i * 24 + j] * u[dofs[j]];
          ref[dofs[i]] += E[e] * acc;
        }
      }
  double scale = 0.0;
  for (double v : ref) scale = std::max(scale, std::fabs(v));
  for (int prec = 0; prec < 2 && !rc; ++prec) {
    rc = vf_apply(s, 0, prec == 0 ? VF_PREC_FP64 : VF_PREC_FP32, u.data(), y.data());
    if (rc) break;
    double err = 0.0;
    for (int i = 0; i < 3 * nn; ++i) err = std::max(err, std::fabs(y[i] - ref[i]));
    if (err > (prec == 0 ? 1e-12 : 1e-5) * scale) {
      g_last_error = "self-test mismatch";
      rc = VF_ERR_CUDA;
    }
  }
  if (rc && s) g_last_error = s->err.empty() ? g_last_error : s->err;
  vf_destroy(s);
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// block right-hand sides
// ---------------------------------------------------------------------------
namespace {

// Point a child at the master's operator data (moduli, masks, diagonals,
// stencils, coarsest factor, damping) -- read-only during solves.
void share_operator(vf_solver* c, const vf_solver* m) {
  c->o = m->o;
  c->lame = m->lame;
  c->mc = m->mc;
  c->mc_lame = m->mc_lame;
  memcpy(c->tab, m->tab, sizeof(c->tab));
  memcpy(c->B0, m->B0, sizeof(c->B0));
  for (size_t i = 0; i < c->L.size(); ++i) {
    Level& d = c->L[i];
    const Level& sl = m->L[i];
    d.g = sl.g; d.zchunk = sl.zchunk; d.szchunk = sl.szchunk; d.mask = sl.mask; d.galerkin = sl.galerkin;
    d.E64 = sl.E64; d.mu64 = sl.mu64; d.minv64 = sl.minv64; d.st64 = sl.st64;
    d.E32 = sl.E32; d.mu32 = sl.mu32; d.minv32 = sl.minv32; d.st32 = sl.st32;
    d.sym64 = sl.sym64; d.sq64 = sl.sq64; d.sym32 = sl.sym32; d.sym16 = sl.sym16; d.sq32 = sl.sq32;
    d.reach = sl.reach; d.smooth_down = sl.smooth_down; d.sym64_ok = sl.sym64_ok;
  }
  c->d_spc = m->d_spc;
  c->d_one = m->d_one;
  c->d_Ainv = m->d_Ainv;
  c->d_Ainv32 = m->d_Ainv32;
  c->d_dense_perm = m->d_dense_perm;
  c->dense_n = m->dense_n;
  c->d_omega = m->d_omega;
  c->d_lambda = m->d_lambda;
  c->d_cheb = m->d_cheb;
  c->h_omega = m->h_omega;
  c->h_lambda = m->h_lambda;
  c->h_mask_ref = m->h_mask_ref;
  c->h_active = m->h_active;
  c->have_active = m->have_active;
  c->d_active_ref = m->d_active_ref;
  c->d_active_pad = m->d_active_pad;
  c->have_fixed = m->have_fixed;
  c->have_material = m->have_material;
  c->last_setup_ms = 0.0;
}

int make_child(vf_solver* m, vf_solver** out) {
  vf_solver* s = new vf_solver();
  s->is_child = true;
  s->device = m->device;
  s->nu = m->nu;
  s->nx = m->nx; s->ny = m->ny; s->nz = m->nz;
  s->L.resize(m->L.size());
  share_operator(s, m);
  auto fail = [&](int code) {
    m->err = "block solve: " + s->err;
    vf_destroy(s);
    return code;
  };
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) { s->err = "stream"; return fail(VF_ERR_CUDA); }
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  cudaEventCreate(&s->ev2);
  auto body = [&]() -> int {
    for (auto& l : s->L) {
      const size_t n = l.g.n;
      for (int k = 0; k < (l.smooth_down ? 5 : 4); ++k) {
        VF_ALLOC(l.w64[k], 3 * n);
        VF_ALLOC(l.w32[k], 3 * n);
      }
    }
    const Grid& g0 = s->L[0].g;
    for (int k = 0; k < 5; ++k) {
      VF_ALLOC(s->k64[k], 3 * (size_t)g0.n);
      VF_ALLOC(s->k32[k], 3 * (size_t)g0.n);
    }
    VF_ALLOC(s->f64, 3 * (size_t)g0.n);
    VF_ALLOC(s->r64, 3 * (size_t)g0.n);
    const size_t nref = 3 * (size_t)g0.nodes_ref();
    VF_ALLOC(s->d_ref_a, nref);
    VF_ALLOC(s->d_ref_b, nref);
    VF_ALLOC(s->d_ref_c, nref);
    VF_ALLOC(s->ks, 1);
    VF_ALLOC(s->d_partials, partials_needed(s));
    VF_ALLOC(s->d_info, 1);
    VF_ALLOC(s->d_err, 1);
    VF_TRY(cudaMallocHost(&s->h_ks, sizeof(KrylovState)));
    memset(s->h_ks, 0, sizeof(KrylovState));
    int rc = ensure_hist(s, 4096);
    if (rc) return rc;
    VF_TRY(cudaStreamSynchronize(s->st));
    return VF_OK;
  };
  int rc = body();
  if (rc) return fail(rc);
  *out = s;
  return VF_OK;
}

}  // namespace

extern "C" {

int vf_solve_block(vf_solver* s, const double* F, int32_t k, double tol, int32_t max_it, uint32_t flags,
                   double* U, vf_solve_info* infos) {
  if (!s || !F || !U || k < 1) return VF_ERR_ARG;
  if (s->is_child) return VF_ERR_STATE;
  if (!s->have_fixed) { s->err = "call set_fixed() before solve()"; return VF_ERR_STATE; }
  if (!s->have_material) { s->err = "call set_material() before solve()"; return VF_ERR_STATE; }
  if (s->nn_on) {   // the stage's activation buffers belong to one solver
    s->err = "block solve: disable the learned stage first (vf_learned_configure enable = 0)";
    return VF_ERR_UNSUPPORTED;
  }
  cudaSetDevice(s->device);
  VF_TRY(cudaStreamSynchronize(s->st));   // the operator is final
  while ((int)s->children.size() < k - 1) {
    vf_solver* c = nullptr;
    int rc = make_child(s, &c);
    if (rc) return rc;
    s->children.push_back(c);
  }
  std::vector<vf_solver*> solvers{s};
  for (int j = 0; j + 1 < k; ++j) {
    vf_solver* c = s->children[j];
    const bool had_graphs = c->chunk[0] || c->chunk[1] || c->chunk[2] || c->chunk[3];
    const double* oldA = c->d_Ainv;
    share_operator(c, s);
    // graphs hold operator pointers and option-dependent launch sequences: re-capture on change
    if (had_graphs && (oldA != c->d_Ainv))
      for (auto& gexe : c->chunk)
        if (gexe) { cudaGraphExecDestroy(gexe); gexe = nullptr; }
    solvers.push_back(c);
  }
  const size_t ndof = 3 * (size_t)s->L[0].g.nodes_ref();
  std::vector<int> rcs(k, VF_OK);
  std::vector<vf_solve_info> inf(k);
  std::vector<std::thread> th;
  for (int j = 0; j < k; ++j) {
    th.emplace_back([&, j]() {
      cudaSetDevice(s->device);
      rcs[j] = vf_solve_cb(solvers[j], F + j * ndof, nullptr, tol, max_it, flags, U + j * ndof, &inf[j], nullptr,
                           nullptr);
    });
  }
  for (auto& t : th) t.join();
  if (infos)
    for (int j = 0; j < k; ++j) infos[j] = inf[j];
  for (int j = 0; j < k; ++j)
    if (rcs[j] != VF_OK && rcs[j] != VF_ERR_STALLED) {
      if (j > 0) s->err = "block solve, right-hand side " + std::to_string(j) + ": " + solvers[j]->err;
      return rcs[j];
    }
  for (int j = 0; j < k; ++j)
    if (rcs[j] != VF_OK) return rcs[j];
  return VF_OK;
}

int vf_solve_batch(vf_solver* const* solvers, int32_t n, const double* const* E, const double* const* nu_elem,
                   const double* const* F, double tol, int32_t max_it, uint32_t flags, double* const* U,
                   vf_solve_info* infos) {
  if (!solvers || !F || !U || n < 1) return VF_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (!solvers[i] || !F[i] || !U[i] || solvers[i]->is_child) return VF_ERR_ARG;
  std::vector<int> rcs(n, VF_OK);
  std::vector<vf_solve_info> inf(n);
  std::vector<std::thread> th;
  th.reserve(n);
  for (int i = 0; i < n; ++i) {
    th.emplace_back([&, i]() {
      vf_solver* s = solvers[i];
      cudaSetDevice(s->device);
      if (E && E[i]) {
        rcs[i] = vf_set_material(s, E[i], nu_elem ? nu_elem[i] : nullptr, flags & VF_SOLVE_DEVICE_PTRS);
        if (rcs[i] != VF_OK) return;
      }
      rcs[i] = vf_solve_cb(s, F[i], nullptr, tol, max_it, flags, U[i], &inf[i], nullptr, nullptr);
    });
  }
  for (auto& t : th) t.join();
  if (infos)
    for (int i = 0; i < n; ++i) infos[i] = inf[i];
  for (int i = 0; i < n; ++i)
    if (rcs[i] != VF_OK && rcs[i] != VF_ERR_STALLED) {
      g_last_error = "batch part " + std::to_string(i) + ": " + solvers[i]->err;
      return rcs[i];
    }
  for (int i = 0; i < n; ++i)
    if (rcs[i] != VF_OK) return rcs[i];
  return VF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// learned preconditioner stage
// ---------------------------------------------------------------------------
extern "C" {

int64_t vf_learned_param_count(void) { return (int64_t)vf::nn_param_count(); }

int vf_learned_configure(vf_solver* s, int32_t level, const float* params, int64_t n_params, int32_t enable) {
  if (!s) return VF_ERR_ARG;
  if (!use_mg(s) || level < 1 || level >= (int)s->L.size()) {
    s->err = "learned stage: level must be a coarse level of the multigrid hierarchy";
    return VF_ERR_ARG;
  }
  if (params && n_params != vf::nn_param_count()) {
    s->err = "learned stage: expected " + std::to_string(vf::nn_param_count()) + " parameters";
    return VF_ERR_ARG;
  }
  cudaSetDevice(s->device);
  if (!s->nn || s->nn_level != level) {
    if (s->nn) { VF_TRY(cudaStreamSynchronize(s->st)); vf::nn_destroy(s->nn); s->nn = nullptr; }
    cudaError_t e = cudaSuccess;
    s->nn = vf::nn_create(s->L[level].g, level, s->st, &e);
    if (!s->nn) { s->err = std::string("learned stage: ") + cudaGetErrorString(e); return VF_ERR_NOMEM; }
    vf::nn_set_error_flag(s->nn, s->d_err);
    s->nn_level = level;
    if (s->have_material) nn_refresh_features(s);
  }
  if (params) VF_TRY(vf::nn_set_weights(s->nn, params, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  const bool on = enable && vf::nn_has_weights(s->nn);
  if (enable && !on) { s->err = "learned stage: no weights"; return VF_ERR_STATE; }
  if (on != s->nn_on) {
    s->nn_on = on;
    for (auto& gexe : s->chunk)   // the captured iterations change
      if (gexe) { cudaGraphExecDestroy(gexe); gexe = nullptr; }
  }
  return VF_OK;
}

int vf_mg_propagate(vf_solver* s, const double* e_in, int32_t n, double* e_out) {
  if (!s || !e_in || !e_out || n < 0) return VF_ERR_ARG;
  if (!s->have_material || !use_mg(s)) { s->err = "set_material first (multigrid)"; return VF_ERR_STATE; }
  cudaSetDevice(s->device);
  Level& l0 = s->L[0];
  const Grid& g = l0.g;
  const size_t nref = 3 * (size_t)g.nodes_ref();
  float** v = s->k32;
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, e_in, sizeof(double) * nref, cudaMemcpyHostToDevice, s->st));
  launch_pack_vec<double>(g, s->d_ref_a, s->r64, l0.mask, s->st);
  launch_convert<double, float>(s->r64, v[0], 3LL * g.n, s->st);
  for (int j = 0; j < n; ++j) {   // e <- e - V(A e), the FP32 V-cycle of the mixed solver
    level_op<float>(s, 0, EPI_APPLY, v[0], v[1], nullptr, nullptr, nullptr, 0);
    vcycle<float>(s, 0, v[1], v[2], nullptr);
    launch_sub_inplace<float>(g, v[0], v[2], s->st);
  }
  launch_convert<float, double>(v[0], s->r64, 3LL * g.n, s->st);
  launch_unpack_vec<double>(g, s->r64, s->d_ref_c, s->st);
  VF_CHECK_LAUNCH();
  VF_TRY(cudaMemcpyAsync(e_out, s->d_ref_c, sizeof(double) * nref, cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  return VF_OK;
}

int vf_level_mask(vf_solver* s, int32_t level, uint8_t* out) {
  if (!s || !out || level < 0 || level >= (int)s->L.size()) return VF_ERR_ARG;
  cudaSetDevice(s->device);
  const Grid& g = s->L[level].g;
  std::vector<uint8_t> pad(g.n);
  VF_TRY(cudaMemcpyAsync(pad.data(), s->L[level].mask, g.n, cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  const int nx1 = g.lx + 1, ny1 = g.ly + 1;
  for (int z = 0; z <= g.lz; ++z)
    for (int y = 0; y <= g.ly; ++y)
      for (int x = 0; x <= g.lx; ++x) out[x + (size_t)nx1 * (y + (size_t)ny1 * z)] = pad[g.idx(x, y, z)];
  return VF_OK;
}

int vf_learned_info(const vf_solver* s, int32_t* dims3, int32_t* level) {
  if (!s || !s->nn) return VF_ERR_STATE;
  int d[3];
  vf::nn_dims(s->nn, d);
  if (dims3) { dims3[0] = d[0]; dims3[1] = d[1]; dims3[2] = d[2]; }
  if (level) *level = s->nn_level;
  return VF_OK;
}

int vf_learned_input(vf_solver* s, const double* r_level, void* in_dev, float* scale_out, double* eref_out) {
  if (!s || !r_level || !in_dev) return VF_ERR_ARG;
  if (!s->nn || !s->have_material) { s->err = "learned stage: configure and set_material first"; return VF_ERR_STATE; }
  cudaSetDevice(s->device);
  Level& lL = s->L[s->nn_level];
  const size_t nref = 3 * (size_t)lL.g.nodes_ref();
  double* pad = lL.w64[3];
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, r_level, sizeof(double) * nref, cudaMemcpyHostToDevice, s->st));
  launch_pack_vec<double>(lL.g, s->d_ref_a, pad, lL.mask, s->st);
  vf::nn_make_input<double>(s->nn, lL.g, pad, nullptr, s->st);
  int d[3];
  vf::nn_dims(s->nn, d);
  VF_TRY(cudaMemcpyAsync(in_dev, vf::nn_input_buffer(s->nn), (size_t)d[0] * d[1] * d[2] * 16 * 2,
                         cudaMemcpyDeviceToDevice, s->st));
  float sc = 0.f;
  double er = 0.0;
  VF_TRY(cudaMemcpyAsync(&sc, vf::nn_scale_buffer(s->nn), sizeof(float), cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaMemcpyAsync(&er, s->d_nn_eref, sizeof(double), cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  VF_CHECK_LAUNCH();
  if (scale_out) *scale_out = sc;
  if (eref_out) *eref_out = er;
  return VF_OK;
}

int vf_learned_apply(vf_solver* s, const double* r_fine, double* e_fine) {
  if (!s || !r_fine || !e_fine) return VF_ERR_ARG;
  if (!s->nn || !vf::nn_has_weights(s->nn) || !s->have_material) {
    s->err = "learned stage: configure with weights and set_material first";
    return VF_ERR_STATE;
  }
  cudaSetDevice(s->device);
  Level& l0 = s->L[0];
  const size_t nref = 3 * (size_t)l0.g.nodes_ref();
  VF_TRY(cudaMemcpyAsync(s->d_ref_a, r_fine, sizeof(double) * nref, cudaMemcpyHostToDevice, s->st));
  double* r = s->k64[1];
  double* e = s->k64[2];
  launch_pack_vec<double>(l0.g, s->d_ref_a, r, l0.mask, s->st);
  const double* cur = r;
  for (int li = 0; li < s->nn_level; ++li) {
    Level& f = s->L[li];
    Level& c = s->L[li + 1];
    launch_restrict<double>(f.g, cur, c.g, c.mask, c.w64[3], nullptr, s->st);
    cur = c.w64[3];
  }
  Level& lL = s->L[s->nn_level];
  vf::nn_make_input<double>(s->nn, lL.g, cur, nullptr, s->st);
  vf::nn_forward(s->nn, nullptr, s->st);
  vf::nn_make_output<double>(s->nn, lL.g, lL.mask, lL.w64[0], nullptr, s->st);
  for (int li = s->nn_level; li >= 1; --li) {
    Level& c = s->L[li];
    Level& f = s->L[li - 1];
    double* target = (li == 1) ? e : f.w64[0];
    cudaMemsetAsync(target, 0, sizeof(double) * 3 * (size_t)f.g.n, s->st);
    launch_prolong_add<double>(c.g, c.w64[0], f.g, f.mask, target, nullptr, s->st);
  }
  launch_unpack_vec<double>(l0.g, e, s->d_ref_c, s->st);
  VF_CHECK_LAUNCH();
  VF_TRY(cudaMemcpyAsync(e_fine, s->d_ref_c, sizeof(double) * nref, cudaMemcpyDeviceToHost, s->st));
  VF_TRY(cudaStreamSynchronize(s->st));
  return VF_OK;
}

}  // extern "C"
