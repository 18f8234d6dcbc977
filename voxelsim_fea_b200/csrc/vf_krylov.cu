// PCG vector kernels (core/multigrid.py:497-546): each is one memory pass
// fused with its FP64 reduction; the scalar recurrences (alpha, beta, ratio,
// convergence / stall / max_it tests) finalize on the device (vf_reduce.cuh).
// Vectors are walked over the whole padded array: ghost entries are zero, so
// they add nothing and the walk stays contiguous.
#include "vf_common.cuh"
#include "vf_reduce.cuh"

namespace vf {

namespace {

// 16-byte vectors: padded vectors hold 3 * px * py * pz values with px a
// multiple of 4, so their length is a multiple of 12 (and of 4 and 2).
template <typename T> struct V16;
template <> struct V16<float> {
  using V = float4;
  static constexpr int W = 4;
  __device__ __forceinline__ static double dot(V a, V b) {
    return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
  }
  __device__ __forceinline__ static V axpy(float s, V x, V y) {   // y + s x
    return make_float4(fmaf(s, x.x, y.x), fmaf(s, x.y, y.y), fmaf(s, x.z, y.z), fmaf(s, x.w, y.w));
  }
};
template <> struct V16<double> {
  using V = double2;
  static constexpr int W = 2;
  __device__ __forceinline__ static double dot(V a, V b) { return a.x * b.x + a.y * b.y; }
  __device__ __forceinline__ static V axpy(double s, V x, V y) { return make_double2(fma(s, x.x, y.x), fma(s, x.y, y.y)); }
};

template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_dot(long long n3, const T* __restrict__ a, const T* __restrict__ b,
                                                     double* partials, KrylovState* ks, int slot) {
  if (ks->done && slot != SLOT_FNORM && slot != SLOT_RZ_INIT && slot != SLOT_OUTER && slot != SLOT_PLAIN) return;
  using H = V16<T>;
  using V = typename H::V;
  const long long nv = n3 / H::W;
  const V* av = reinterpret_cast<const V*>(a);
  const V* bv = reinterpret_cast<const V*>(b);
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x)
    s += H::dot(__ldg(av + i), __ldg(bv + i));
  reduce_and_finalize(s, partials, ks, slot, nullptr);
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_cg_update(long long n3, T* __restrict__ x, const T* __restrict__ p,
                                                           T* __restrict__ r, const T* __restrict__ Ap,
                                                           double* partials, KrylovState* ks, double* hist) {
  if (ks->done) return;
  using H = V16<T>;
  using V = typename H::V;
  const T alpha = (T)ks->alpha;
  const long long nv = n3 / H::W;
  V* xv = reinterpret_cast<V*>(x);
  V* rv = reinterpret_cast<V*>(r);
  const V* pv = reinterpret_cast<const V*>(p);
  const V* av = reinterpret_cast<const V*>(Ap);
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const V pi = __ldg(pv + i), ai = __ldg(av + i);
    xv[i] = H::axpy(alpha, pi, xv[i]);
    const V ri = H::axpy(-alpha, ai, rv[i]);
    rv[i] = ri;
    s += H::dot(ri, ri);
  }
  reduce_and_finalize(s, partials, ks, SLOT_RR, hist);
}

// (r.z, z.Ap) in one pass -> flexible-CG beta
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_dot_fcg(long long n3, const T* __restrict__ r, const T* __restrict__ z,
                                                         const T* __restrict__ Ap, double* partials, KrylovState* ks) {
  if (ks->done) return;
  using H = V16<T>;
  using V = typename H::V;
  const long long nv = n3 / H::W;
  const V* rv = reinterpret_cast<const V*>(r);
  const V* zv = reinterpret_cast<const V*>(z);
  const V* av = reinterpret_cast<const V*>(Ap);
  double s1 = 0.0, s2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
    const V zz = __ldg(zv + i);
    s1 += H::dot(__ldg(rv + i), zz);
    s2 += H::dot(zz, __ldg(av + i));
  }
  reduce2_and_finalize(s1, s2, partials, ks, SLOT_FCG);
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_p_update(long long n3, T* __restrict__ p, const T* __restrict__ z,
                                                          const KrylovState* ks) {
  if (ks->done) return;
  using H = V16<T>;
  using V = typename H::V;
  const bool restart = ks->restart != 0;
  const T beta = restart ? (T)0 : (T)ks->beta;
  const long long nv = n3 / H::W;
  V* pv = reinterpret_cast<V*>(p);
  const V* zv = reinterpret_cast<const V*>(z);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x)
    pv[i] = restart ? __ldg(zv + i) : H::axpy(beta, pv[i], __ldg(zv + i));
}

// FP64 outer PCG around an FP32 preconditioner: the FP64 recurrences of x,
// r, p keep the Krylov space of the FP64 solve; the V-cycle reads an FP32
// copy of r (written by the update pass) and returns z in FP32, which the
// direction update widens.  x += alpha p is deferred to the direction update
// (which reads p anyway), so p is read once per iteration, not twice.  Four
// values per thread step (n3 is a multiple of 12): two double2 and one
// float4 access per vector.
__global__ void __launch_bounds__(kVecThreads) k_cg_update_split(long long n3, double* __restrict__ r,
                                                                 const double* __restrict__ Ap, float* __restrict__ r32,
                                                                 double* partials, KrylovState* ks, double* hist) {
  if (ks->done) return;
  const double alpha = ks->alpha;
  const long long n4 = n3 / 4;
  double2* rv = reinterpret_cast<double2*>(r);
  const double2* av = reinterpret_cast<const double2*>(Ap);
  float4* r4 = reinterpret_cast<float4*>(r32);
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const double2 a0 = __ldg(av + 2 * i), a1 = __ldg(av + 2 * i + 1);
    double2 q0 = rv[2 * i], q1 = rv[2 * i + 1];
    q0.x = fma(-alpha, a0.x, q0.x); q0.y = fma(-alpha, a0.y, q0.y);
    q1.x = fma(-alpha, a1.x, q1.x); q1.y = fma(-alpha, a1.y, q1.y);
    rv[2 * i] = q0; rv[2 * i + 1] = q1;
    r4[i] = make_float4((float)q0.x, (float)q0.y, (float)q1.x, (float)q1.y);
    s += q0.x * q0.x + q0.y * q0.y + q1.x * q1.x + q1.y * q1.y;
  }
  reduce_and_finalize(s, partials, ks, SLOT_RR, hist);
}

// x += alpha p (the iteration's deferred solution update), then p = z + beta p
// (p FP64, z FP32).  The x update runs once per completed iteration -- also
// the one whose residual test ended the solve, when p stays -- tracked by
// ks->x_it, which the last CTA advances.
__global__ void __launch_bounds__(kVecThreads) k_p_update_split(long long n3, double* __restrict__ x,
                                                                double* __restrict__ p, const float* __restrict__ z,
                                                                KrylovState* ks) {
  const int it = ks->it;
  const bool do_x = it > ks->x_it;
  const bool do_p = !ks->done;
  if (!do_x && !do_p) return;
  const double alpha = do_x ? ks->alpha : 0.0;
  const bool restart = ks->restart != 0;
  const double beta = restart ? 0.0 : ks->beta;
  const long long n4 = n3 / 4;
  double2* xv = reinterpret_cast<double2*>(x);
  double2* pv = reinterpret_cast<double2*>(p);
  const float4* zv = reinterpret_cast<const float4*>(z);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    double2 p0 = pv[2 * i], p1 = pv[2 * i + 1];
    if (do_x) {
      double2 x0 = xv[2 * i], x1 = xv[2 * i + 1];
      x0.x = fma(alpha, p0.x, x0.x); x0.y = fma(alpha, p0.y, x0.y);
      x1.x = fma(alpha, p1.x, x1.x); x1.y = fma(alpha, p1.y, x1.y);
      xv[2 * i] = x0; xv[2 * i + 1] = x1;
    }
    if (do_p) {
      const float4 zz = __ldg(zv + i);
      p0.x = fma(beta, p0.x, (double)zz.x); p0.y = fma(beta, p0.y, (double)zz.y);
      p1.x = fma(beta, p1.x, (double)zz.z); p1.y = fma(beta, p1.y, (double)zz.w);
      pv[2 * i] = p0; pv[2 * i + 1] = p1;
    }
  }
  if (do_x) {   // last CTA: this iteration's alpha p is in x
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned prev = atomicAdd(&ks->counter[11], 1u);
      if (prev == gridDim.x - 1) {
        ks->x_it = it;
        ks->counter[11] = 0u;
        __threadfence();
      }
    }
  }
}

// (r.z, z.Ap) with r, z FP32 and Ap FP64 -> flexible-CG beta
__global__ void __launch_bounds__(kVecThreads) k_dot_fcg_split(long long n3, const float* __restrict__ r,
                                                               const float* __restrict__ z,
                                                               const double* __restrict__ Ap, double* partials,
                                                               KrylovState* ks) {
  if (ks->done) return;
  const long long n4 = n3 / 4;
  const float4* rv = reinterpret_cast<const float4*>(r);
  const float4* zv = reinterpret_cast<const float4*>(z);
  const double2* av = reinterpret_cast<const double2*>(Ap);
  double s1 = 0.0, s2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 rr = __ldg(rv + i), zz = __ldg(zv + i);
    const double2 a0 = __ldg(av + 2 * i), a1 = __ldg(av + 2 * i + 1);
    s1 += (double)rr.x * zz.x + (double)rr.y * zz.y + (double)rr.z * zz.z + (double)rr.w * zz.w;
    s2 += (double)zz.x * a0.x + (double)zz.y * a0.y + (double)zz.z * a1.x + (double)zz.w * a1.y;
  }
  reduce2_and_finalize(s1, s2, partials, ks, SLOT_FCG);
}

// y = s x (FP64; y may be x)
__global__ void k_scale64(long long n3, const double* x, double* y, double sc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    y[i] = sc * x[i];
}

template <typename T>
__global__ void k_jacobi_precond(int n, const T* __restrict__ r, const T* __restrict__ minv,
                                 const uint8_t* __restrict__ mask, T* __restrict__ z, const KrylovState* ks) {
  if (ks && ks->done) return;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint8_t m = mask[p];
    const long long p3 = 3 * (long long)p;
    z[p3] = (m & 1) ? minv[p3] * r[p3] : (T)0;
    z[p3 + 1] = (m & 2) ? minv[p3 + 1] * r[p3 + 1] : (T)0;
    z[p3 + 2] = (m & 4) ? minv[p3 + 2] * r[p3 + 2] : (T)0;
  }
}

template <typename T>
__global__ void k_copy(long long n3, const T* __restrict__ s, T* __restrict__ d, const KrylovState* ks) {
  if (ks && ks->done) return;
  const long long n16 = n3 * (long long)sizeof(T) / 16;   // 16-byte chunks
  const float4* sv = reinterpret_cast<const float4*>(s);
  float4* dv = reinterpret_cast<float4*>(d);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += (long long)gridDim.x * blockDim.x)
    dv[i] = __ldg(sv + i);
}

// Mixed precision: r32 = r64 / ||r64|| (inner solves see a unit right-hand
// side, keeping FP32 far from under/overflow), remember the scale.
__global__ void k_ir_prepare(long long n3, const double* __restrict__ r64, float* __restrict__ r32, KrylovState* ks) {
  const double s = sqrt(ks->rr);
  const double inv = s > 0.0 ? 1.0 / s : 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    r32[i] = (float)(r64[i] * inv);
  if (blockIdx.x == 0 && threadIdx.x == 0) ks->scale = s;
}

__global__ void k_ir_accumulate(long long n3, double* __restrict__ x64, const float* __restrict__ d32,
                                const KrylovState* ks) {
  const double s = ks->scale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    x64[i] += s * (double)d32[i];
}

// z += gamma c, gamma = (c.r1) / (c.A c): the A-norm-optimal step along the
// learned correction c (0 when c.A c is not positive)
template <typename T>
__global__ void k_axpy_gamma(long long n3, T* __restrict__ z, const T* __restrict__ c, const KrylovState* ks,
                             const int* skip) {
  if (skip && *skip) return;
  const double den = ks->gden;
  const T g = (den > 0.0) ? (T)(ks->gnum / den) : (T)0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    z[i] += g * c[i];
}

// y -= x (no state)
template <typename T>
__global__ void k_sub_inplace(long long n3, T* __restrict__ y, const T* __restrict__ x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    y[i] -= x[i];
}

// r32 = r64 / scale with the scale fixed for the whole mixed solve
__global__ void k_ir_replace(long long n3, const double* __restrict__ r64, float* __restrict__ r32,
                             const KrylovState* ks) {
  const double s = ks->scale;
  const double inv = s > 0.0 ? 1.0 / s : 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    r32[i] = (float)(r64[i] * inv);
}

__global__ void k_sub_from(long long n3, const double* __restrict__ f, double* __restrict__ r) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    r[i] = f[i] - r[i];
}

// Power iteration on D^-1 A: x_0 = deterministic pseudo-random free vector.
template <typename T>
__global__ void k_power_init(long long n, T* __restrict__ x, const uint8_t* __restrict__ mask) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const uint8_t m = mask[p];
    for (int c = 0; c < 3; ++c) {
      unsigned long long h = (unsigned long long)(3 * p + c) * 0x9E3779B97F4A7C15ULL;
      h ^= h >> 31; h *= 0xBF58476D1CE4E5B9ULL; h ^= h >> 29;
      const double v = (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
      x[3 * p + c] = ((m >> c) & 1) ? (T)v : (T)0;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_power_scale(long long n, T* __restrict__ y,
                                                             const T* __restrict__ minv, double* partials,
                                                             KrylovState* ks) {
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const T v = y[i] * minv[i];
    y[i] = v;
    s += (double)v * (double)v;
  }
  reduce_and_finalize(s, partials, ks, SLOT_PLAIN, nullptr);
}

template <typename T>
__global__ void k_power_normalize(long long n, const T* __restrict__ y, T* __restrict__ x, const KrylovState* ks) {
  const T inv = ks->rr > 0.0 ? (T)(1.0 / sqrt(ks->rr)) : (T)0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = y[i] * inv;
}

// omega_l = omega_rel * 2 / (safety * lambda), lambda = ||D^-1 A x|| for unit x.
__global__ void k_power_omega(const KrylovState* ks, double omega_rel, double safety, double* omega_out,
                              double* lambda_out) {
  const double lam = sqrt(ks->rr) * safety;
  *lambda_out = lam;
  *omega_out = lam > 0.0 ? omega_rel * 2.0 / lam : omega_rel;
}

// Chebyshev smoothing steps per level (three-term recurrence on the interval
// [beta / ratio, beta] of D^-1 A_l, beta = the padded lambda_max estimate):
// step 0: x += (1/theta) Minv r; step k: d_k = c1 d_(k-1) + c2 Minv r,
// x += d_k with rho_k = 1 / (2 sigma - rho_(k-1)), c1 = rho_k rho_(k-1),
// c2 = 2 rho_k / delta.  coef[(l * 2 + k) * 2 + {0, 1}] = {c1, c2}.
__global__ void k_cheb_coefs(const double* lambda, int nl, int ratio, double* coef) {
  const int l = threadIdx.x;
  if (l >= nl) return;
  const double beta = lambda[l];
  double* c = coef + 4 * l;
  if (!(beta > 0.0)) {   // no free DOF on the level: leave it unchanged
    c[0] = c[1] = c[2] = c[3] = 0.0;
    return;
  }
  const double alpha = beta / ratio;
  const double theta = 0.5 * (beta + alpha), delta = 0.5 * (beta - alpha), sigma = theta / delta;
  const double rho0 = 1.0 / sigma;
  const double rho1 = 1.0 / (2.0 * sigma - rho0);
  c[0] = 0.0;
  c[1] = 1.0 / theta;
  c[2] = rho1 * rho0;
  c[3] = 2.0 * rho1 / delta;
}

}  // namespace

void launch_cheb_coefs(const double* lambda, int nl, int ratio, double* coef, cudaStream_t st) {
  launch_k(k_cheb_coefs, 1, 32, 0, st, lambda, nl, ratio, coef);
}

template <typename T>
void launch_power_init(const Grid& g, T* x, const uint8_t* mask, cudaStream_t st) {
  launch_k(k_power_init<T>, kVecBlocks, kVecThreads, 0, st, (long long)g.n, x, mask);
}
template <typename T>
void launch_power_scale(const Grid& g, T* y, const T* minv3, double* partials, KrylovState* ks, cudaStream_t st) {
  launch_k(k_power_scale<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, y, minv3, partials, ks);
}
template <typename T>
void launch_power_normalize(const Grid& g, const T* y, T* x, const KrylovState* ks, cudaStream_t st) {
  launch_k(k_power_normalize<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, y, x, ks);
}
#define VF_INST_POWER(T)                                                                                   \
  template void launch_power_init<T>(const Grid&, T*, const uint8_t*, cudaStream_t);                       \
  template void launch_power_scale<T>(const Grid&, T*, const T*, double*, KrylovState*, cudaStream_t);     \
  template void launch_power_normalize<T>(const Grid&, const T*, T*, const KrylovState*, cudaStream_t);
VF_INST_POWER(double)
VF_INST_POWER(float)
#undef VF_INST_POWER
void launch_power_omega(const KrylovState* ks, double omega_rel, double safety, double* omega_out,
                        double* lambda_out, cudaStream_t st) {
  launch_k(k_power_omega, 1, 1, 0, st, ks, omega_rel, safety, omega_out, lambda_out);
}

template <typename T>
void launch_dot(const Grid& g, const T* a, const T* b, double* partials, KrylovState* ks, int slot, cudaStream_t st) {
  launch_k(k_dot<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, a, b, partials, ks, slot);
}
template <typename T>
void launch_cg_update(const Grid& g, T* x, const T* p, T* r, const T* Ap, double* partials, KrylovState* ks,
                      double* hist, cudaStream_t st) {
  launch_k(k_cg_update<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, x, p, r, Ap, partials, ks, hist);
}
template <typename T>
void launch_p_update(const Grid& g, T* p, const T* z, KrylovState* ks, cudaStream_t st) {
  launch_k(k_p_update<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, p, z, ks);
}
template <typename T>
void launch_jacobi_precond(const Grid& g, const T* r, const T* minv3, const uint8_t* mask, T* z,
                           const KrylovState* ks, cudaStream_t st) {
  launch_k(k_jacobi_precond<T>, kVecBlocks, kVecThreads, 0, st, g.n, r, minv3, mask, z, ks);
}
template <typename T>
void launch_copy_vec(const Grid& g, const T* src, T* dst, const KrylovState* ks, cudaStream_t st) {
  launch_k(k_copy<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, src, dst, ks);
}
void launch_norm2_f64(const Grid& g, const double* v, double* partials, KrylovState* ks, int slot, cudaStream_t st) {
  launch_k(k_dot<double>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, v, v, partials, ks, slot);
}
void launch_ir_prepare(const Grid& g, const double* r64, float* r32, KrylovState* ks, cudaStream_t st) {
  launch_k(k_ir_prepare, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, r64, r32, ks);
}
void launch_ir_accumulate(const Grid& g, double* x64, const float* d32, const KrylovState* ks, cudaStream_t st) {
  launch_k(k_ir_accumulate, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, x64, d32, ks);
}
void launch_ir_replace(const Grid& g, const double* r64, float* r32, const KrylovState* ks, cudaStream_t st) {
  launch_k(k_ir_replace, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, r64, r32, ks);
}
template <typename T>
void launch_axpy_gamma(const Grid& g, T* z, const T* c, const KrylovState* ks, const int* skip, cudaStream_t st) {
  launch_k(k_axpy_gamma<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, z, c, ks, skip);
}
template <typename T>
void launch_sub_inplace(const Grid& g, T* y, const T* x, cudaStream_t st) {
  launch_k(k_sub_inplace<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, y, x);
}
template void launch_sub_inplace<float>(const Grid&, float*, const float*, cudaStream_t);
template void launch_sub_inplace<double>(const Grid&, double*, const double*, cudaStream_t);
template void launch_axpy_gamma<float>(const Grid&, float*, const float*, const KrylovState*, const int*, cudaStream_t);
template void launch_axpy_gamma<double>(const Grid&, double*, const double*, const KrylovState*, const int*,
                                        cudaStream_t);
void launch_sub_from(const Grid& g, const double* f, double* r, cudaStream_t st) {
  launch_k(k_sub_from, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, f, r);
}

void launch_cg_update_split(const Grid& g, double* r, const double* Ap, float* r32, double* partials,
                            KrylovState* ks, double* hist, cudaStream_t st) {
  launch_k(k_cg_update_split, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, r, Ap, r32, partials, ks, hist);
}
void launch_p_update_split(const Grid& g, double* x, double* p, const float* z, KrylovState* ks, cudaStream_t st) {
  launch_k(k_p_update_split, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, x, p, z, ks);
}
void launch_dot_fcg_split(const Grid& g, const float* r, const float* z, const double* Ap, double* partials,
                          KrylovState* ks, cudaStream_t st) {
  launch_k(k_dot_fcg_split, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, r, z, Ap, partials, ks);
}
void launch_scale64(const Grid& g, const double* x, double* y, double sc, cudaStream_t st) {
  launch_k(k_scale64, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, x, y, sc);
}

template <typename T>
void launch_dot_fcg(const Grid& g, const T* r, const T* z, const T* Ap, double* partials, KrylovState* ks,
                    cudaStream_t st) {
  launch_k(k_dot_fcg<T>, kVecBlocks, kVecThreads, 0, st, 3LL * g.n, r, z, Ap, partials, ks);
}

#define VF_INST(T)                                                                                            \
  template void launch_dot<T>(const Grid&, const T*, const T*, double*, KrylovState*, int, cudaStream_t);    \
  template void launch_cg_update<T>(const Grid&, T*, const T*, T*, const T*, double*, KrylovState*, double*, cudaStream_t); \
  template void launch_p_update<T>(const Grid&, T*, const T*, KrylovState*, cudaStream_t);                   \
  template void launch_dot_fcg<T>(const Grid&, const T*, const T*, const T*, double*, KrylovState*, cudaStream_t); \
  template void launch_jacobi_precond<T>(const Grid&, const T*, const T*, const uint8_t*, T*, const KrylovState*, cudaStream_t); \
  template void launch_copy_vec<T>(const Grid&, const T*, T*, const KrylovState*, cudaStream_t);
VF_INST(double)
VF_INST(float)
#undef VF_INST

}  // namespace vf
