// Fine-level matrix-free hex8 operator family (and the rediscretized coarse
// levels of the reference hierarchy, which use the same element operator with
// a coarser modulus field):
//
//   y_n = sum over the 8 voxels e around node n of  E_e * Ke[a_e(n), :] u_e
//
// i.e. the reference's gather / (ue @ KE.T) * E / bincount scatter-add
// (core/multigrid.py:318-341, core/fea.py:374-386) recast as a node-centric
// 27-neighbour gather: every output is written by exactly one thread, with a
// fixed summation order, so results are deterministic and need no atomics.
//
// Ke is passed BY VALUE in the kernel parameter block (constant bank), so each
// solver can carry its own Poisson ratio, and an FMA reads its Ke operand
// straight from the constant bank.  A per-voxel Poisson ratio uses the exact
// split Ke(E, nu) = lam*K_lam + mu*K_mu.
//
// Epilogues fused into the same pass (one read of u, E, mask; one write):
//   EPI_APPLY   y = mask(K u)                [+ per-CTA partial of u.y]
//   EPI_SMOOTH  u' = u + w*mask(Minv*(b - mask(K u)))   (multigrid.py:399-401)
//   EPI_RESID   r = b - mask(K u)                        (multigrid.py:431)
#include "vf_common.cuh"
#include "vf_reduce.cuh"

namespace vf {

template <typename T>
struct KTab {
  T a[576];   // Ke(nu) at E = 1, or K_lam when LAME
  T b[576];   // K_mu when LAME (unused otherwise)
};

namespace {

constexpr int kOpThreads = 256;

template <typename T, bool LAME>
__device__ __forceinline__ void fine_Ku(const Grid& g, int x, int y, int z, const T* __restrict__ u,
                                        const T* __restrict__ E, const T* __restrict__ MU,
                                        const KTab<T>& K, T& a0, T& a1, T& a2) {
  a0 = 0; a1 = 0; a2 = 0;
#pragma unroll
  for (int ez = -1; ez <= 0; ++ez)
#pragma unroll
    for (int ey = -1; ey <= 0; ++ey)
#pragma unroll
      for (int ex = -1; ex <= 0; ++ex) {
        const int ka = corner_k(-ex, -ey, -ez);
        const int q = g.idx(x + ex, y + ey, z + ez);
        const T Ee = __ldg(E + q);
        const T Me = LAME ? __ldg(MU + q) : (T)0;
        T t0 = 0, t1 = 0, t2 = 0, s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
        for (int bz = 0; bz < 2; ++bz)
#pragma unroll
          for (int by = 0; by < 2; ++by)
#pragma unroll
            for (int bx = 0; bx < 2; ++bx) {
              const int kb = corner_k(bx, by, bz);
              const int m = g.idx(x + ex + bx, y + ey + by, z + ez + bz);
              const T u0 = __ldg(u + 3 * m), u1 = __ldg(u + 3 * m + 1), u2 = __ldg(u + 3 * m + 2);
              const int r0 = (3 * ka) * 24 + 3 * kb, r1 = r0 + 24, r2 = r0 + 48;
              t0 += K.a[r0] * u0 + K.a[r0 + 1] * u1 + K.a[r0 + 2] * u2;
              t1 += K.a[r1] * u0 + K.a[r1 + 1] * u1 + K.a[r1 + 2] * u2;
              t2 += K.a[r2] * u0 + K.a[r2 + 1] * u1 + K.a[r2 + 2] * u2;
              if (LAME) {
                s0 += K.b[r0] * u0 + K.b[r0 + 1] * u1 + K.b[r0 + 2] * u2;
                s1 += K.b[r1] * u0 + K.b[r1 + 1] * u1 + K.b[r1 + 2] * u2;
                s2 += K.b[r2] * u0 + K.b[r2 + 1] * u1 + K.b[r2 + 2] * u2;
              }
            }
        a0 += Ee * t0; a1 += Ee * t1; a2 += Ee * t2;
        if (LAME) { a0 += Me * s0; a1 += Me * s1; a2 += Me * s2; }
      }
}

template <typename T, bool LAME, int EPI>
__global__ void __launch_bounds__(kOpThreads) k_fine_op(Grid g, OpArgs a, const KTab<T> K) {
  KrylovState* ks = a.ks;
  if (ks && ks->done) return;
  const T* __restrict__ u = (const T*)a.u;
  T* __restrict__ out = (T*)a.out;
  const T* __restrict__ b = (const T*)a.b;
  const T* __restrict__ minv = (const T*)a.minv;
  const T* __restrict__ E = (const T*)a.E;
  const T* __restrict__ MU = (const T*)a.mu;
  const uint8_t* __restrict__ mask = a.mask;
  const T w = a.omega_dev ? (T)(*a.omega_dev) : (T)a.omega;
  const int nx1 = g.lx + 1, ny1 = g.ly + 1;
  const int nint = nx1 * ny1 * (g.lz + 1);
  double dot = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int x = t % nx1;
    const int r = t / nx1;
    const int y = r % ny1;
    const int z = r / ny1;
    const int p = g.idx(x, y, z);
    T k0, k1, k2;
    fine_Ku<T, LAME>(g, x, y, z, u, E, MU, K, k0, k1, k2);
    const uint8_t m = mask[p];
    k0 = (m & 1) ? k0 : (T)0;
    k1 = (m & 2) ? k1 : (T)0;
    k2 = (m & 4) ? k2 : (T)0;
    const long long p3 = 3 * (long long)p;
    if (EPI == EPI_APPLY) {
      out[p3] = k0; out[p3 + 1] = k1; out[p3 + 2] = k2;
      if (a.dot_partials)
        dot += (double)u[p3] * (double)k0 + (double)u[p3 + 1] * (double)k1 + (double)u[p3 + 2] * (double)k2;
    } else if (EPI == EPI_SMOOTH) {
      const T r0 = b[p3] - k0, r1 = b[p3 + 1] - k1, r2 = b[p3 + 2] - k2;
      out[p3] = u[p3] + ((m & 1) ? w * (minv[p3] * r0) : (T)0);
      out[p3 + 1] = u[p3 + 1] + ((m & 2) ? w * (minv[p3 + 1] * r1) : (T)0);
      out[p3 + 2] = u[p3 + 2] + ((m & 4) ? w * (minv[p3 + 2] * r2) : (T)0);
    } else {
      out[p3] = b[p3] - k0; out[p3 + 1] = b[p3 + 1] - k1; out[p3 + 2] = b[p3 + 2] - k2;
    }
  }
  if (EPI == EPI_APPLY && a.dot_partials && ks) reduce_and_finalize(dot, a.dot_partials, ks, a.dot_slot, nullptr);
}

template <typename T>
KTab<T> make_tab(const double* tab, bool lame) {
  KTab<T> K;
  for (int i = 0; i < 576; ++i) {
    K.a[i] = (T)(lame ? tab[576 + i] : tab[i]);
    K.b[i] = (T)(lame ? tab[1152 + i] : 0.0);
  }
  return K;
}

}  // namespace

template <typename T>
int fine_op_grid_blocks(const Grid& g) {
  long long nint = (long long)(g.lx + 1) * (g.ly + 1) * (g.lz + 1);
  long long b = (nint + kOpThreads - 1) / kOpThreads;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

template <typename T>
void launch_fine_op(const Grid& g, int epi, const OpArgs& a, cudaStream_t st) {
  const bool lame = a.mu != nullptr;
  const KTab<T> K = make_tab<T>(a.ke_tab, lame);
  const int blocks = fine_op_grid_blocks<T>(g);
#define VF_L(L, EP) launch_k(k_fine_op<T, L, EP>, blocks, kOpThreads, 0, st, g, a, K)
  if (lame) {
    if (epi == EPI_APPLY) VF_L(true, EPI_APPLY);
    else if (epi == EPI_SMOOTH) VF_L(true, EPI_SMOOTH);
    else VF_L(true, EPI_RESID);
  } else {
    if (epi == EPI_APPLY) VF_L(false, EPI_APPLY);
    else if (epi == EPI_SMOOTH) VF_L(false, EPI_SMOOTH);
    else VF_L(false, EPI_RESID);
  }
#undef VF_L
}

template void launch_fine_op<double>(const Grid&, int, const OpArgs&, cudaStream_t);
template void launch_fine_op<float>(const Grid&, int, const OpArgs&, cudaStream_t);
template int fine_op_grid_blocks<double>(const Grid&);
template int fine_op_grid_blocks<float>(const Grid&);

}  // namespace vf
