// Layout conversion (reference arrays <-> padded device layout) and the
// per-level set-up kernels: Dirichlet-mask injection (core/multigrid.py:255-278),
// 2x2x2 modulus averaging (multigrid.py:281-292) and the Jacobi inverse
// diagonal (multigrid.py:300-304).  All grid-stride, memory-bound, one pass.
#include <atomic>

#include "vf_common.cuh"

namespace vf {

static std::atomic<unsigned long long> g_direct{0};

void count_launch(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return;
  g_direct.fetch_add(1, std::memory_order_relaxed);
}

unsigned long long direct_launches() { return g_direct.load(); }

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148 * 64) b = 148 * 64;
  if (b < 1) b = 1;
  return (int)b;
}

__device__ __forceinline__ void decode(const Grid& g, int p, int& x, int& y, int& z) {
  x = p % g.px - 1;
  int t = p / g.px;
  y = t % g.py - 1;
  z = t / g.py - 1;
}

template <typename T>
__global__ void k_pack_vec(Grid g, const double* __restrict__ ref, T* __restrict__ pad,
                           const uint8_t* __restrict__ mask) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    T v0 = 0, v1 = 0, v2 = 0;
    if (x >= 0 && x <= g.lx && y >= 0 && y <= g.ly && z >= 0 && z <= g.lz) {
      long long r = x + (long long)(g.lx + 1) * (y + (long long)(g.ly + 1) * z);
      uint8_t m = mask ? mask[p] : kFreeAll;
      v0 = (m & 1) ? (T)ref[3 * r + 0] : (T)0;
      v1 = (m & 2) ? (T)ref[3 * r + 1] : (T)0;
      v2 = (m & 4) ? (T)ref[3 * r + 2] : (T)0;
    }
    pad[3 * (long long)p + 0] = v0;
    pad[3 * (long long)p + 1] = v1;
    pad[3 * (long long)p + 2] = v2;
  }
}

template <typename T>
__global__ void k_unpack_vec(Grid g, const T* __restrict__ pad, double* __restrict__ ref) {
  const int nref = g.nodes_ref();
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nref; r += gridDim.x * blockDim.x) {
    int x = r % (g.lx + 1);
    int t = r / (g.lx + 1);
    int y = t % (g.ly + 1);
    int z = t / (g.ly + 1);
    long long p = g.idx(x, y, z);
    ref[3 * (long long)r + 0] = (double)pad[3 * p + 0];
    ref[3 * (long long)r + 1] = (double)pad[3 * p + 1];
    ref[3 * (long long)r + 2] = (double)pad[3 * p + 2];
  }
}

template <typename T>
__global__ void k_pack_elem(Grid g, const double* __restrict__ ref, T* __restrict__ pad,
                            const uint8_t* __restrict__ active, double scale) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    T v = 0;
    if (x >= 0 && x < g.lx && y >= 0 && y < g.ly && z >= 0 && z < g.lz) {
      long long e = ((long long)x * g.ly + y) * g.lz + z;
      if (!active || active[e]) v = (T)(ref[e] * scale);
    }
    pad[p] = v;
  }
}

template <typename T>
__global__ void k_pack_lame(Grid g, const double* __restrict__ E, const double* __restrict__ nu_elem,
                            double nu, const uint8_t* __restrict__ active, double scale,
                            T* __restrict__ lam, T* __restrict__ mu) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    T l = 0, m = 0;
    if (x >= 0 && x < g.lx && y >= 0 && y < g.ly && z >= 0 && z < g.lz) {
      long long e = ((long long)x * g.ly + y) * g.lz + z;
      if (!active || active[e]) {
        double n = nu_elem ? nu_elem[e] : nu;
        double Ee = E[e] * scale;
        l = (T)(Ee * n / ((1.0 + n) * (1.0 - 2.0 * n)));
        m = (T)(Ee / (2.0 * (1.0 + n)));
      }
    }
    lam[p] = l;
    mu[p] = m;
  }
}

__global__ void k_pack_mask(Grid g, const uint8_t* __restrict__ ref, uint8_t* __restrict__ pad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    uint8_t m = 0;
    if (x >= 0 && x <= g.lx && y >= 0 && y <= g.ly && z >= 0 && z <= g.lz)
      m = ref ? ref[x + (long long)(g.lx + 1) * (y + (long long)(g.ly + 1) * z)] : kFreeAll;
    pad[p] = m;
  }
}

// Coarse node J keeps the free bits of the collocated fine node 2J
// (core/multigrid.py:264-277).
__global__ void k_inject_mask(Grid f, const uint8_t* __restrict__ fm, Grid c, uint8_t* __restrict__ cm) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < c.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(c, p, x, y, z);
    uint8_t m = 0;
    if (x >= 0 && x <= c.lx && y >= 0 && y <= c.ly && z >= 0 && z <= c.lz) m = fm[f.idx(2 * x, 2 * y, 2 * z)];
    cm[p] = m;
  }
}

// Coarse modulus = 2 * mean of the 8 children (the children already carry
// the 2^l factor of their level, so this is mean(E_unscaled) * 2^(l+1),
// core/multigrid.py:290-292).
template <typename T>
__global__ void k_coarsen_E(Grid f, const T* __restrict__ Ef, Grid c, T* __restrict__ Ec) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < c.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(c, p, x, y, z);
    T v = 0;
    if (x >= 0 && x < c.lx && y >= 0 && y < c.ly && z >= 0 && z < c.lz) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int i = 0; i < 2; ++i) s += (double)Ef[f.idx(2 * x + i, 2 * y + j, 2 * z + k)];
      v = (T)(s * 0.25);
    }
    Ec[p] = v;
  }
}

template <typename T>
__global__ void k_scale(T* v, long long n, double s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = (T)((double)v[i] * s);
}

// d_n = sum over the 8 elements around n of diag(K_e) (uniform over the 24
// local DOFs for the isotropic unit cube); zero -> 1 (multigrid.py:300-304).
template <typename T>
__global__ void k_inv_diag_fine(Grid g, const T* __restrict__ E, const T* __restrict__ mu, double dL,
                                double dM, T* __restrict__ minv3) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    if (!(x >= 0 && x <= g.lx && y >= 0 && y <= g.ly && z >= 0 && z <= g.lz)) {
      minv3[3 * (long long)p] = 0; minv3[3 * (long long)p + 1] = 0; minv3[3 * (long long)p + 2] = 0;
      continue;
    }
    double d = 0.0;
#pragma unroll
    for (int ez = -1; ez <= 0; ++ez)
#pragma unroll
      for (int ey = -1; ey <= 0; ++ey)
#pragma unroll
        for (int ex = -1; ex <= 0; ++ex) {
          int q = g.idx(x + ex, y + ey, z + ez);
          d += (double)E[q] * dL;
          if (mu) d += (double)mu[q] * dM;
        }
    double m = (d == 0.0) ? 1.0 : 1.0 / d;
    minv3[3 * (long long)p] = (T)m;
    minv3[3 * (long long)p + 1] = (T)m;
    minv3[3 * (long long)p + 2] = (T)m;
  }
}

template <typename Ts, typename Td>
__global__ void k_convert(const Ts* __restrict__ s, Td* __restrict__ d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d[i] = (Td)s[i];
}

// Jacobi method: a node is part of the system iff an active element touches it
// (core/fea.py:271-279); unused nodes become non-free.  active_pad holds the
// per-element active flag in the padded element layout.
__global__ void k_used_mask(Grid g, const uint8_t* __restrict__ active_pad, uint8_t* __restrict__ mask) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    if (!(x >= 0 && x <= g.lx && y >= 0 && y <= g.ly && z >= 0 && z <= g.lz)) continue;
    int used = 0;
#pragma unroll
    for (int ez = -1; ez <= 0; ++ez)
#pragma unroll
      for (int ey = -1; ey <= 0; ++ey)
#pragma unroll
        for (int ex = -1; ex <= 0; ++ex) used |= active_pad[g.idx(x + ex, y + ey, z + ez)];
    if (!used) mask[p] = 0;
  }
}

__global__ void k_pack_active(Grid g, const uint8_t* __restrict__ ref, uint8_t* __restrict__ pad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    uint8_t v = 0;
    if (x >= 0 && x < g.lx && y >= 0 && y < g.ly && z >= 0 && z < g.lz)
      v = ref ? (ref[((long long)x * g.ly + y) * g.lz + z] != 0) : 1;
    pad[p] = v;
  }
}

}  // namespace

template <typename T>
void launch_pack_vec(const Grid& g, const double* ref, T* pad, const uint8_t* mask, cudaStream_t st) {
  launch_k(k_pack_vec<T>, blocks_for(g.n), kThreads, 0, st, g, ref, pad, mask);
}
template <typename T>
void launch_unpack_vec(const Grid& g, const T* pad, double* ref, cudaStream_t st) {
  launch_k(k_unpack_vec<T>, blocks_for(g.nodes_ref()), kThreads, 0, st, g, pad, ref);
}
template <typename T>
void launch_pack_elem(const Grid& g, const double* ref, T* pad, const uint8_t* active, double scale, cudaStream_t st) {
  launch_k(k_pack_elem<T>, blocks_for(g.n), kThreads, 0, st, g, ref, pad, active, scale);
}
template <typename T>
void launch_pack_lame(const Grid& g, const double* E, const double* nu_elem, double nu, const uint8_t* active,
                      double scale, T* lam, T* mu, cudaStream_t st) {
  launch_k(k_pack_lame<T>, blocks_for(g.n), kThreads, 0, st, g, E, nu_elem, nu, active, scale, lam, mu);
}
void launch_pack_mask(const Grid& g, const uint8_t* ref_mask, uint8_t* pad_mask, cudaStream_t st) {
  launch_k(k_pack_mask, blocks_for(g.n), kThreads, 0, st, g, ref_mask, pad_mask);
}
void launch_pack_active(const Grid& g, const uint8_t* ref, uint8_t* pad, cudaStream_t st) {
  launch_k(k_pack_active, blocks_for(g.n), kThreads, 0, st, g, ref, pad);
}
void launch_inject_mask(const Grid& f, const uint8_t* fmask, const Grid& c, uint8_t* cmask, cudaStream_t st) {
  launch_k(k_inject_mask, blocks_for(c.n), kThreads, 0, st, f, fmask, c, cmask);
}
template <typename T>
void launch_coarsen_E(const Grid& f, const T* Ef, const Grid& c, T* Ec, cudaStream_t st) {
  launch_k(k_coarsen_E<T>, blocks_for(c.n), kThreads, 0, st, f, Ef, c, Ec);
}
template <typename T>
void launch_scale(T* v, long long n, double s, cudaStream_t st) {
  launch_k(k_scale<T>, blocks_for(n), kThreads, 0, st, v, n, s);
}
template <typename T>
void launch_inv_diag_fine(const Grid& g, const T* E, const T* mu, double dL, double dM, T* minv3, cudaStream_t st) {
  launch_k(k_inv_diag_fine<T>, blocks_for(g.n), kThreads, 0, st, g, E, mu, dL, dM, minv3);
}
template <typename Ts, typename Td>
void launch_convert(const Ts* src, Td* dst, long long n, cudaStream_t st) {
  launch_k(k_convert<Ts, Td>, blocks_for(n), kThreads, 0, st, src, dst, n);
}
void launch_used_mask(const Grid& g, const uint8_t* active_pad, uint8_t* mask, cudaStream_t st) {
  launch_k(k_used_mask, blocks_for(g.n), kThreads, 0, st, g, active_pad, mask);
}

#define VF_INST(T)                                                                                   \
  template void launch_pack_vec<T>(const Grid&, const double*, T*, const uint8_t*, cudaStream_t);     \
  template void launch_unpack_vec<T>(const Grid&, const T*, double*, cudaStream_t);                 \
  template void launch_pack_elem<T>(const Grid&, const double*, T*, const uint8_t*, double, cudaStream_t); \
  template void launch_pack_lame<T>(const Grid&, const double*, const double*, double, const uint8_t*, double, T*, T*, cudaStream_t); \
  template void launch_coarsen_E<T>(const Grid&, const T*, const Grid&, T*, cudaStream_t);          \
  template void launch_scale<T>(T*, long long, double, cudaStream_t);                               \
  template void launch_inv_diag_fine<T>(const Grid&, const T*, const T*, double, double, T*, cudaStream_t);
VF_INST(double)
VF_INST(float)
#undef VF_INST
template void launch_convert<double, float>(const double*, float*, long long, cudaStream_t);
template void launch_convert<float, double>(const float*, double*, long long, cudaStream_t);

}  // namespace vf
