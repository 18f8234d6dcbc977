// Assembled coarse operators of the robust (Galerkin) hierarchy.
//
// The reference rediscretizes coarse levels (2x2x2 mean modulus, injected
// Dirichlet mask; core/multigrid.py:255-315).  Under the void/solid contrast
// of noise geometry that hierarchy stops converging, so this library can build
// instead the Galerkin operators
//
//     A_{l+1} = D_{l+1} P^T D_l A_l D_l P D_{l+1}
//
// with P the reference's trilinear prolongation (multigrid.py:42-73).  They are
// stored as node-centric 27-point stencils of 3x3 blocks, SoA:
//     st[(s*9 + r*3 + c) * n + p],  s = (dz+1)*9 + (dy+1)*3 + (dx+1)
// = coupling of DOF r of node p with DOF c of node p + (dx,dy,dz).  Applying
// one is a deterministic gather (one thread per output node).
//
// Build kernels (FP64, once per set_material):
//   * galerkin_from_fine: level 0 (matrix-free hex8) -> level 1.  A coarse
//     element E with 8 fine children e contributes sum_e P_e^T D_e K_e D_e P_e.
//     For a child whose 24 DOFs are all free this is E_e * G[child] with G a
//     fixed 24x24 table (P^T Ke P, precomputed on the host); children that
//     touch a Dirichlet DOF take the masked general path.
//   * galerkin_from_stencil: level l -> l+1 for l >= 1 (stencil RAP).
//   * stencil_mask_and_diag: D_{l+1} = {DOFs with a non-zero Galerkin
//     diagonal}; zero their rows/columns; Jacobi inverse diagonal.
#include <cuda_fp16.h>

#include <type_traits>

#include "vf_common.cuh"
#include "vf_reduce.cuh"

namespace vf {

namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ int sidx(int dx, int dy, int dz) { return (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1); }

__device__ __forceinline__ void decode(const Grid& g, int p, int& x, int& y, int& z) {
  x = p % g.px - 1;
  int t = p / g.px;
  y = t % g.py - 1;
  z = t / g.py - 1;
}

template <typename T, int EPI>
__global__ void __launch_bounds__(256) k_stencil_op(Grid g, OpArgs a, const T* __restrict__ st) {
  KrylovState* ks = a.ks;
  if (ks && ks->done) return;
  const T* __restrict__ u = (const T*)a.u;
  T* __restrict__ out = (T*)a.out;
  const T* __restrict__ b = (const T*)a.b;
  const T* __restrict__ minv = (const T*)a.minv;
  const uint8_t* __restrict__ mask = a.mask;
  const T w = a.omega_dev ? (T)(*a.omega_dev) : (T)a.omega;
  const int nx1 = g.lx + 1, ny1 = g.ly + 1;
  const int nint = nx1 * ny1 * (g.lz + 1);
  const long long n = g.n;
  double dot = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int x = t % nx1;
    const int rr = t / nx1;
    const int y = rr % ny1;
    const int z = rr / ny1;
    const int p = g.idx(x, y, z);
    T k0 = 0, k1 = 0, k2 = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const int s = sidx(dx, dy, dz);
          const int q = g.idx(x + dx, y + dy, z + dz);
          const T u0 = __ldg(u + 3 * q), u1 = __ldg(u + 3 * q + 1), u2 = __ldg(u + 3 * q + 2);
          const T* B = st + (long long)s * 9 * n + p;
          k0 += __ldg(B) * u0 + __ldg(B + n) * u1 + __ldg(B + 2 * n) * u2;
          k1 += __ldg(B + 3 * n) * u0 + __ldg(B + 4 * n) * u1 + __ldg(B + 5 * n) * u2;
          k2 += __ldg(B + 6 * n) * u0 + __ldg(B + 7 * n) * u1 + __ldg(B + 8 * n) * u2;
        }
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

// 1-D trilinear weight of a coarse node at fine offset d (in fine spacings).
__device__ __forceinline__ double w1(int d) { return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0); }

// Per fine element: 1 if all 8 of its nodes have all 3 DOFs free.
__global__ void k_elem_allfree(Grid f, const uint8_t* __restrict__ m, uint8_t* __restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < f.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(f, p, x, y, z);
    uint8_t v = 0;
    if (x >= 0 && x < f.lx && y >= 0 && y < f.ly && z >= 0 && z < f.lz) {
      uint8_t a = 7;
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int i = 0; i < 2; ++i) a &= m[f.idx(x + i, y + j, z + k)];
      v = (a == 7);
    }
    out[p] = v;
  }
}

// Level 0 -> 1.  One thread per coarse interior node N; loops over the 27
// output blocks.  Gtab: [8 child positions][24][24] of P_c^T K P_c for K =
// Ke(nu) (and, with lame, a second table for K_mu after K_lam).  Ktab: the
// plain 24x24 (or K_lam, K_mu) for the masked path.
__global__ void __launch_bounds__(kThreads) k_galerkin_from_fine(Grid f, const double* __restrict__ E,
                                                                 const double* __restrict__ MU,
                                                                 const uint8_t* __restrict__ fmask,
                                                                 const uint8_t* __restrict__ allfree,
                                                                 Grid c, double* __restrict__ stc,
                                                                 const double* __restrict__ Gtab,
                                                                 const double* __restrict__ Ktab, int lame) {
  const int nx1 = c.lx + 1, ny1 = c.ly + 1;
  const int nint = nx1 * ny1 * (c.lz + 1);
  const long long n = c.n;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int X = t % nx1;
    const int rr = t / nx1;
    const int Y = rr % ny1;
    const int Z = rr / ny1;
    const int p = c.idx(X, Y, Z);
    for (int s = 0; s < 27; ++s) {
      const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
      double acc[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) acc[k] = 0.0;
      const int MX = X + dx, MY = Y + dy, MZ = Z + dz;
      if (MX >= 0 && MX <= c.lx && MY >= 0 && MY <= c.ly && MZ >= 0 && MZ <= c.lz) {
        // coarse elements (lower corner L) containing both N and M
        for (int lz = Z - 1; lz <= Z; ++lz) {
          if (lz < 0 || lz >= c.lz || MZ - lz < 0 || MZ - lz > 1) continue;
          for (int ly = Y - 1; ly <= Y; ++ly) {
            if (ly < 0 || ly >= c.ly || MY - ly < 0 || MY - ly > 1) continue;
            for (int lx = X - 1; lx <= X; ++lx) {
              if (lx < 0 || lx >= c.lx || MX - lx < 0 || MX - lx > 1) continue;
              const int aNx = X - lx, aNy = Y - ly, aNz = Z - lz;
              const int aMx = MX - lx, aMy = MY - ly, aMz = MZ - lz;
              const int aN = corner_k(aNx, aNy, aNz), aM = corner_k(aMx, aMy, aMz);
              for (int ch = 0; ch < 8; ++ch) {
                const int ci = ch & 1, cj = (ch >> 1) & 1, ck = ch >> 2;
                const int q = f.idx(2 * lx + ci, 2 * ly + cj, 2 * lz + ck);
                const double Ee = E[q];
                const double Me = lame ? MU[q] : 0.0;
                if (Ee == 0.0 && Me == 0.0) continue;
                if (allfree[q]) {
                  const double* G = Gtab + (size_t)ch * 576;
#pragma unroll
                  for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                      double v = Ee * G[(3 * aN + r) * 24 + 3 * aM + cc];
                      if (lame) v += Me * G[8 * 576 + (3 * aN + r) * 24 + 3 * aM + cc];
                      acc[r * 3 + cc] += v;
                    }
                } else {
                  // masked general path: sum_{i,i'} wN(i) wM(i') m(i,r) m(i',c) K[(i,r),(i',c)]
                  uint8_t mi[8];
                  double wN[8], wM[8];
                  for (int i = 0; i < 8; ++i) {
                    const int ox = (i == 1 || i == 2 || i == 5 || i == 6);
                    const int oy = (i == 2 || i == 3 || i == 6 || i == 7);
                    const int oz = (i >= 4);
                    const int fx = ci + ox, fy = cj + oy, fz = ck + oz;   // fine offset within E, 0..2
                    mi[i] = fmask[f.idx(2 * lx + fx, 2 * ly + fy, 2 * lz + fz)];
                    wN[i] = w1(fx - 2 * aNx) * w1(fy - 2 * aNy) * w1(fz - 2 * aNz);
                    wM[i] = w1(fx - 2 * aMx) * w1(fy - 2 * aMy) * w1(fz - 2 * aMz);
                  }
                  for (int i = 0; i < 8; ++i) {
                    if (wN[i] == 0.0) continue;
                    for (int j = 0; j < 8; ++j) {
                      if (wM[j] == 0.0) continue;
                      const double ww = wN[i] * wM[j];
                      for (int r = 0; r < 3; ++r) {
                        if (!((mi[i] >> r) & 1)) continue;
                        for (int cc = 0; cc < 3; ++cc) {
                          if (!((mi[j] >> cc) & 1)) continue;
                          const int kk = (3 * i + r) * 24 + 3 * j + cc;
                          double kv = Ee * Ktab[kk];
                          if (lame) kv += Me * Ktab[576 + kk];
                          acc[r * 3 + cc] += ww * kv;
                        }
                      }
                    }
                  }
                }
              }
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) stc[((long long)s * 9 + k) * n + p] = acc[k];
    }
  }
}

// Level l -> l+1 by stencil RAP (fine stencil already masked).  One thread
// per (coarse node, offset s) for the diagonal and the 13 upper offsets
// s = 13..26 (consecutive threads: consecutive nodes of one offset); the 13
// lower blocks are the transposed upper blocks of the neighbours
// (k_stencil_mirror), so the coarse stencil is exactly symmetric.
__global__ void __launch_bounds__(kThreads) k_galerkin_from_stencil(Grid f, const double* __restrict__ stf,
                                                                    Grid c, double* __restrict__ stc) {
  const int nx1 = c.lx + 1, ny1 = c.ly + 1;
  const long long nint = (long long)nx1 * ny1 * (c.lz + 1);
  const long long nf = f.n, nc = c.n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 14 * nint;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = 13 + (int)(t / nint);
    const int node = (int)(t % nint);
    const int X = node % nx1;
    const int rr = node / nx1;
    const int Y = rr % ny1;
    const int Z = rr / ny1;
    const int p = c.idx(X, Y, Z);
    {
      const int Dx = s % 3 - 1, Dy = (s / 3) % 3 - 1, Dz = s / 9 - 1;
      double acc[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) acc[k] = 0.0;
      const int MX = X + Dx, MY = Y + Dy, MZ = Z + Dz;
      if (MX >= 0 && MX <= c.lx && MY >= 0 && MY <= c.ly && MZ >= 0 && MZ <= c.lz) {
        for (int iz = -1; iz <= 1; ++iz)
          for (int iy = -1; iy <= 1; ++iy)
            for (int ix = -1; ix <= 1; ++ix) {
              const int fx = 2 * X + ix, fy = 2 * Y + iy, fz = 2 * Z + iz;
              const double wi = w1(ix) * w1(iy) * w1(iz);
              const int fp = f.idx(fx, fy, fz);
              for (int jz = -1; jz <= 1; ++jz) {
                const int sz = 2 * MZ + jz - fz;
                if (sz < -1 || sz > 1) continue;
                for (int jy = -1; jy <= 1; ++jy) {
                  const int sy = 2 * MY + jy - fy;
                  if (sy < -1 || sy > 1) continue;
                  for (int jx = -1; jx <= 1; ++jx) {
                    const int sx = 2 * MX + jx - fx;
                    if (sx < -1 || sx > 1) continue;
                    const double ww = wi * w1(jx) * w1(jy) * w1(jz);
                    const double* B = stf + (long long)sidx(sx, sy, sz) * 9 * nf + fp;
#pragma unroll
                    for (int k = 0; k < 9; ++k) acc[k] += ww * B[k * nf];
                  }
                }
              }
            }
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) stc[((long long)s * 9 + k) * nc + p] = acc[k];
    }
  }
}

// Lower offsets s = 0..12 from the upper ones: block (s, p)[r][c] =
// block (26 - s, p + off(s))[c][r] (zero where the neighbour is outside).
__global__ void __launch_bounds__(kThreads) k_stencil_mirror(Grid c, double* __restrict__ stc) {
  const int nx1 = c.lx + 1, ny1 = c.ly + 1;
  const long long nint = (long long)nx1 * ny1 * (c.lz + 1);
  const long long nc = c.n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 13 * nint;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t / nint);
    const int node = (int)(t % nint);
    const int X = node % nx1;
    const int rr = node / nx1;
    const int Y = rr % ny1;
    const int Z = rr / ny1;
    const int p = c.idx(X, Y, Z);
    const int MX = X + s % 3 - 1, MY = Y + (s / 3) % 3 - 1, MZ = Z + s / 9 - 1;
    const bool in = MX >= 0 && MX <= c.lx && MY >= 0 && MY <= c.ly && MZ >= 0 && MZ <= c.lz;
    const long long q = in ? c.idx(MX, MY, MZ) : 0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
        stc[((long long)s * 9 + 3 * r + cc) * nc + p] = in ? stc[((long long)(26 - s) * 9 + 3 * cc + r) * nc + q] : 0.0;
  }
}

// Stencil of the element operator itself (sum_e E_e Ke, masked by D): used for
// a direct coarsest solve on a rediscretized level.
__global__ void __launch_bounds__(kThreads) k_stencil_from_elements(Grid g, const double* __restrict__ E,
                                                                    const double* __restrict__ MU,
                                                                    const uint8_t* __restrict__ mask,
                                                                    double* __restrict__ st,
                                                                    const double* __restrict__ Ktab, int lame) {
  const int nx1 = g.lx + 1, ny1 = g.ly + 1;
  const int nint = nx1 * ny1 * (g.lz + 1);
  const long long n = g.n;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int X = t % nx1;
    const int rr = t / nx1;
    const int Y = rr % ny1;
    const int Z = rr / ny1;
    const int p = g.idx(X, Y, Z);
    const uint8_t mp = mask[p];
    for (int s = 0; s < 27; ++s) {
      const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
      double acc[9];
      for (int k = 0; k < 9; ++k) acc[k] = 0.0;
      const int MX = X + dx, MY = Y + dy, MZ = Z + dz;
      const uint8_t mq = mask[g.idx(MX, MY, MZ)];
      for (int lz = Z - 1; lz <= Z; ++lz) {
        if (MZ - lz < 0 || MZ - lz > 1) continue;
        for (int ly = Y - 1; ly <= Y; ++ly) {
          if (MY - ly < 0 || MY - ly > 1) continue;
          for (int lx = X - 1; lx <= X; ++lx) {
            if (MX - lx < 0 || MX - lx > 1) continue;
            const int q = g.idx(lx, ly, lz);
            const double Ee = E[q], Me = lame ? MU[q] : 0.0;
            const int aN = corner_k(X - lx, Y - ly, Z - lz), aM = corner_k(MX - lx, MY - ly, MZ - lz);
            for (int r = 0; r < 3; ++r)
              for (int cc = 0; cc < 3; ++cc) {
                const int kk = (3 * aN + r) * 24 + 3 * aM + cc;
                acc[r * 3 + cc] += Ee * Ktab[kk] + (lame ? Me * Ktab[576 + kk] : 0.0);
              }
          }
        }
      }
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
          const bool keep = ((mp >> r) & 1) && ((mq >> cc) & 1);
          st[((long long)s * 9 + r * 3 + cc) * n + p] = keep ? acc[r * 3 + cc] : 0.0;
        }
    }
  }
}

// Coarse free mask from the Galerkin diagonal (D_{l+1}).
__global__ void k_mask_from_diag(Grid c, const double* __restrict__ st, uint8_t* __restrict__ cmask) {
  const long long n = c.n;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < c.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(c, p, x, y, z);
    uint8_t m = 0;
    if (x >= 0 && x <= c.lx && y >= 0 && y <= c.ly && z >= 0 && z <= c.lz) {
      const int s0 = 13;   // (0,0,0)
      for (int r = 0; r < 3; ++r)
        if (st[((long long)s0 * 9 + r * 4) * n + p] > 0.0) m |= (uint8_t)(1 << r);
    }
    cmask[p] = m;
  }
}

// Zero rows/columns of non-free DOFs; Minv = 1/diag (0 for non-free).
__global__ void k_apply_mask_diag(Grid c, double* __restrict__ st, const uint8_t* __restrict__ cmask,
                                  double* __restrict__ minv3) {
  const long long n = c.n;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < c.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(c, p, x, y, z);
    const bool inside = (x >= 0 && x <= c.lx && y >= 0 && y <= c.ly && z >= 0 && z <= c.lz);
    const uint8_t mp = cmask[p];
    for (int s = 0; s < 27; ++s) {
      const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
      uint8_t mq = 0;
      if (inside) mq = cmask[c.idx(x + dx, y + dy, z + dz)];
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
          const bool keep = inside && ((mp >> r) & 1) && ((mq >> cc) & 1);
          if (!keep) st[((long long)s * 9 + r * 3 + cc) * n + p] = 0.0;
        }
    }
    for (int r = 0; r < 3; ++r) {
      const double d = st[((long long)13 * 9 + r * 4) * n + p];
      minv3[3 * (long long)p + r] = ((mp >> r) & 1) && d != 0.0 ? 1.0 / d : 0.0;
    }
  }
}

inline int blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 32) b = 148 * 32;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

template <typename T>
int stencil_op_grid_blocks(const Grid& g) {
  long long nint = (long long)(g.lx + 1) * (g.ly + 1) * (g.lz + 1);
  long long b = (nint + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

template <typename T>
void launch_stencil_op(const Grid& g, int epi, const OpArgs& a, const T* stencil, cudaStream_t st) {
  const int blocks = stencil_op_grid_blocks<T>(g);
  if (epi == EPI_APPLY) launch_k(k_stencil_op<T, EPI_APPLY>, blocks, 256, 0, st, g, a, stencil);
  else if (epi == EPI_SMOOTH) launch_k(k_stencil_op<T, EPI_SMOOTH>, blocks, 256, 0, st, g, a, stencil);
  else launch_k(k_stencil_op<T, EPI_RESID>, blocks, 256, 0, st, g, a, stencil);
}
template void launch_stencil_op<double>(const Grid&, int, const OpArgs&, const double*, cudaStream_t);
template void launch_stencil_op<float>(const Grid&, int, const OpArgs&, const float*, cudaStream_t);
template int stencil_op_grid_blocks<double>(const Grid&);
template int stencil_op_grid_blocks<float>(const Grid&);

void launch_elem_allfree(const Grid& f, const uint8_t* fmask, uint8_t* allfree, cudaStream_t st) {
  launch_k(k_elem_allfree, blocks_for(f.n, 256), 256, 0, st, f, fmask, allfree);
}

void launch_galerkin_from_fine(const Grid& f, const double* E, const double* mu, const uint8_t* fmask,
                               const uint8_t* allfree, const Grid& c, double* stencil_c, const double* Gtab,
                               const double* Ktab, int lame, cudaStream_t st) {
  long long nint = (long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1);
  launch_k(k_galerkin_from_fine, blocks_for(nint, kThreads), kThreads, 0, st, f, E, mu, fmask, allfree, c, stencil_c,
                                                                        Gtab, Ktab, lame);
}

void launch_galerkin_from_stencil(const Grid& f, const double* stencil_f, const Grid& c, double* stencil_c,
                                  cudaStream_t st) {
  long long nint = (long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1);
  launch_k(k_galerkin_from_stencil, blocks_for(14 * nint, kThreads), kThreads, 0, st, f, stencil_f, c, stencil_c);
  launch_k(k_stencil_mirror, blocks_for(13 * nint, kThreads), kThreads, 0, st, c, stencil_c);
}

void launch_stencil_from_elements(const Grid& g, const double* E, const double* mu, const uint8_t* mask,
                                  double* stencil, const double* Ktab, int lame, cudaStream_t st) {
  long long nint = (long long)(g.lx + 1) * (g.ly + 1) * (g.lz + 1);
  launch_k(k_stencil_from_elements, blocks_for(nint, kThreads), kThreads, 0, st, g, E, mu, mask, stencil, Ktab, lame);
}

void launch_galerkin_mask(const Grid& c, double* stencil, uint8_t* cmask, double* minv3, cudaStream_t st) {
  launch_k(k_mask_from_diag, blocks_for(c.n, 256), 256, 0, st, c, stencil, cmask);
  launch_k(k_apply_mask_diag, blocks_for(c.n, 256), 256, 0, st, c, stencil, cmask, minv3);
}

void launch_stencil_diag(const Grid& c, double* stencil, const uint8_t* cmask, double* minv3, cudaStream_t st) {
  launch_k(k_apply_mask_diag, blocks_for(c.n, 256), 256, 0, st, c, stencil, cmask, minv3);
}

// ---------------------------------------------------------------------------
// Symmetric, diagonally scaled Galerkin stencils (default coarse storage).
//
// A Galerkin operator is symmetric, so only the diagonal block (6 values) and
// the 13 "upper" neighbour blocks (offsets s = 14..26, 9 values each) are
// stored: 123 values per node; the 13 lower blocks are read transposed from
// the neighbour that stores them.  Values are the symmetrically scaled
// A~ = D^-1/2 A D^-1/2 (unit diagonal, |entries| <= 1 for an SPD operator), so
// half precision keeps its relative precision over any stiffness contrast;
// the apply computes y = D^1/2 A~ (D^1/2 u) with sqrtd = D^1/2 per DOF (0 on
// non-free DOFs).  Value order within a node, k in [0, 128):
//   k = 0..5   diagonal block (r,c) = (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
//   k = 6 + 9*(s-14) + 3*r + c   upper block s, DOF r of p with DOF c of p+off(s)
//   k = 123..127 zero padding
// Storage is warp-chunked (SymLayout): 16-byte chunk j of 32 consecutive nodes
// is contiguous, so a warp loads a chunk of its 32 nodes in one 512-byte
// transaction whatever the alignment of its first node.
// ---------------------------------------------------------------------------
namespace {

template <typename S> __device__ __forceinline__ S st_from(double v);
template <> __device__ __forceinline__ float st_from<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ double st_from<double>(double v) { return v; }
template <> __device__ __forceinline__ __half st_from<__half>(double v) { return __double2half(v); }
__host__ __device__ constexpr int diag_r(int k) { return k < 3 ? 0 : (k < 5 ? 1 : 2); }
__host__ __device__ constexpr int diag_c(int k) { return k < 3 ? k : (k < 5 ? k - 2 : 2); }

template <typename S>
__global__ void k_stencil_compress(Grid g, const double* __restrict__ st, const uint8_t* __restrict__ mask,
                                   S* __restrict__ stc, typename SymLayout<S>::Q* __restrict__ sqrtd) {
  using L = SymLayout<S>;
  using Q = typename L::Q;
  const long long n = g.n;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    const bool inside = (x >= 0 && x <= g.lx && y >= 0 && y <= g.ly && z >= 0 && z <= g.lz);
    double sp[3];
    for (int r = 0; r < 3; ++r) {
      const double d = st[((long long)13 * 9 + r * 4) * n + p];
      sp[r] = (inside && ((mask[p] >> r) & 1) && d > 0.0) ? 1.0 / sqrt(d) : 0.0;
      sqrtd[3 * (long long)p + r] = (Q)(sp[r] > 0.0 ? 1.0 / sp[r] : 0.0);
    }
    for (int k = 0; k < 6; ++k) {
      const int r = diag_r(k), c = diag_c(k);
      stc[L::off(p, k)] = st_from<S>(st[((long long)13 * 9 + r * 3 + c) * n + p] * sp[r] * sp[c]);
    }
    for (int s = 14; s < 27; ++s) {
      const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
      double sq[3] = {0.0, 0.0, 0.0};
      if (inside) {
        const int q = g.idx(x + dx, y + dy, z + dz);
        for (int c = 0; c < 3; ++c) {
          const double d = st[((long long)13 * 9 + c * 4) * n + q];
          sq[c] = (((mask[q] >> c) & 1) && d > 0.0) ? 1.0 / sqrt(d) : 0.0;
        }
      }
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          const double v = inside ? st[((long long)s * 9 + r * 3 + c) * n + p] * sp[r] * sq[c] : 0.0;
          stc[L::off(p, 6 + 9 * (s - 14) + 3 * r + c)] = st_from<S>(v);
        }
    }
    for (int k = 123; k < 128; ++k) stc[L::off(p, k)] = st_from<S>(0.0);
  }
}

// One 16-byte chunk of stencil values, unpacked to the accumulation type.
template <typename S, typename A> struct Chunk;
template <> struct Chunk<__half, float> {
  float v[8];
  __device__ __forceinline__ void load(const __half* base) {
    const uint4 w = __ldg(reinterpret_cast<const uint4*>(base));
    const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      __half2 h;
      memcpy(&h, &ws[i], 4);
      const float2 f = __half22float2(h);
      v[2 * i] = f.x; v[2 * i + 1] = f.y;
    }
  }
};
template <> struct Chunk<float, float> {
  float v[4];
  __device__ __forceinline__ void load(const float* base) {
    const float4 w = __ldg(reinterpret_cast<const float4*>(base));
    v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
  }
};
template <> struct Chunk<double, double> {
  double v[2];
  __device__ __forceinline__ void load(const double* base) {
    const double2 w = __ldg(reinterpret_cast<const double2*>(base));
    v[0] = w.x; v[1] = w.y;
  }
};

constexpr int SX = 32, SY = 8;   // node tile of the marching stencil kernel

// y = mask(D^1/2 A~ D^1/2 u) with the epilogues of the fine operator.  A CTA
// owns a 32 x 8 tile of node columns and marches along z over `zchunk`
// planes; v = D^1/2 u of the halo tile lives in a 4-plane shared ring (one
// barrier per plane: the slot written for plane z+1 was last read two steps
// earlier), the next plane is prefetched into registers while the current one
// is computed, and the stencil values stream through coalesced 16-byte loads.
// 4 CTAs (32 warps) per SM at <= 64 registers: the kernel is latency bound on
// its stencil loads, and more resident warps hide more of it
template <typename T, typename S, int EPI>
__global__ void __launch_bounds__(SX * SY, 4) k_sym_march(Grid g, OpArgs a, const S* __restrict__ stc,
                                                           const T* __restrict__ sqd, int zchunk) {
  using Lay = SymLayout<S>;
  using A = typename std::conditional<sizeof(T) == 8, double, float>::type;
  constexpr int VPC = Lay::VPC;
  constexpr int HX = SX + 2, HY = SY + 2, NH = HX * HY;
  constexpr int NTH = SX * SY;
  constexpr int NL = (NH + NTH - 1) / NTH;
  __shared__ A vs[4][3][HY][HX];

  KrylovState* ks = a.ks;
  if (ks && ks->done) return;
  const T* __restrict__ u = (const T*)a.u;
  // out may be the step field dprev (the smoothed prolongation updates x in
  // place: each element is read and written by the same thread); a null rhs
  // reads as zero
  T* out = (T*)a.out;
  const T* b = (const T*)a.b;
  const T* __restrict__ minv = (const T*)a.minv;
  const uint8_t* __restrict__ mask = a.mask;
  const T w = a.omega_dev ? (T)(*a.omega_dev) : (T)a.omega;
  const T* dprev = (const T*)a.dprev;
  T* dout = (T*)a.dout;
  const T c1 = a.c1_dev ? (T)(*a.c1_dev) : (T)0;

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SX + tx;
  const int X0 = blockIdx.x * SX, Y0 = blockIdx.y * SY;
  const int zb = blockIdx.z * zchunk;
  const int ze = min(zb + zchunk, g.lz + 1);
  const int sz = g.px * g.py;
  const int x = X0 + tx, y = Y0 + ty;
  const bool active = (x <= g.lx) && (y <= g.ly);

  // halo elements of this thread: in-plane storage offset (or -1)
  int hoff[NL];
  int hsl[NL];
#pragma unroll
  for (int q = 0; q < NL; ++q) {
    const int e = tid + q * NTH;
    const int i = e % HX, j = e / HX;
    const int xs = X0 + i, ys = Y0 + j;   // storage coordinates (x + 1, y + 1)
    hsl[q] = e < NH ? e : -1;
    hoff[q] = (e < NH && xs < g.px && ys < g.py) ? ys * g.px + xs : -1;
  }
  A pv[NL][3];
  auto fetch = [&](int zz) {   // logical plane zz in [-1, lz + 1]
#pragma unroll
    for (int q = 0; q < NL; ++q) {
      const bool ok = hoff[q] >= 0;
      const long long p3 = ok ? 3LL * ((long long)(zz + 1) * sz + hoff[q]) : 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) pv[q][c] = ok ? (A)__ldg(sqd + p3 + c) * (A)__ldg(u + p3 + c) : (A)0;
    }
  };
  auto store = [&](int zz) {
    const int slot = (zz + 1) & 3;
#pragma unroll
    for (int q = 0; q < NL; ++q)
      if (hsl[q] >= 0) {
        const int i = hsl[q] % HX, j = hsl[q] / HX;
#pragma unroll
        for (int c = 0; c < 3; ++c) vs[slot][c][j][i] = pv[q][c];
      }
  };

  double dot = 0.0;
  fetch(zb - 1);
  store(zb - 1);
  fetch(zb);
  store(zb);
  if (zb + 1 <= g.lz + 1) fetch(zb + 1);
#pragma unroll 1
  for (int z = zb; z < ze; ++z) {
    store(z + 1);                         // plane z+1 <= lz+1 always (z <= lz)
    if (z + 2 <= g.lz + 1) fetch(z + 2);
    __syncthreads();
    if (!active) continue;
    const int p = g.idx(x, y, z);
    const int s0 = (z + 1) & 3;
    auto V = [&](int dx, int dy, int dz, int c) -> A {
      return vs[(s0 + dz + 4) & 3][c][ty + 1 + dy][tx + 1 + dx];
    };
    A acc[3] = {(A)0, (A)0, (A)0};
    // own values: diagonal block and the 13 upper blocks
    const S* own = stc + Lay::off(p, 0);
#pragma unroll
    for (int j = 0; j < 123 / VPC + 1; ++j) {
      Chunk<S, A> ch;
      ch.load(own + (long long)j * 32 * VPC);
#pragma unroll
      for (int i = 0; i < VPC; ++i) {
        const int k = j * VPC + i;
        if (k < 6) {
          const int r = diag_r(k), c = diag_c(k);
          acc[r] += ch.v[i] * V(0, 0, 0, c);
          if (r != c) acc[c] += ch.v[i] * V(0, 0, 0, r);
        } else if (k < 123) {
          const int s = 14 + (k - 6) / 9, rc = (k - 6) % 9;
          acc[rc / 3] += ch.v[i] * V(s % 3 - 1, (s / 3) % 3 - 1, s / 9 - 1, rc % 3);
        }
      }
    }
    // lower blocks: block s of q = p - off(s), transposed
#pragma unroll
    for (int s = 14; s < 27; ++s) {
      const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
      const int q = p - ((dz * g.py + dy) * g.px + dx);
      const int k0 = 6 + 9 * (s - 14);
      const S* base = stc + Lay::off(q, 0);
#pragma unroll
      for (int j = k0 / VPC; j <= (k0 + 8) / VPC; ++j) {
        Chunk<S, A> ch;
        ch.load(base + (long long)j * 32 * VPC);
#pragma unroll
        for (int i = 0; i < VPC; ++i) {
          const int k = j * VPC + i;
          if (k >= k0 && k < k0 + 9) {
            const int r = (k - k0) / 3, c = (k - k0) % 3;
            acc[c] += ch.v[i] * V(-dx, -dy, -dz, r);
          }
        }
      }
    }
    const uint8_t m = mask[p];
    const long long p3 = 3 * (long long)p;
    const T k0 = (m & 1) ? (T)(acc[0] * (A)sqd[p3]) : (T)0;
    const T k1 = (m & 2) ? (T)(acc[1] * (A)sqd[p3 + 1]) : (T)0;
    const T k2 = (m & 4) ? (T)(acc[2] * (A)sqd[p3 + 2]) : (T)0;
    const T b0 = b ? b[p3] : (T)0, b1 = b ? b[p3 + 1] : (T)0, b2 = b ? b[p3 + 2] : (T)0;
    if (EPI == EPI_APPLY) {
      out[p3] = k0; out[p3 + 1] = k1; out[p3 + 2] = k2;
      if (a.dot_partials)
        dot += (double)u[p3] * (double)k0 + (double)u[p3 + 1] * (double)k1 + (double)u[p3 + 2] * (double)k2;
    } else if (EPI == EPI_SMOOTH) {
      const T r0 = b0 - k0, r1 = b1 - k1, r2 = b2 - k2;
      const T u0 = u[p3], u1 = u[p3 + 1], u2 = u[p3 + 2];
      T o0 = u0 + ((m & 1) ? w * (minv[p3] * r0) : (T)0);
      T o1 = u1 + ((m & 2) ? w * (minv[p3 + 1] * r1) : (T)0);
      T o2 = u2 + ((m & 4) ? w * (minv[p3 + 2] * r2) : (T)0);
      if (dprev) { o0 += c1 * dprev[p3]; o1 += c1 * dprev[p3 + 1]; o2 += c1 * dprev[p3 + 2]; }
      out[p3] = o0; out[p3 + 1] = o1; out[p3 + 2] = o2;
      if (dout) { dout[p3] = o0 - u0; dout[p3 + 1] = o1 - u1; dout[p3 + 2] = o2 - u2; }
    } else {
      out[p3] = b0 - k0; out[p3 + 1] = b1 - k1; out[p3 + 2] = b2 - k2;
    }
  }
  if (EPI == EPI_APPLY && a.dot_partials && ks) reduce_and_finalize(dot, a.dot_partials, ks, a.dot_slot, nullptr);
}

}  // namespace

template <typename S>
void launch_stencil_compress(const Grid& g, const double* st, const uint8_t* mask, S* stc,
                             typename SymLayout<S>::Q* sqrtd, cudaStream_t st_) {
  launch_k(k_stencil_compress<S>, blocks_for(g.n, 256), 256, 0, st_, g, st, mask, stc, sqrtd);
}
template void launch_stencil_compress<__half>(const Grid&, const double*, const uint8_t*, __half*, float*, cudaStream_t);
template void launch_stencil_compress<float>(const Grid&, const double*, const uint8_t*, float*, float*, cudaStream_t);
template void launch_stencil_compress<double>(const Grid&, const double*, const uint8_t*, double*, double*, cudaStream_t);

// z-planes per CTA of the marching stencil kernel: about 4 CTAs per SM.
int sym_zchunk(const Grid& g) {
  const long long tiles = (long long)((g.lx + 1 + SX - 1) / SX) * ((g.ly + 1 + SY - 1) / SY);
  long long nz = (4LL * 148 + tiles - 1) / tiles;
  if (nz < 1) nz = 1;
  const int planes = g.lz + 1;
  return (int)((planes + nz - 1) / nz);
}

template <typename T, typename S>
void launch_stencil_sym_op(const Grid& g, int epi, const OpArgs& a, const S* stc, const T* sqrtd, int zchunk,
                           cudaStream_t st) {
  if (zchunk < 1) zchunk = sym_zchunk(g);
  const dim3 grid((g.lx + 1 + SX - 1) / SX, (g.ly + 1 + SY - 1) / SY, (g.lz + 1 + zchunk - 1) / zchunk);
  const dim3 block(SX, SY);
  if (epi == EPI_APPLY) launch_k(k_sym_march<T, S, EPI_APPLY>, grid, block, 0, st, g, a, stc, sqrtd, zchunk);
  else if (epi == EPI_SMOOTH) launch_k(k_sym_march<T, S, EPI_SMOOTH>, grid, block, 0, st, g, a, stc, sqrtd, zchunk);
  else launch_k(k_sym_march<T, S, EPI_RESID>, grid, block, 0, st, g, a, stc, sqrtd, zchunk);
}
template void launch_stencil_sym_op<float, __half>(const Grid&, int, const OpArgs&, const __half*, const float*, int, cudaStream_t);
template void launch_stencil_sym_op<float, float>(const Grid&, int, const OpArgs&, const float*, const float*, int, cudaStream_t);
template void launch_stencil_sym_op<double, double>(const Grid&, int, const OpArgs&, const double*, const double*, int, cudaStream_t);

}  // namespace vf
