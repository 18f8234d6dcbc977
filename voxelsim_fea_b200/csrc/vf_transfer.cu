// Grid transfers of the V-cycle, in gather form (no atomics, deterministic):
//
//   restriction  r_c[J] = D_c sum_{d in {-1,0,1}^3} w(d) r_f[2J + d]
//                w(d) = prod_k (d_k == 0 ? 1 : 1/2)
//     == R = P^T of the reference's trilinear P, scattered there with
//        bincount (core/multigrid.py:404-416); the reference's clipped
//        corners carry weight 0 (multigrid.py:62-72), so the gather is exact.
//   prolongation u_f[i] += D_f sum_J w(i - 2J) e_c[J]     (multigrid.py:418-424, 434)
//   first sweep  u = w * D (Minv b)   -- the first damped-Jacobi sweep of a
//     V-cycle starts from u = 0, where b - A u = b exactly (multigrid.py:430).
#include "vf_common.cuh"

namespace vf {

namespace {

__global__ void __launch_bounds__(256) k_restrict_d(Grid f, const double* __restrict__ rf, Grid c,
                                                    const uint8_t* __restrict__ cm, double* __restrict__ rc,
                                                    const KrylovState* ks) {
  if (ks && ks->done) return;
  const int nx1 = c.lx + 1, ny1 = c.ly + 1, nint = nx1 * ny1 * (c.lz + 1);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int X = t % nx1, rr = t / nx1, Y = rr % ny1, Z = rr / ny1;
    double a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const double w = (dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0);
          const long long q = 3 * (long long)f.idx(2 * X + dx, 2 * Y + dy, 2 * Z + dz);
          a0 += w * rf[q]; a1 += w * rf[q + 1]; a2 += w * rf[q + 2];
        }
    const int p = c.idx(X, Y, Z);
    const uint8_t m = cm[p];
    rc[3 * (long long)p] = (m & 1) ? a0 : 0.0;
    rc[3 * (long long)p + 1] = (m & 2) ? a1 : 0.0;
    rc[3 * (long long)p + 2] = (m & 4) ? a2 : 0.0;
  }
}

__global__ void __launch_bounds__(256) k_restrict_f(Grid f, const float* __restrict__ rf, Grid c,
                                                    const uint8_t* __restrict__ cm, float* __restrict__ rc,
                                                    const KrylovState* ks) {
  if (ks && ks->done) return;
  const int nx1 = c.lx + 1, ny1 = c.ly + 1, nint = nx1 * ny1 * (c.lz + 1);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int X = t % nx1, rr = t / nx1, Y = rr % ny1, Z = rr / ny1;
    float a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy) {
        // the three fine nodes 2X-1 .. 2X+1 of this row are 9 consecutive
        // values starting on an 8-byte boundary (storage x = 2X, rows a
        // multiple of 4 nodes long): four float2 loads and one float
        const long long q = 3 * (long long)f.idx(2 * X - 1, 2 * Y + dy, 2 * Z + dz);
        const float2* q2 = reinterpret_cast<const float2*>(rf + q);
        const float2 v01 = __ldg(q2), v23 = __ldg(q2 + 1), v45 = __ldg(q2 + 2), v67 = __ldg(q2 + 3);
        const float v8 = __ldg(rf + q + 8);
        const float r[9] = {v01.x, v01.y, v23.x, v23.y, v45.x, v45.y, v67.x, v67.y, v8};
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const float w = (dx ? 0.5f : 1.0f) * (dy ? 0.5f : 1.0f) * (dz ? 0.5f : 1.0f);
          const int o = 3 * (dx + 1);
          a0 += w * r[o]; a1 += w * r[o + 1]; a2 += w * r[o + 2];
        }
      }
    const int p = c.idx(X, Y, Z);
    const uint8_t m = cm[p];
    rc[3 * (long long)p] = (m & 1) ? a0 : 0.0f;
    rc[3 * (long long)p + 1] = (m & 2) ? a1 : 0.0f;
    rc[3 * (long long)p + 2] = (m & 4) ? a2 : 0.0f;
  }
}

// Restriction fused with the coarse level's first smoothing step from zero:
// the restricted residual rc (kept: the coarse level's right-hand side) and
// uc = w * (Minv rc), the same sums and products as k_restrict_* followed by
// k_jacobi_from_zero (ghost entries of uc stay untouched: they hold zeros).
template <typename T>
__global__ void __launch_bounds__(256) k_restrict_first(Grid f, const T* __restrict__ rf, Grid c,
                                                        const uint8_t* __restrict__ cm, T* __restrict__ rc,
                                                        const T* __restrict__ minvc, const double* __restrict__ wdev,
                                                        T* __restrict__ uc, const KrylovState* ks) {
  if (ks && ks->done) return;
  const T w = (T)(*wdev);
  const int nx1 = c.lx + 1, ny1 = c.ly + 1, nint = nx1 * ny1 * (c.lz + 1);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int X = t % nx1, rr = t / nx1, Y = rr % ny1, Z = rr / ny1;
    T a0 = 0, a1 = 0, a2 = 0;
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
          const long long q = 3 * (long long)f.idx(2 * X - 1, 2 * Y + dy, 2 * Z + dz);
          const float2* q2 = reinterpret_cast<const float2*>(rf + q);
          const float2 v01 = __ldg(q2), v23 = __ldg(q2 + 1), v45 = __ldg(q2 + 2), v67 = __ldg(q2 + 3);
          const float v8 = __ldg(rf + q + 8);
          const float r[9] = {v01.x, v01.y, v23.x, v23.y, v45.x, v45.y, v67.x, v67.y, v8};
#pragma unroll
          for (int dx = -1; dx <= 1; ++dx) {
            const float wt = (dx ? 0.5f : 1.0f) * (dy ? 0.5f : 1.0f) * (dz ? 0.5f : 1.0f);
            const int o = 3 * (dx + 1);
            a0 += wt * r[o]; a1 += wt * r[o + 1]; a2 += wt * r[o + 2];
          }
        }
    } else {
#pragma unroll
      for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
          for (int dx = -1; dx <= 1; ++dx) {
            const double wt = (dx ? 0.5 : 1.0) * (dy ? 0.5 : 1.0) * (dz ? 0.5 : 1.0);
            const long long q = 3 * (long long)f.idx(2 * X + dx, 2 * Y + dy, 2 * Z + dz);
            a0 += wt * rf[q]; a1 += wt * rf[q + 1]; a2 += wt * rf[q + 2];
          }
    }
    const int p = c.idx(X, Y, Z);
    const uint8_t m = cm[p];
    const long long p3 = 3 * (long long)p;
    const T b0 = (m & 1) ? a0 : (T)0, b1 = (m & 2) ? a1 : (T)0, b2 = (m & 4) ? a2 : (T)0;
    rc[p3] = b0; rc[p3 + 1] = b1; rc[p3 + 2] = b2;
    uc[p3] = (m & 1) ? w * (minvc[p3] * b0) : (T)0;
    uc[p3 + 1] = (m & 2) ? w * (minvc[p3 + 1] * b1) : (T)0;
    uc[p3 + 2] = (m & 4) ? w * (minvc[p3 + 2] * b2) : (T)0;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong_add(Grid c, const T* __restrict__ ec, Grid f,
                                                     const uint8_t* __restrict__ fm, T* __restrict__ uf,
                                                     const KrylovState* ks) {
  if (ks && ks->done) return;
  const int nx1 = f.lx + 1, ny1 = f.ly + 1, nint = nx1 * ny1 * (f.lz + 1);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += gridDim.x * blockDim.x) {
    const int x = t % nx1, rr = t / nx1, y = rr % ny1, z = rr / ny1;
    const int p = f.idx(x, y, z);
    const uint8_t m = fm[p];
    if (!m) continue;
    // all eight coarse corners, weight 0 on the unused ones: the loads are
    // independent (one latency) and x0+1 <= c.lx+1 stays on the padded grid
    const int x0 = x >> 1, y0 = y >> 1, z0 = z >> 1;
    const T wx[2] = {(x & 1) ? (T)0.5 : (T)1, (x & 1) ? (T)0.5 : (T)0};
    const T wy[2] = {(y & 1) ? (T)0.5 : (T)1, (y & 1) ? (T)0.5 : (T)0};
    const T wz[2] = {(z & 1) ? (T)0.5 : (T)1, (z & 1) ? (T)0.5 : (T)0};
    T e0 = 0, e1 = 0, e2 = 0;
#pragma unroll
    for (int kz = 0; kz < 2; ++kz)
#pragma unroll
      for (int ky = 0; ky < 2; ++ky)
#pragma unroll
        for (int kx = 0; kx < 2; ++kx) {
          const T w = wx[kx] * wy[ky] * wz[kz];
          const long long q = 3 * (long long)c.idx(x0 + kx, y0 + ky, z0 + kz);
          e0 += w * __ldg(ec + q); e1 += w * __ldg(ec + q + 1); e2 += w * __ldg(ec + q + 2);
        }
    const long long p3 = 3 * (long long)p;
    if (m & 1) uf[p3] += e0;
    if (m & 2) uf[p3 + 1] += e1;
    if (m & 4) uf[p3 + 2] += e2;
  }
}

// The same prolongation, four consecutive storage nodes of a row per thread:
// their 12 values are 48 contiguous, 16-byte aligned bytes (px is a multiple
// of 4), read and written as whole vectors.
template <typename T> struct Vec12;
template <> struct Vec12<float> {
  float4 v[3];
  __device__ __forceinline__ void load(const float* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    v[0] = q[0]; v[1] = q[1]; v[2] = q[2];
  }
  __device__ __forceinline__ void store(float* p) const {
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = v[0]; q[1] = v[1]; q[2] = v[2];
  }
  __device__ __forceinline__ float& at(int i) { return reinterpret_cast<float*>(v)[i]; }
};
template <> struct Vec12<double> {
  double2 v[6];
  __device__ __forceinline__ void load(const double* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] = q[k];
  }
  __device__ __forceinline__ void store(double* p) const {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int k = 0; k < 6; ++k) q[k] = v[k];
  }
  __device__ __forceinline__ double& at(int i) { return reinterpret_cast<double*>(v)[i]; }
};

// Four consecutive storage nodes per thread (one 16-byte-aligned group of
// u): their coarse parents lie in the three coarse columns 2 gx - 1 .. 2 gx + 1
// of at most two coarse rows and planes, loaded once for the four nodes, and
// only where a weight is non-zero (an even fine coordinate has one parent on
// that axis).  The sums keep the order of the 8-corner loop over (kz, ky, kx)
// with the zero-weight terms left out, which does not change them.
template <typename T>
__global__ void __launch_bounds__(256) k_prolong_add4(Grid c, const T* __restrict__ ec, Grid f,
                                                      const uint8_t* __restrict__ fm, T* __restrict__ uf,
                                                      const KrylovState* ks) {
  if (ks && ks->done) return;
  const int gpr = f.px / 4;                        // 4-node groups per storage row
  const long long ngroups = (long long)gpr * (f.ly + 1) * (f.lz + 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ngroups;
       t += (long long)gridDim.x * blockDim.x) {
    const int gx = (int)(t % gpr);
    const long long rr = t / gpr;
    const int y = (int)(rr % (f.ly + 1)), z = (int)(rr / (f.ly + 1));
    const int p0 = f.idx(-1, y, z) + 4 * gx;        // storage x = 4 gx .. 4 gx + 3
    const uint32_t m4 = *reinterpret_cast<const uint32_t*>(fm + p0);
    if (!m4) continue;
    Vec12<T> u;
    u.load(uf + 3LL * p0);
    const int y0 = y >> 1, z0 = z >> 1;
    const int ny = (y & 1) ? 2 : 1, nz = (z & 1) ? 2 : 1;
    const T wy[2] = {(y & 1) ? (T)0.5 : (T)1, (y & 1) ? (T)0.5 : (T)0};
    const T wz[2] = {(z & 1) ? (T)0.5 : (T)1, (z & 1) ? (T)0.5 : (T)0};
    // node j (logical x = 4 gx - 1 + j) uses coarse column ci = (x >> 1) - (2 gx - 1)
    // and, for odd x, ci + 1: j = 0 -> {0, 1}, 1 -> {1}, 2 -> {1, 2}, 3 -> {2}
    const bool a0 = (m4 & 0xffu) != 0, a1 = (m4 & 0xff00u) != 0, a2 = (m4 & 0xff0000u) != 0,
               a3 = (m4 & 0xff000000u) != 0;
    const bool need[3] = {a0, a0 || a1 || a2, a2 || a3};
    T cv[2][2][3][3];
#pragma unroll
    for (int kz = 0; kz < 2; ++kz)
#pragma unroll
      for (int ky = 0; ky < 2; ++ky)
#pragma unroll
        for (int ci = 0; ci < 3; ++ci) {
          const bool ld = kz < nz && ky < ny && need[ci];
          const long long q = ld ? 3 * (long long)c.idx(2 * gx - 1 + ci, y0 + ky, z0 + kz) : 0;
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) cv[kz][ky][ci][cc] = ld ? __ldg(ec + q + cc) : (T)0;
        }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint8_t m = (uint8_t)(m4 >> (8 * j));
      if (!m) continue;
      const int x = 4 * gx + j - 1;
      const int cb = (j + 1) >> 1;                   // coarse column of x >> 1: 0, 1, 1, 2
      const int nx = (x & 1) ? 2 : 1;
      const T wx[2] = {(x & 1) ? (T)0.5 : (T)1, (x & 1) ? (T)0.5 : (T)0};
      T e0 = 0, e1 = 0, e2 = 0;
#pragma unroll
      for (int kz = 0; kz < 2; ++kz)
#pragma unroll
        for (int ky = 0; ky < 2; ++ky)
#pragma unroll
          for (int kx = 0; kx < 2; ++kx) {
            if (kz >= nz || ky >= ny || kx >= nx) continue;
            const T w = wx[kx] * wy[ky] * wz[kz];
            const T* v = cv[kz][ky][cb + kx];
            e0 += w * v[0]; e1 += w * v[1]; e2 += w * v[2];
          }
      if (m & 1) u.at(3 * j) += e0;
      if (m & 2) u.at(3 * j + 1) += e1;
      if (m & 4) u.at(3 * j + 2) += e2;
    }
    u.store(uf + 3LL * p0);
  }
}

template <typename T>
__global__ void k_jacobi_from_zero(Grid g, const T* __restrict__ b, const T* __restrict__ minv,
                                   const uint8_t* __restrict__ mask, T w0, const double* __restrict__ wdev,
                                   T* __restrict__ u, const KrylovState* ks) {
  if (ks && ks->done) return;
  const T w = wdev ? (T)(*wdev) : w0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    const uint8_t m = mask[p];
    const long long p3 = 3 * (long long)p;
    u[p3] = (m & 1) ? w * (minv[p3] * b[p3]) : (T)0;
    u[p3 + 1] = (m & 2) ? w * (minv[p3 + 1] * b[p3 + 1]) : (T)0;
    u[p3 + 2] = (m & 4) ? w * (minv[p3 + 2] * b[p3 + 2]) : (T)0;
  }
}

inline int blocks_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

template <>
void launch_restrict<double>(const Grid& f, const double* rf, const Grid& c, const uint8_t* cmask, double* rc,
                             const KrylovState* ks, cudaStream_t st) {
  launch_k(k_restrict_d, blocks_for((long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1)), 256, 0, st, f, rf, c, cmask, rc, ks);
}
template <>
void launch_restrict<float>(const Grid& f, const float* rf, const Grid& c, const uint8_t* cmask, float* rc,
                            const KrylovState* ks, cudaStream_t st) {
  launch_k(k_restrict_f, blocks_for((long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1)), 256, 0, st, f, rf, c, cmask, rc, ks);
}

template <typename T>
void launch_restrict_first(const Grid& f, const T* rf, const Grid& c, const uint8_t* cmask, T* rc, const T* minvc,
                           const double* wdev, T* uc, const KrylovState* ks, cudaStream_t st) {
  launch_k(k_restrict_first<T>, blocks_for((long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1)), 256, 0, st, f, rf, c,
           cmask, rc, minvc, wdev, uc, ks);
}
template void launch_restrict_first<float>(const Grid&, const float*, const Grid&, const uint8_t*, float*,
                                           const float*, const double*, float*, const KrylovState*, cudaStream_t);
template void launch_restrict_first<double>(const Grid&, const double*, const Grid&, const uint8_t*, double*,
                                            const double*, const double*, double*, const KrylovState*, cudaStream_t);

template <typename T>
void launch_prolong_add(const Grid& c, const T* ec, const Grid& f, const uint8_t* fmask, T* uf,
                        const KrylovState* ks, cudaStream_t st) {
  launch_k(k_prolong_add4<T>, blocks_for((long long)(f.px / 4) * (f.ly + 1) * (f.lz + 1)), 256, 0, st, c, ec, f, fmask,
           uf, ks);
}

template <typename T>
void launch_jacobi_from_zero(const Grid& g, const T* b, const T* minv3, const uint8_t* mask, double omega,
                             const double* omega_dev, T* u, const KrylovState* ks, cudaStream_t st) {
  launch_k(k_jacobi_from_zero<T>, blocks_for(g.n), 256, 0, st, g, b, minv3, mask, (T)omega, omega_dev, u, ks);
}

template void launch_prolong_add<double>(const Grid&, const double*, const Grid&, const uint8_t*, double*, const KrylovState*, cudaStream_t);
template void launch_prolong_add<float>(const Grid&, const float*, const Grid&, const uint8_t*, float*, const KrylovState*, cudaStream_t);
template void launch_jacobi_from_zero<double>(const Grid&, const double*, const double*, const uint8_t*, double, const double*, double*, const KrylovState*, cudaStream_t);
template void launch_jacobi_from_zero<float>(const Grid&, const float*, const float*, const uint8_t*, double, const double*, float*, const KrylovState*, cudaStream_t);

}  // namespace vf
