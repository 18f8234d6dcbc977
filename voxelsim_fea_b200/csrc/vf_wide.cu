// Wide Galerkin levels: the coarse space with a smoothed prolongation.
//
// The robust hierarchy's coarse operators A_{l+1} = D P^T A_l P D use the
// reference's trilinear P (core/multigrid.py:42-73).  On the transfer from a
// Galerkin level l to l+1 this library can instead use the smoothed
// prolongation of smoothed aggregation,
//
//     P_s = D_l (I - c_l D_l^-1 A_l) P,     c_l = (4/3) / lambda_l,
//
// lambda_l the padded power-iteration estimate of lambda_max(D_l^-1 A_l),
// and A_{l+1} = D_{l+1} P_s^T A_l P_s D_{l+1}.  The smoothed basis functions
// reach one fine node further, so the coarse operator couples each node with
// the nodes up to two (in general: R) coarse spacings away: 125 blocks of
// 3x3 per node instead of 27.  The transfers themselves need no new kernel
// (vf_solver.cu): restriction P_s^T r = P^T (r - c A (Minv r)) and
// prolongation x += P_s e = t - c Minv A t (t = P e) are the level's own
// residual and sweep kernels.
//
// Set-up (FP64, once per set_material), for the transfer l -> l+1:
//   k_prolong_blocks  the 3x3 blocks P_s[i][J] of every fine node i
//                     ((Pr+1)^3 coarse slots per node, stored entry-major
//                     and slot-fastest per node; Pr = 1 + R_l when
//                     smoothed, 1 for the trilinear P);
//   k_rap_b           B = A_l P_s, (Pr+R_l+1)^3 coarse slots per fine node;
//   k_rap_c           the diagonal and upper blocks of A_{l+1} = P_s^T B, one
//                     CTA per coarse node, P_s[.][I] staged in shared memory;
//   k_wide_mirror     the lower blocks as the neighbours' transposed upper
//                     ones (the coarse operator is exactly symmetric);
//   k_wide_mask_diag  D_{l+1} = DOFs with a positive diagonal, rows / columns
//                     of the others zeroed, inverse diagonal.
// Full stencils: st[(s*9 + 3r + c) * n + p], s = ((dz+R)*W + (dy+R))*W + (dx+R),
// W = 2R+1: coupling of DOF r of node p with DOF c of node p + (dx,dy,dz).
//
// Apply (V-cycle): symmetric, diagonally scaled storage as on the 27-block
// levels (vf_stencil.cu) -- the diagonal block (6 values) and the upper
// blocks s > center (9 values each) of A~ = D^-1/2 A D^-1/2, FP16 for the
// FP32 V-cycle, warp-chunked so a warp loads one 16-byte chunk of 32
// consecutive nodes at once; the lower blocks are read transposed from the
// neighbour that stores them.  One thread per padded node; the vector is read
// through the L1 (the coarse levels are small).
#include <cuda_fp16.h>

#include <type_traits>

#include "vf_common.cuh"
#include "vf_reduce.cuh"

namespace vf {

namespace {

__host__ __device__ constexpr int wide_w(int R) { return 2 * R + 1; }
__host__ __device__ constexpr int wide_nb(int R) { return (2 * R + 1) * (2 * R + 1) * (2 * R + 1); }

// 1-D trilinear weight of a coarse node at fine offset d
__device__ __forceinline__ double tw(int d) { return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0); }
// ceil(v / 2) for any sign
__device__ __forceinline__ int ceil_half(int v) { return v >= 0 ? (v + 1) / 2 : -((-v) / 2); }

__device__ __forceinline__ bool inside(const Grid& g, int x, int y, int z) {
  return x >= 0 && x <= g.lx && y >= 0 && y <= g.ly && z >= 0 && z <= g.lz;
}

__device__ __forceinline__ void interior_xyz(const Grid& g, long long t, int& x, int& y, int& z) {
  const int nx1 = g.lx + 1, ny1 = g.ly + 1;
  x = (int)(t % nx1);
  const long long r = t / nx1;
  y = (int)(r % ny1);
  z = (int)(r / ny1);
}

__device__ __forceinline__ void decode(const Grid& g, int p, int& x, int& y, int& z) {
  x = p % g.px - 1;
  const int t = p / g.px;
  y = t % g.py - 1;
  z = t / g.py - 1;
}

inline int blocks_for(long long n, int threads, long long cap = 148LL * 64) {
  long long b = (n + threads - 1) / threads;
  if (b > cap) b = cap;
  return (int)(b < 1 ? 1 : b);
}

// ---- set-up ----------------------------------------------------------------

// CTAs of the set-up products handle NG consecutive interior nodes x NS
// slots (NG = kSetupThreads / NS); the level-l blocks of those nodes are
// staged once in shared memory instead of being re-read by every slot.
constexpr int kSetupThreads = 256;

// Stage the full stencil blocks of nodes [n0, n0 + NG) in sA[(node * NB + s) * 9 + k].
__device__ __forceinline__ void stage_blocks(const Grid& f, const double* __restrict__ stf, int NB, long long n0,
                                             int NG, long long nint, double* sA) {
  const long long nf = f.n;
  for (int e = threadIdx.x; e < NG * NB * 9; e += blockDim.x) {
    const int nl = e / (NB * 9), rem = e % (NB * 9), s = rem / 9, k = rem % 9;
    double v = 0.0;
    if (n0 + nl < nint) {
      int x, y, z;
      interior_xyz(f, n0 + nl, x, y, z);
      v = stf[((long long)s * 9 + k) * nf + f.idx(x, y, z)];
    }
    sA[e] = v;
  }
}

// P_s[i][J] per fine interior node i and coarse slot (ax, ay, az), J = jlo(i) + a,
// jlo = ceil((i - Pr) / 2) per axis; psb[(p * 9 + 3r + c) * NS + slot] (slot fastest:
// the consecutive slots a warp reads or writes are consecutive words).
// smoothed: *cdev != 0 (the blocks of A staged); else the trilinear D P.
__global__ void __launch_bounds__(kSetupThreads) k_prolong_blocks(Grid f, const double* __restrict__ stf, int Rf,
                                                                  const uint8_t* __restrict__ fm,
                                                                  const double* __restrict__ minvf,
                                                                  const double* __restrict__ cdev, int Pr, Grid c,
                                                                  double* __restrict__ psb) {
  extern __shared__ double sA[];
  const int NA = Pr + 1, NS = NA * NA * NA, NG = kSetupThreads / NS;
  const int W = wide_w(Rf), NB = wide_nb(Rf);
  const long long nint = (long long)(f.lx + 1) * (f.ly + 1) * (f.lz + 1);
  const double cc = cdev ? *cdev : 0.0;
  for (long long n0 = (long long)blockIdx.x * NG; n0 < nint; n0 += (long long)gridDim.x * NG) {
    if (cdev) {
      __syncthreads();
      stage_blocks(f, stf, NB, n0, NG, nint, sA);
      __syncthreads();
    }
    const int nl = threadIdx.x / NS, slot = threadIdx.x % NS;
    if (nl >= NG || n0 + nl >= nint) continue;
    int x, y, z;
    interior_xyz(f, n0 + nl, x, y, z);
    const int p = f.idx(x, y, z);
    const int ax = slot % NA, ay = (slot / NA) % NA, az = slot / (NA * NA);
    const int Jx = ceil_half(x - Pr) + ax, Jy = ceil_half(y - Pr) + ay, Jz = ceil_half(z - Pr) + az;
    double blk[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) blk[k] = 0.0;
    if (inside(c, Jx, Jy, Jz)) {
      const uint8_t m = fm[p];
      const double w = tw(x - 2 * Jx) * tw(y - 2 * Jy) * tw(z - 2 * Jz);
#pragma unroll
      for (int r = 0; r < 3; ++r)
        if ((m >> r) & 1) blk[4 * r] = w;
      if (cdev && cc != 0.0 && m) {
        // - c Minv_i sum_d A[i][d] w(i + d, J)
        double acc[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[k] = 0.0;
        const double* A = sA + (long long)nl * NB * 9;
        for (int s = 0; s < NB; ++s) {
          const int dx = s % W - Rf, dy = (s / W) % W - Rf, dz = s / (W * W) - Rf;
          const double wk = tw(x + dx - 2 * Jx) * tw(y + dy - 2 * Jy) * tw(z + dz - 2 * Jz);
          if (wk == 0.0 || !inside(f, x + dx, y + dy, z + dz)) continue;
#pragma unroll
          for (int k = 0; k < 9; ++k) acc[k] += wk * A[s * 9 + k];
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const double mr = minvf[3LL * p + r];
#pragma unroll
          for (int k = 0; k < 3; ++k) blk[3 * r + k] -= cc * mr * acc[3 * r + k];
        }
      }
    }
    double* out = psb + (long long)p * NS * 9 + slot;
#pragma unroll
    for (int k = 0; k < 9; ++k) out[k * NS] = blk[k];
  }
}

// B[k][J] = sum_d A[k][d] P_s[k + d][J] per fine interior node k and coarse
// slot b, J = ceil((k - Pr - Rf) / 2) + b per axis; bsb[(p * 9 + 3r + c) * NSB + b].
__global__ void __launch_bounds__(kSetupThreads) k_rap_b(Grid f, const double* __restrict__ stf, int Rf,
                                                         const double* __restrict__ psb, int Pr, Grid c,
                                                         double* __restrict__ bsb) {
  extern __shared__ double sA[];
  const int NA = Pr + 1, NS = NA * NA * NA;
  const int NBA = Pr + Rf + 1, NSB = NBA * NBA * NBA, NG = kSetupThreads / NSB;
  const int W = wide_w(Rf), NB = wide_nb(Rf);
  const long long nint = (long long)(f.lx + 1) * (f.ly + 1) * (f.lz + 1);
  for (long long n0 = (long long)blockIdx.x * NG; n0 < nint; n0 += (long long)gridDim.x * NG) {
    __syncthreads();
    stage_blocks(f, stf, NB, n0, NG, nint, sA);
    __syncthreads();
    const int nl = threadIdx.x / NSB, b = threadIdx.x % NSB;
    if (nl >= NG || n0 + nl >= nint) continue;
    int x, y, z;
    interior_xyz(f, n0 + nl, x, y, z);
    const int p = f.idx(x, y, z);
    const int Jx = ceil_half(x - Pr - Rf) + b % NBA, Jy = ceil_half(y - Pr - Rf) + (b / NBA) % NBA;
    const int Jz = ceil_half(z - Pr - Rf) + b / (NBA * NBA);
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    if (inside(c, Jx, Jy, Jz)) {
      const double* As = sA + (long long)nl * NB * 9;
      for (int s = 0; s < NB; ++s) {
        const int ix = x + s % W - Rf, iy = y + (s / W) % W - Rf, iz = z + s / (W * W) - Rf;
        if (!inside(f, ix, iy, iz)) continue;
        const int ax = Jx - ceil_half(ix - Pr), ay = Jy - ceil_half(iy - Pr), az = Jz - ceil_half(iz - Pr);
        if (ax < 0 || ax > Pr || ay < 0 || ay > Pr || az < 0 || az > Pr) continue;
        const double* P = psb + (long long)f.idx(ix, iy, iz) * NS * 9 + (az * NA + ay) * NA + ax;
        const double* A = As + s * 9;
        double Pv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Pv[k] = P[k * NS];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int cc = 0; cc < 3; ++cc)
            acc[3 * r + cc] += A[3 * r] * Pv[cc] + A[3 * r + 1] * Pv[3 + cc] + A[3 * r + 2] * Pv[6 + cc];
      }
    }
    double* out = bsb + (long long)p * NSB * 9 + b;
#pragma unroll
    for (int k = 0; k < 9; ++k) out[k * NSB] = acc[k];
  }
}

// A_{l+1}[I][I + D] = sum_i P_s[i][I]^T B[i][I + D] for the diagonal and the
// upper offsets D of reach Rc: one CTA per coarse interior node I, P_s[.][I]
// of the (2Pr+1)^3 fine nodes around 2I in shared memory, one thread per D.
constexpr int kRapThreads = 64;
__global__ void __launch_bounds__(kRapThreads) k_rap_c(Grid f, int Rf, const double* __restrict__ psb, int Pr,
                                                       const double* __restrict__ bsb, Grid c, int Rc,
                                                       double* __restrict__ stc) {
  extern __shared__ double sps[];   // [(2Pr+1)^3][9]
  const int NA = Pr + 1, NS = NA * NA * NA;
  const int NBA = Pr + Rf + 1, NSB = NBA * NBA * NBA;
  const int WI = 2 * Pr + 1, NI = WI * WI * WI;
  const int Wc = wide_w(Rc), NBc = wide_nb(Rc), SC = NBc / 2;
  const long long nint = (long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1);
  const long long nc = c.n;
  for (long long node = blockIdx.x; node < nint; node += gridDim.x) {
    int X, Y, Z;
    interior_xyz(c, node, X, Y, Z);
    const int pI = c.idx(X, Y, Z);
    __syncthreads();   // the previous node's readers are done with sps
    for (int e = threadIdx.x; e < NI * 9; e += blockDim.x) {
      const int i = e / 9, k = e % 9;
      const int ix = 2 * X + i % WI - Pr, iy = 2 * Y + (i / WI) % WI - Pr, iz = 2 * Z + i / (WI * WI) - Pr;
      double v = 0.0;
      if (inside(f, ix, iy, iz)) {
        const int ax = X - ceil_half(ix - Pr), ay = Y - ceil_half(iy - Pr), az = Z - ceil_half(iz - Pr);
        v = psb[((long long)f.idx(ix, iy, iz) * 9 + k) * NS + (az * NA + ay) * NA + ax];
      }
      sps[e] = v;
    }
    __syncthreads();
    for (int u = threadIdx.x; u <= SC; u += blockDim.x) {
      const int s = SC + u;   // center and upper offsets
      const int Dx = s % Wc - Rc, Dy = (s / Wc) % Wc - Rc, Dz = s / (Wc * Wc) - Rc;
      const int Jx = X + Dx, Jy = Y + Dy, Jz = Z + Dz;
      double acc[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) acc[k] = 0.0;
      if (inside(c, Jx, Jy, Jz)) {
        for (int i = 0; i < NI; ++i) {
          const int ix = 2 * X + i % WI - Pr, iy = 2 * Y + (i / WI) % WI - Pr, iz = 2 * Z + i / (WI * WI) - Pr;
          if (!inside(f, ix, iy, iz)) continue;
          const int bx = Jx - ceil_half(ix - Pr - Rf), by = Jy - ceil_half(iy - Pr - Rf);
          const int bz = Jz - ceil_half(iz - Pr - Rf);
          if (bx < 0 || bx >= NBA || by < 0 || by >= NBA || bz < 0 || bz >= NBA) continue;
          const double* P = sps + i * 9;
          const double* B = bsb + (long long)f.idx(ix, iy, iz) * NSB * 9 + (bz * NBA + by) * NBA + bx;
          double Bv[9];
#pragma unroll
          for (int k = 0; k < 9; ++k) Bv[k] = B[k * NSB];
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
              acc[3 * r + cc] += P[r] * Bv[cc] + P[3 + r] * Bv[3 + cc] + P[6 + r] * Bv[6 + cc];
        }
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) stc[((long long)s * 9 + k) * nc + pI] = acc[k];
    }
  }
}

// ---- set-up products with the reaches fixed at compile time ------------------
// The hierarchies this library builds use two (R_l, Pr) pairs: (1, 2) for the
// smoothed transfer from a 27-block level and (2, 1) for the trilinear
// transfer below a 125-block level, both giving R_{l+1} = 2.  The kernels
// below compute exactly the sums of k_prolong_blocks / k_rap_b (the same
// terms, added in the same order) but with W, NB and the slot counts as
// constants and the contributing offsets found per axis instead of by testing
// all NB of them: the generic kernels spend most of their time on runtime
// divisions and range tests, not on the FP64 products.  (The coarse product
// stays generic: a compile-time version held twice the registers and ran
// slower; so did a B product that staged the neighbours' P_s rows in shared
// memory.)

// Padded-storage index and interior coordinates of the interior nodes
// [n0, n0 + NG) of grid f (-1 past the end), for a CTA's staging.
template <int NG>
__device__ __forceinline__ void node_table(const Grid& f, long long n0, long long nint, int* sp) {
  if (threadIdx.x < NG) {
    int v = -1;
    if (n0 + threadIdx.x < nint) {
      int x, y, z;
      interior_xyz(f, n0 + threadIdx.x, x, y, z);
      v = f.idx(x, y, z);
    }
    sp[threadIdx.x] = v;
  }
}

template <int RF, int PR, bool SMOOTHED>
__global__ void __launch_bounds__(kSetupThreads) k_prolong_blocks_t(Grid f, const double* __restrict__ stf,
                                                                    const uint8_t* __restrict__ fm,
                                                                    const double* __restrict__ minvf,
                                                                    const double* __restrict__ cdev, Grid c,
                                                                    double* __restrict__ psb) {
  constexpr int NA = PR + 1, NS = NA * NA * NA, NG = kSetupThreads / NS;
  constexpr int W = 2 * RF + 1, NB = W * W * W;
  __shared__ double sA[SMOOTHED ? NG * NB * 9 : 1];
  __shared__ int sp[NG];
  const long long nint = (long long)(f.lx + 1) * (f.ly + 1) * (f.lz + 1);
  const long long nf = f.n;
  const double cc = SMOOTHED ? *cdev : 0.0;
  const int sxy = f.px * f.py;
  for (long long n0 = (long long)blockIdx.x * NG; n0 < nint; n0 += (long long)gridDim.x * NG) {
    __syncthreads();   // the previous group's readers are done with sA / sp
    node_table<NG>(f, n0, nint, sp);
    __syncthreads();
    if (SMOOTHED) {
      for (int e = threadIdx.x; e < NG * NB * 9; e += blockDim.x) {
        const int nl = e / (NB * 9), rem = e - nl * (NB * 9);
        const int p = sp[nl];
        sA[e] = p >= 0 ? stf[(long long)rem * nf + p] : 0.0;
      }
      __syncthreads();
    }
    const int nl = threadIdx.x / NS, slot = threadIdx.x - nl * NS;
    if (nl >= NG) continue;
    const int p = sp[nl];
    if (p < 0) continue;
    const int z = p / sxy - 1, rxy = p - (z + 1) * sxy, y = rxy / f.px - 1, x = rxy - (y + 1) * f.px - 1;
    const int ax = slot % NA, ay = (slot / NA) % NA, az = slot / (NA * NA);
    const int Jx = ceil_half(x - PR) + ax, Jy = ceil_half(y - PR) + ay, Jz = ceil_half(z - PR) + az;
    double blk[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) blk[k] = 0.0;
    if (inside(c, Jx, Jy, Jz)) {
      const uint8_t m = fm[p];
      const double w = tw(x - 2 * Jx) * tw(y - 2 * Jy) * tw(z - 2 * Jz);
#pragma unroll
      for (int r = 0; r < 3; ++r)
        if ((m >> r) & 1) blk[4 * r] = w;
      if (SMOOTHED && cc != 0.0 && m) {
        double wx[W], wy[W], wz[W];
#pragma unroll
        for (int d = 0; d < W; ++d) {
          const int ix = x + d - RF, iy = y + d - RF, iz = z + d - RF;
          wx[d] = (ix >= 0 && ix <= f.lx) ? tw(ix - 2 * Jx) : 0.0;
          wy[d] = (iy >= 0 && iy <= f.ly) ? tw(iy - 2 * Jy) : 0.0;
          wz[d] = (iz >= 0 && iz <= f.lz) ? tw(iz - 2 * Jz) : 0.0;
        }
        double acc[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[k] = 0.0;
        const double* A = sA + nl * NB * 9;
#pragma unroll
        for (int dz = 0; dz < W; ++dz) {
          if (wz[dz] == 0.0) continue;
#pragma unroll
          for (int dy = 0; dy < W; ++dy) {
            if (wy[dy] == 0.0) continue;
#pragma unroll
            for (int dx = 0; dx < W; ++dx) {
              if (wx[dx] == 0.0) continue;
              const double wk = wx[dx] * wy[dy] * wz[dz];
              const double* As = A + ((dz * W + dy) * W + dx) * 9;
#pragma unroll
              for (int k = 0; k < 9; ++k) acc[k] += wk * As[k];
            }
          }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const double mr = minvf[3LL * p + r];
#pragma unroll
          for (int k = 0; k < 3; ++k) blk[3 * r + k] -= cc * mr * acc[3 * r + k];
        }
      }
    }
    double* out = psb + (long long)p * NS * 9 + slot;
#pragma unroll
    for (int k = 0; k < 9; ++k) out[k * NS] = blk[k];
  }
}

template <int RF, int PR>
__global__ void __launch_bounds__(kSetupThreads, 4) k_rap_b_t(Grid f, const double* __restrict__ stf,
                                                           const double* __restrict__ psb, Grid c,
                                                           double* __restrict__ bsb) {
  constexpr int NA = PR + 1, NS = NA * NA * NA;
  constexpr int NBA = PR + RF + 1, NSB = NBA * NBA * NBA, NG = kSetupThreads / NSB;
  constexpr int W = 2 * RF + 1, NB = W * W * W;
  __shared__ double sA[NG * NB * 9];
  __shared__ int sp[NG];
  const long long nint = (long long)(f.lx + 1) * (f.ly + 1) * (f.lz + 1);
  const long long nf = f.n;
  const int sxy = f.px * f.py;
  for (long long n0 = (long long)blockIdx.x * NG; n0 < nint; n0 += (long long)gridDim.x * NG) {
    __syncthreads();
    node_table<NG>(f, n0, nint, sp);
    __syncthreads();
    for (int e = threadIdx.x; e < NG * NB * 9; e += blockDim.x) {
      const int nl = e / (NB * 9), rem = e - nl * (NB * 9);
      const int p = sp[nl];
      sA[e] = p >= 0 ? stf[(long long)rem * nf + p] : 0.0;
    }
    __syncthreads();
    const int nl = threadIdx.x / NSB, b = threadIdx.x - nl * NSB;
    if (nl >= NG) continue;
    const int p = sp[nl];
    if (p < 0) continue;
    const int z = p / sxy - 1, rxy = p - (z + 1) * sxy, y = rxy / f.px - 1, x = rxy - (y + 1) * f.px - 1;
    const int Jx = ceil_half(x - PR - RF) + b % NBA, Jy = ceil_half(y - PR - RF) + (b / NBA) % NBA;
    const int Jz = ceil_half(z - PR - RF) + b / (NBA * NBA);
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    if (inside(c, Jx, Jy, Jz)) {
      // per axis: slot of J in the P_s row of fine node x + d - RF (-1: none)
      int sx[W], sy[W], sz[W];
#pragma unroll
      for (int d = 0; d < W; ++d) {
        const int ix = x + d - RF, iy = y + d - RF, iz = z + d - RF;
        const int ax = Jx - ceil_half(ix - PR), ay = Jy - ceil_half(iy - PR), az = Jz - ceil_half(iz - PR);
        sx[d] = (ix >= 0 && ix <= f.lx && ax >= 0 && ax <= PR) ? ax : -1;
        sy[d] = (iy >= 0 && iy <= f.ly && ay >= 0 && ay <= PR) ? ay : -1;
        sz[d] = (iz >= 0 && iz <= f.lz && az >= 0 && az <= PR) ? az : -1;
      }
      const double* As = sA + nl * NB * 9;
#pragma unroll
      for (int dz = 0; dz < W; ++dz) {
        if (sz[dz] < 0) continue;
#pragma unroll
        for (int dy = 0; dy < W; ++dy) {
          if (sy[dy] < 0) continue;
#pragma unroll
          for (int dx = 0; dx < W; ++dx) {
            if (sx[dx] < 0) continue;
            const int q = p + (dx - RF) + f.px * ((dy - RF) + f.py * (dz - RF));
            const double* P = psb + (long long)q * NS * 9 + (sz[dz] * NA + sy[dy]) * NA + sx[dx];
            const double* A = As + ((dz * W + dy) * W + dx) * 9;
            double Pv[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) Pv[k] = __ldg(P + k * NS);
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
              for (int cc = 0; cc < 3; ++cc)
                acc[3 * r + cc] += A[3 * r] * Pv[cc] + A[3 * r + 1] * Pv[3 + cc] + A[3 * r + 2] * Pv[6 + cc];
          }
        }
      }
    }
    double* out = bsb + (long long)p * NSB * 9 + b;
#pragma unroll
    for (int k = 0; k < 9; ++k) out[k * NSB] = acc[k];
  }
}

// Lower offsets from the upper ones: block (s, p)[r][c] = block (NB-1-s, p + off(s))[c][r].
__global__ void k_wide_mirror(Grid c, int R, double* __restrict__ stc) {
  const int W = wide_w(R), NB = wide_nb(R), SC = NB / 2;
  const long long nint = (long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1);
  const long long nc = c.n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)SC * nint;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t / nint);
    int X, Y, Z;
    interior_xyz(c, t % nint, X, Y, Z);
    const int p = c.idx(X, Y, Z);
    const int MX = X + s % W - R, MY = Y + (s / W) % W - R, MZ = Z + s / (W * W) - R;
    const bool in = inside(c, MX, MY, MZ);
    const long long q = in ? c.idx(MX, MY, MZ) : 0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
        stc[((long long)s * 9 + 3 * r + cc) * nc + p] =
            in ? stc[((long long)(NB - 1 - s) * 9 + 3 * cc + r) * nc + q] : 0.0;
  }
}

// D_{l+1} from the diagonal, rows / columns of the other DOFs zeroed, Minv.
__global__ void k_wide_mask_from_diag(Grid c, int R, const double* __restrict__ st, uint8_t* __restrict__ cmask) {
  const int SC = wide_nb(R) / 2;
  const long long n = c.n;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < c.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(c, p, x, y, z);
    uint8_t m = 0;
    if (inside(c, x, y, z))
      for (int r = 0; r < 3; ++r)
        if (st[((long long)SC * 9 + 4 * r) * n + p] > 0.0) m |= (uint8_t)(1 << r);
    cmask[p] = m;
  }
}

__global__ void k_wide_apply_mask(Grid c, int R, double* __restrict__ st, const uint8_t* __restrict__ cmask,
                                  double* __restrict__ minv3) {
  const int W = wide_w(R), NB = wide_nb(R), SC = NB / 2;
  const long long n = c.n;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < c.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(c, p, x, y, z);
    const bool in = inside(c, x, y, z);
    const uint8_t mp = cmask[p];
    for (int s = 0; s < NB; ++s) {
      const int qx = x + s % W - R, qy = y + (s / W) % W - R, qz = z + s / (W * W) - R;
      const uint8_t mq = (in && inside(c, qx, qy, qz)) ? cmask[c.idx(qx, qy, qz)] : (uint8_t)0;
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc)
          if (!(in && ((mp >> r) & 1) && ((mq >> cc) & 1))) st[((long long)s * 9 + 3 * r + cc) * n + p] = 0.0;
    }
    for (int r = 0; r < 3; ++r) {
      const double d = st[((long long)SC * 9 + 4 * r) * n + p];
      minv3[3LL * p + r] = ((mp >> r) & 1) && d != 0.0 ? 1.0 / d : 0.0;
    }
  }
}

// ---- scaled symmetric storage ----------------------------------------------
template <typename S> __device__ __forceinline__ S to_s(double v);
template <> __device__ __forceinline__ float to_s<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ double to_s<double>(double v) { return v; }
template <> __device__ __forceinline__ __half to_s<__half>(double v) { return __double2half(v); }

template <typename S, int R>
__global__ void k_wide_compress(Grid g, const double* __restrict__ st, const uint8_t* __restrict__ mask,
                                S* __restrict__ stc, typename WideLayout<S, R>::Q* __restrict__ sqrtd) {
  using L = WideLayout<S, R>;
  using Q = typename L::Q;
  constexpr int W = 2 * R + 1, NB = W * W * W, SC = NB / 2, G = L::G;
  const long long n = g.n;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x) {
    int x, y, z;
    decode(g, p, x, y, z);
    const bool in = inside(g, x, y, z);
    double sp[3];
    for (int r = 0; r < 3; ++r) {
      const double d = in ? st[((long long)SC * 9 + 4 * r) * n + p] : 0.0;
      sp[r] = (in && ((mask[p] >> r) & 1) && d > 0.0) ? 1.0 / sqrt(d) : 0.0;
      sqrtd[3LL * p + r] = (Q)(sp[r] > 0.0 ? 1.0 / sp[r] : 0.0);
    }
    for (int u = 0; u < L::G * L::NJ; ++u) {
      const long long v = (long long)p * G + u % G;
      const int k0 = 9 * (u / G);
      if (u >= L::NBLK) {
        for (int k = 0; k < 9; ++k) stc[L::off(v, k0 + k)] = to_s<S>(0.0);
        continue;
      }
      const int s = (u == L::NU) ? SC : SC + 1 + u;
      const int qx = x + s % W - R, qy = y + (s / W) % W - R, qz = z + s / (W * W) - R;
      double sq[3] = {0.0, 0.0, 0.0};
      if (in && inside(g, qx, qy, qz)) {
        const int q = g.idx(qx, qy, qz);
        for (int cc = 0; cc < 3; ++cc) {
          const double d = st[((long long)SC * 9 + 4 * cc) * n + q];
          sq[cc] = (((mask[q] >> cc) & 1) && d > 0.0) ? 1.0 / sqrt(d) : 0.0;
        }
      }
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
          const double val = (sp[r] != 0.0 && sq[cc] != 0.0) ? st[((long long)s * 9 + 3 * r + cc) * n + p] * sp[r] * sq[cc]
                                                             : 0.0;
          stc[L::off(v, k0 + 3 * r + cc)] = to_s<S>(val);
        }
    }
    for (int gl = 0; gl < G; ++gl)
      for (int k = 9 * L::NJ; k < L::NVL; ++k) stc[L::off((long long)p * G + gl, k)] = to_s<S>(0.0);
  }
}

// One 16-byte chunk, unpacked to the accumulation type.
template <typename S, typename A> struct WChunk;
template <> struct WChunk<__half, float> {
  float v[8];
  __device__ __forceinline__ void load(const __half* base) {
    const uint4 w = __ldg(reinterpret_cast<const uint4*>(base));
    const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      __half2 h;
      memcpy(&h, &ws[i], 4);
      const float2 f = __half22float2(h);
      v[2 * i] = f.x;
      v[2 * i + 1] = f.y;
    }
  }
};
template <> struct WChunk<float, float> {
  float v[4];
  __device__ __forceinline__ void load(const float* base) {
    const float4 w = __ldg(reinterpret_cast<const float4*>(base));
    v[0] = w.x; v[1] = w.y; v[2] = w.z; v[3] = w.w;
  }
};
template <> struct WChunk<double, double> {
  double v[2];
  __device__ __forceinline__ void load(const double* base) {
    const double2 w = __ldg(reinterpret_cast<const double2*>(base));
    v[0] = w.x; v[1] = w.y;
  }
};

// The 9 values of slot jj of virtual node v (chunks straddled as needed).
template <typename S, typename A, typename L, int JJ>
__device__ __forceinline__ void load_block(const S* __restrict__ stc, long long v, A (&blk)[9]) {
  constexpr int VPC = L::VPC, K0 = 9 * JJ;
#pragma unroll
  for (int j = K0 / VPC; j <= (K0 + 8) / VPC; ++j) {
    WChunk<S, A> ch;
    ch.load(stc + L::off(v, j * VPC));
#pragma unroll
    for (int i = 0; i < VPC; ++i) {
      const int k = j * VPC + i;
      if (k >= K0 && k < K0 + 9) blk[k - K0] = ch.v[i];
    }
  }
}

template <typename S, typename A, typename L, int JJ>
struct WideBlocks {
  // acc (this node's rows) += own block u = lane + G*JJ applied to the
  // neighbour p + off(s); for an upper block also the transposed upper block
  // u of the node p - off(s) (lane and slot are the same there).
  template <typename VF>
  __device__ __forceinline__ static void run(const S* __restrict__ stc, const Grid& g, int p, int lane, int x, int y,
                                             int z, A (&acc)[3], VF V) {
    constexpr int R = (L::W - 1) / 2, W = L::W, SC = L::NB / 2;
    const int u = lane + L::G * JJ;
    if (u < L::NBLK) {
      const int s = (u == L::NU) ? SC : SC + 1 + u;
      const int dx = s % W - R, dy = (s / W) % W - R, dz = s / (W * W) - R;
      const long long v = (long long)p * L::G + lane;
      if (inside(g, x + dx, y + dy, z + dz)) {
        const int q = g.idx(x + dx, y + dy, z + dz);
        A blk[9];
        load_block<S, A, L, JJ>(stc, v, blk);
        const A v0 = V(q, 0), v1 = V(q, 1), v2 = V(q, 2);
#pragma unroll
        for (int r = 0; r < 3; ++r) acc[r] += blk[3 * r] * v0 + blk[3 * r + 1] * v1 + blk[3 * r + 2] * v2;
      }
      if (u < L::NU && inside(g, x - dx, y - dy, z - dz)) {
        const int q = g.idx(x - dx, y - dy, z - dz);
        A blk[9];
        load_block<S, A, L, JJ>(stc, (long long)q * L::G + lane, blk);
        const A w0 = V(q, 0), w1 = V(q, 1), w2 = V(q, 2);
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] += blk[c] * w0 + blk[3 + c] * w1 + blk[6 + c] * w2;
      }
    }
    if constexpr (JJ + 1 < L::NJ) WideBlocks<S, A, L, JJ + 1>::run(stc, g, p, lane, x, y, z, acc, V);
  }
};

// y = mask(D^1/2 A~ D^1/2 u) with the epilogues of the other level kernels
// (APPLY, SMOOTH with the Chebyshev step fields, RESID; a null rhs reads as
// zero).  G = 8 lanes per node: each lane applies its own blocks and the
// transposed blocks of the same lane and slot of the lower neighbours, the
// partial sums meet through warp shuffles, and lanes 0..2 write component
// 0..2 of the node.
template <typename T, typename S, int R, int EPI>
__global__ void __launch_bounds__(128) k_wide_op(Grid g, OpArgs a, const S* __restrict__ stc,
                                                 const T* __restrict__ sqd) {
  using L = WideLayout<S, R>;
  using A = typename std::conditional<sizeof(T) == 8, double, float>::type;
  constexpr int G = L::G;
  KrylovState* ks = a.ks;
  if (ks && ks->done) return;
  const T* __restrict__ u = (const T*)a.u;
  T* out = (T*)a.out;
  const T* b = (const T*)a.b;
  const T* __restrict__ minv = (const T*)a.minv;
  const uint8_t* __restrict__ mask = a.mask;
  const T w = a.omega_dev ? (T)(*a.omega_dev) : (T)a.omega;
  const T* dprev = (const T*)a.dprev;
  T* dout = (T*)a.dout;
  const T c1 = a.c1_dev ? (T)(*a.c1_dev) : (T)0;
  auto V = [&](int q, int c) -> A { return (A)__ldg(sqd + 3LL * q + c) * (A)__ldg(u + 3LL * q + c); };
  double dot = 0.0;
  // whole warps iterate together (the shuffles need every lane)
  const long long nv = ((long long)g.n * G + 31) / 32 * 32;
  for (long long vv = blockIdx.x * (long long)blockDim.x + threadIdx.x; vv < nv;
       vv += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(vv / G), lane = (int)(vv % G);
    int x = -1, y = -1, z = -1;
    if (p < g.n) decode(g, p, x, y, z);
    const bool in = p < g.n && inside(g, x, y, z);
    const uint8_t m = in ? mask[p] : (uint8_t)0;
    A acc[3] = {(A)0, (A)0, (A)0};
    if (m) WideBlocks<S, A, L, 0>::run(stc, g, p, lane, x, y, z, acc, V);
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    }
    if (!in || lane >= 3) continue;
    const int c = lane;
    const long long pc = 3LL * p + c;
    const A ac = c == 0 ? acc[0] : (c == 1 ? acc[1] : acc[2]);
    const T kc = ((m >> c) & 1) ? (T)(ac * (A)sqd[pc]) : (T)0;
    const T bc = b ? b[pc] : (T)0;
    if (EPI == EPI_APPLY) {
      out[pc] = kc;
      if (a.dot_partials) dot += (double)u[pc] * (double)kc;
    } else if (EPI == EPI_SMOOTH) {
      const T u0 = u[pc];
      T o = u0 + (((m >> c) & 1) ? w * (minv[pc] * (bc - kc)) : (T)0);
      if (dprev) o += c1 * dprev[pc];
      out[pc] = o;
      if (dout) dout[pc] = o - u0;
    } else {
      out[pc] = bc - kc;
    }
  }
  if (EPI == EPI_APPLY && a.dot_partials && ks) reduce_and_finalize(dot, a.dot_partials, ks, a.dot_slot, nullptr);
}

// Dense row-major A of a reach-R level (reference node order, DOF 3*node + c),
// identity rows on non-free DOFs.
__global__ void k_wide_dense_assemble(Grid c, int R, const double* __restrict__ st, const uint8_t* __restrict__ cm,
                                      double* __restrict__ A, int n) {
  const int W = wide_w(R), NB = wide_nb(R), SC = NB / 2;
  const int nx1 = c.lx + 1, ny1 = c.ly + 1;
  const long long nint = (long long)nx1 * ny1 * (c.lz + 1);
  const long long ns = c.n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nint * NB;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / NB), s = (int)(t % NB);
    int x, y, z;
    interior_xyz(c, r, x, y, z);
    const int X = x + s % W - R, Y = y + (s / W) % W - R, Z = z + s / (W * W) - R;
    if (!inside(c, X, Y, Z)) continue;
    const int q = X + nx1 * (Y + ny1 * Z);
    const int p = c.idx(x, y, z);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        A[(long long)(3 * r + i) * n + 3 * q + j] = st[((long long)s * 9 + 3 * i + j) * ns + p];
    if (s == SC) {
      const uint8_t m = cm[p];
      for (int i = 0; i < 3; ++i)
        if (!((m >> i) & 1)) A[(long long)(3 * r + i) * n + 3 * r + i] = 1.0;
    }
  }
}

__global__ void k_smoothing_coef(const double* __restrict__ lambda, double* __restrict__ coef) {
  const double l = *lambda;
  *coef = l > 0.0 ? (4.0 / 3.0) / l : 0.0;
}

}  // namespace

// ---- launchers ---------------------------------------------------------------
void launch_smoothing_coef(const double* lambda, double* coef, cudaStream_t st) {
  launch_k(k_smoothing_coef, 1, 1, 0, st, lambda, coef);
}

size_t wide_prolong_count(const Grid& f, int Pr) { return (size_t)f.n * (Pr + 1) * (Pr + 1) * (Pr + 1) * 9; }
size_t wide_rapb_count(const Grid& f, int Pr, int Rf) {
  const size_t a = (size_t)(Pr + Rf + 1);
  return (size_t)f.n * a * a * a * 9;
}

void launch_wide_galerkin(const Grid& f, const double* stf, int Rf, const uint8_t* fmask, const double* minvf,
                          const double* cdev, int Pr, const Grid& c, double* stc, int Rc, double* psb, double* bsb,
                          cudaStream_t st) {
  const long long nintf = (long long)(f.lx + 1) * (f.ly + 1) * (f.lz + 1);
  const long long nintc = (long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1);
  const int NS = (Pr + 1) * (Pr + 1) * (Pr + 1), NBA = Pr + Rf + 1, NSB = NBA * NBA * NBA;
  const int ngp = kSetupThreads / NS, ngb = kSetupThreads / NSB;
  const int gp = (int)std::min<long long>((nintf + ngp - 1) / ngp, 148LL * 64);
  const int gb = (int)std::min<long long>((nintf + ngb - 1) / ngb, 148LL * 64);
  const int gc = (int)std::min<long long>(nintc, 148LL * 256);
  const size_t smem_c = sizeof(double) * (2 * Pr + 1) * (2 * Pr + 1) * (2 * Pr + 1) * 9;   // k_rap_c
  // the two pairs the hierarchy builds (see k_prolong_blocks_t)
#define VF_WIDE_FIXED(RF_, PR_, SM_)                                                                          \
  do {                                                                                                        \
    launch_k(k_prolong_blocks_t<RF_, PR_, SM_>, gp, kSetupThreads, 0, st, f, stf, fmask, minvf, cdev, c, psb); \
    launch_k(k_rap_b_t<RF_, PR_>, gb, kSetupThreads, 0, st, f, stf, (const double*)psb, c, bsb);             \
    launch_k(k_rap_c, gc, kRapThreads, smem_c, st, f, Rf, (const double*)psb, Pr, (const double*)bsb, c, Rc, stc); \
    launch_k(k_wide_mirror, blocks_for((long long)(wide_nb(Rc) / 2) * nintc, 128), 128, 0, st, c, Rc, stc);    \
    return;                                                                                                   \
  } while (0)
  if (Rf == 1 && Pr == 2 && Rc == 2 && cdev) VF_WIDE_FIXED(1, 2, true);
  if (Rf == 2 && Pr == 1 && Rc == 2 && !cdev) VF_WIDE_FIXED(2, 1, false);
#undef VF_WIDE_FIXED
  const size_t smem_p = cdev ? sizeof(double) * ngp * wide_nb(Rf) * 9 : 0;
  const size_t smem_b = sizeof(double) * ngb * wide_nb(Rf) * 9;
  launch_k(k_prolong_blocks, (int)std::min<long long>((nintf + ngp - 1) / ngp, 148LL * 64), kSetupThreads, smem_p, st,
           f, stf, Rf, fmask, minvf, cdev, Pr, c, psb);
  launch_k(k_rap_b, (int)std::min<long long>((nintf + ngb - 1) / ngb, 148LL * 64), kSetupThreads, smem_b, st, f, stf,
           Rf, psb, Pr, c, bsb);
  const int WI = 2 * Pr + 1;
  const size_t smem = sizeof(double) * WI * WI * WI * 9;
  launch_k(k_rap_c, (int)std::min<long long>(nintc, 148LL * 256), kRapThreads, smem, st, f, Rf, psb, Pr, bsb, c, Rc,
           stc);
  launch_k(k_wide_mirror, blocks_for((long long)(wide_nb(Rc) / 2) * nintc, 128), 128, 0, st, c, Rc, stc);
}

void launch_wide_mask(const Grid& c, int R, double* stc, uint8_t* cmask, double* minv3, cudaStream_t st) {
  launch_k(k_wide_mask_from_diag, blocks_for(c.n, 256), 256, 0, st, c, R, stc, cmask);
  launch_k(k_wide_apply_mask, blocks_for(c.n, 128), 128, 0, st, c, R, stc, cmask, minv3);
}

template <typename S, int R>
void launch_wide_compress(const Grid& g, const double* st, const uint8_t* mask, S* stc,
                          typename WideLayout<S, R>::Q* sqrtd, cudaStream_t st_) {
  launch_k(k_wide_compress<S, R>, blocks_for(g.n, 128), 128, 0, st_, g, st, mask, stc, sqrtd);
}
template void launch_wide_compress<__half, 2>(const Grid&, const double*, const uint8_t*, __half*, float*, cudaStream_t);
template void launch_wide_compress<float, 2>(const Grid&, const double*, const uint8_t*, float*, float*, cudaStream_t);
template void launch_wide_compress<double, 2>(const Grid&, const double*, const uint8_t*, double*, double*, cudaStream_t);

template <typename T, typename S, int R>
void launch_wide_op(const Grid& g, int epi, const OpArgs& a, const S* stc, const T* sqrtd, cudaStream_t st) {
  const int blocks = wide_op_grid_blocks(g);
  if (epi == EPI_APPLY) launch_k(k_wide_op<T, S, R, EPI_APPLY>, blocks, 128, 0, st, g, a, stc, sqrtd);
  else if (epi == EPI_SMOOTH) launch_k(k_wide_op<T, S, R, EPI_SMOOTH>, blocks, 128, 0, st, g, a, stc, sqrtd);
  else launch_k(k_wide_op<T, S, R, EPI_RESID>, blocks, 128, 0, st, g, a, stc, sqrtd);
}
template void launch_wide_op<float, __half, 2>(const Grid&, int, const OpArgs&, const __half*, const float*, cudaStream_t);
template void launch_wide_op<float, float, 2>(const Grid&, int, const OpArgs&, const float*, const float*, cudaStream_t);
template void launch_wide_op<double, double, 2>(const Grid&, int, const OpArgs&, const double*, const double*,
                                                cudaStream_t);
int wide_op_grid_blocks(const Grid& g) { return blocks_for((long long)g.n * 8, 128, 148LL * 32); }

int wide_dense_assemble(const Grid& c, int R, const double* stencil, const uint8_t* cmask, double* A, int n,
                        cudaStream_t st) {
  cudaMemsetAsync(A, 0, sizeof(double) * (size_t)n * n, st);
  const long long work = (long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1) * wide_nb(R);
  launch_k(k_wide_dense_assemble, blocks_for(work, 256, 148LL * 256), 256, 0, st, c, R, stencil, cmask, A, n);
  return 0;
}

}  // namespace vf
