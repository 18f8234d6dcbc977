// Fine-level hex8 operator, modal z-marching form (default kernel).
//
// Same operator as vf_matvec.cu (y_n = sum_e E_e Ke[a_e(n), :] u_e, the
// reference's core/multigrid.py:318-341), computed with far fewer
// instructions:
//
// * The trilinear field of a voxel is expanded in the tensor-product basis
//   xi^p eta^q zeta^r (p, q, r in {0,1}); the coefficients are an
//   unnormalised 3-D Walsh-Hadamard transform of the 8 corner values.  With
//   2x2x2 Gauss quadrature (exact here) these basis functions are orthogonal,
//   so the strain energy is a sum of independent per-mode quadratic forms and
//   Ke u = H^T B(H u) with B a handful of FMAs per mode (weights 3^-|m|).
//   The factorisation reproduces the reference Ke to rounding (tests compare
//   against the oracle's 24x24 Ke).
// * The transform is separable and shared: a CTA owns a 32 x TY tile of node
//   columns and marches along z.  Per z-plane a thread forms the 2-D (x,y)
//   transform of its voxel column's face once; the voxel between planes k-1
//   and k combines the two faces (z stage); the transposed transform goes back
//   face by face, and the four face corners are summed across neighbouring
//   threads through shared memory -- each node output is written by exactly
//   one thread, in a fixed order (deterministic).
// * Every streamed input (halo plane of u, the voxel modulus, the epilogue's
//   rhs and inverse diagonal) is staged by cp.async into a 4-deep shared-memory
//   ring two planes ahead, so global latency overlaps the arithmetic without
//   holding registers; 2 CTAs of 256 threads fit per SM.
// * FP32: every thread carries TWO independent z-ranges packed in float2, so
//   the arithmetic is the sm_100 packed FP32 instructions (__fadd2/__fmul2/
//   __ffma2) with no cross-lane shuffles.  FP64: one z-range per thread.
//
// Tile bookkeeping: thread (tx, ty) owns node column (X0-1+tx, Y0-1+ty) and
// the voxel column with that lower corner; outputs are produced for
// tx >= 1, ty >= 1 (a node needs the four voxel columns around it), so a tile
// advances by (31, TY-1) columns.  One node row/column of halo is loaded.
#include <atomic>
#include <cmath>

#include "vf_common.cuh"
#include "vf_reduce.cuh"
#include "vf_modal.cuh"

namespace vf {

namespace {

using namespace modal;

constexpr int TX = 32;
constexpr int NSTAGE = 4;

// Asynchronous copy of one element (ES = 4 or 8 bytes), zero-filled when invalid.
template <unsigned ES>
__device__ __forceinline__ void cp_el(unsigned dst, const void* src, bool ok) {
  static_assert(ES == 4 || ES == 8, "cp.async element size");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(src), "n"(ES), "r"(ok ? (int)ES : 0));
}

// Shared-memory layout of one pipeline stage (one z-plane per lane); arrays a
// variant does not use shrink to one row.
template <typename P, int TY, bool LAME, int EPI>
struct Stage {
  P u[3][TY + 1][TX + 1];                   // node values, halo tile
  P e[TY][TX];                              // modulus (or lambda) of the voxel
  P m[LAME ? TY : 1][TX];                   // mu (per-voxel Poisson ratio)
  P b[3][EPI != EPI_APPLY ? TY : 1][TX];    // right-hand side (SMOOTH / RESID)
  P d[3][EPI == EPI_SMOOTH ? TY : 1][TX];   // inverse diagonal (SMOOTH)
};

template <typename T, bool LAME, int EPI, int TY>
__global__ void __launch_bounds__(TX * TY, 2) k_modal_op(Grid g, OpArgs a, ModalConst mc, int zchunk) {
  using O = Pack<T>;
  using P = typename O::P;
  using St = Stage<P, TY, LAME, EPI>;
  constexpr int L = O::L;
  constexpr int NTH = TX * TY;
  constexpr int NHALO = (TX + 1) * (TY + 1);
  constexpr int NLOAD = (NHALO + NTH - 1) / NTH;
  constexpr unsigned ES = sizeof(T);
  KrylovState* ks = a.ks;
  if (ks && ks->done) return;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  St* stg = reinterpret_cast<St*>(smem_raw);
  P (*s_c)[3][TY][TX] = reinterpret_cast<P (*)[3][TY][TX]>(smem_raw + NSTAGE * sizeof(St));
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smem_raw);

  const T* __restrict__ u = (const T*)a.u;
  T* __restrict__ out = (T*)a.out;
  const T* __restrict__ bvec = (const T*)a.b;
  const T* __restrict__ minv = (const T*)a.minv;
  const T* __restrict__ Ev = (const T*)a.E;
  const T* __restrict__ MUv = (const T*)a.mu;
  const uint8_t* __restrict__ mask = a.mask;
  const T w = a.omega_dev ? (T)(*a.omega_dev) : (T)a.omega;
  const T* dprev = (const T*)a.dprev;
  T* dout = (T*)a.dout;
  const T c1 = a.c1_dev ? (T)(*a.c1_dev) : (T)0;

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TY - 1);
  const int Xc = X0 - 1 + tx, Yc = Y0 - 1 + ty;
  const int zb = blockIdx.z * zchunk;
  const int ze = min(zb + zchunk, g.lz + 1);
  const int H = (ze - zb + L - 1) / L;
  const int sz = g.px * g.py;   // 3 * px * py * pz < 2^31 (checked at creation)
  const bool col_in = (Xc + 1 < g.px) && (Yc + 1 < g.py);
  const int colbase = col_in ? (Yc + 1) * g.px + (Xc + 1) : 0;
  const bool out_col = tx >= 1 && ty >= 1 && Xc <= g.lx && Yc <= g.ly;

  // Step s reads node plane z = z0[l] + s of lane l (storage plane z + 1),
  // valid while z + 1 < pz  <=>  s < smax[l]; output planes of the lane are
  // z0[l] + 1 .. oend[l] - 1.
  int z0[L], smax[L], oend[L];
#pragma unroll
  for (int l = 0; l < L; ++l) {
    z0[l] = zb + l * H - 1;
    smax[l] = g.pz - (z0[l] + 1);
    oend[l] = min(min(zb + l * H + H, ze), g.lz + 1);
  }
  // per-thread copy descriptors of the halo tile: global offset in plane, shared offset
  int gu[NLOAD], su[NLOAD];
  bool hok[NLOAD];
#pragma unroll
  for (int q = 0; q < NLOAD; ++q) {
    const int e = tid + q * NTH;
    const int i = e % (TX + 1), j = e / (TX + 1);
    const int x = X0 - 1 + i, y = Y0 - 1 + j;
    hok[q] = (e < NHALO) && (x + 1 < g.px) && (y + 1 < g.py);
    gu[q] = hok[q] ? 3 * ((y + 1) * g.px + (x + 1)) : 0;
    su[q] = (e < NHALO) ? (int)(((char*)&stg[0].u[0][j][i]) - (char*)stg) : 0;
  }
  const int so_e = (int)(((char*)&stg[0].e[ty][tx]) - (char*)stg);
  const int so_m = LAME ? (int)(((char*)&stg[0].m[LAME ? ty : 0][tx]) - (char*)stg) : 0;
  const int so_b = EPI != EPI_APPLY ? (int)(((char*)&stg[0].b[0][EPI != EPI_APPLY ? ty : 0][tx]) - (char*)stg) : 0;
  const int so_d = EPI == EPI_SMOOTH ? (int)(((char*)&stg[0].d[0][EPI == EPI_SMOOTH ? ty : 0][tx]) - (char*)stg) : 0;
  constexpr int SU_C = (TY + 1) * (TX + 1) * sizeof(P);
  constexpr int SB_C = (EPI != EPI_APPLY ? TY : 1) * TX * sizeof(P);
  constexpr int SD_C = (EPI == EPI_SMOOTH ? TY : 1) * TX * sizeof(P);

  auto issue = [&](int s) {
    const unsigned st_base = sbase + (unsigned)((s % NSTAGE) * sizeof(St));
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const bool pok = s < smax[l];
      const int poff = (z0[l] + 1 + s) * sz;
#pragma unroll
      for (int q = 0; q < NLOAD; ++q) {
        if (tid + q * NTH < NHALO) {
          const bool ok = pok && hok[q];
          const T* src = u + (ok ? 3 * poff + gu[q] : 0);
          const unsigned dst = st_base + su[q] + l * ES;
#pragma unroll
          for (int c = 0; c < 3; ++c) cp_el<ES>(dst + c * SU_C, src + c, ok);
        }
      }
      const bool ok = pok && col_in;
      const int qe = ok ? poff + colbase : 0;
      cp_el<ES>(st_base + so_e + l * ES, Ev + qe, ok);
      if (LAME) cp_el<ES>(st_base + so_m + l * ES, MUv + qe, ok);
      if (EPI != EPI_APPLY) {
#pragma unroll
        for (int c = 0; c < 3; ++c) cp_el<ES>(st_base + so_b + c * SB_C + l * ES, bvec + 3 * qe + c, ok);
      }
      if (EPI == EPI_SMOOTH) {
#pragma unroll
        for (int c = 0; c < 3; ++c) cp_el<ES>(st_base + so_d + c * SD_C + l * ES, minv + 3 * qe + c, ok);
      }
    }
  };

  P hiPrev[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int m = 0; m < 4; ++m) hiPrev[c][m] = O::zero();
  double dot = 0.0;
  const int nsteps = H + 2;

  // One z-step: face transform of plane s into Fc; voxel (s-1, s) from Fp, Fc;
  // output of plane s-1.
  auto step = [&](const int s, P (&Fc)[3][4], const P (&Fp)[3][4]) {
    cp_async_wait<1>();
    __syncthreads();                       // stage s visible; step s-1 fully done
    if (s + 2 < nsteps) issue(s + 2);      // overwrites the stage of step s-2
    cp_async_commit();
    uint8_t mk[L];
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const int zs = z0[l] + s - 1;        // logical plane finished at this step
      mk[l] = (s >= 2 && out_col && zs < oend[l]) ? mask[(zs + 1) * sz + colbase] : (uint8_t)0;
    }
    const St& S = stg[s % NSTAGE];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const P u00 = S.u[c][ty][tx], u10 = S.u[c][ty][tx + 1];
      const P u01 = S.u[c][ty + 1][tx], u11 = S.u[c][ty + 1][tx + 1];
      const P e0 = O::add(u10, u00), e1 = O::sub(u10, u00);
      const P e2 = O::add(u11, u01), e3 = O::sub(u11, u01);
      Fc[c][0] = O::add(e0, e2);
      Fc[c][1] = O::add(e1, e3);
      Fc[c][2] = O::sub(e2, e0);
      Fc[c][3] = O::sub(e3, e1);
    }
    if (s >= 1) {
      const St& Sp = stg[(s - 1) % NSTAGE];
      P A[3][8];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          A[c][m] = O::add(Fp[c][m], Fc[c][m]);
          A[c][m + 4] = O::sub(Fc[c][m], Fp[c][m]);
        }
      const P El = Sp.e[ty][tx];
      const P Em = LAME ? Sp.m[LAME ? ty : 0][tx] : El;
      P B[3][8];
      modal_physics<O, P, T>(A, B, El, Em, mc);
      // transposed z stage: lower face completes plane s-1, upper face pending
      P acc[3][4];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc[c][0] = O::sub(hiPrev[c][0], B[c][4]);   // B[c][0] = 0 (constant mode)
        const P hi0 = B[c][4];
#pragma unroll
        for (int m = 1; m < 4; ++m) {
          acc[c][m] = O::add(hiPrev[c][m], O::sub(B[c][m], B[c][m + 4]));
          hiPrev[c][m] = O::add(B[c][m], B[c][m + 4]);
        }
        hiPrev[c][0] = hi0;
      }
      // transposed face transform: corner contributions of plane s-1
      P c00[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const P t0 = O::sub(acc[c][0], acc[c][2]), t1 = O::sub(acc[c][1], acc[c][3]);
        const P t2 = O::add(acc[c][0], acc[c][2]), t3 = O::add(acc[c][1], acc[c][3]);
        c00[c] = O::sub(t0, t1);
        s_c[0][c][ty][tx] = O::add(t0, t1);   // -> node (X+1, Y)
        s_c[1][c][ty][tx] = O::sub(t2, t3);   // -> node (X, Y+1)
        s_c[2][c][ty][tx] = O::add(t2, t3);   // -> node (X+1, Y+1)
      }
      __syncthreads();
      if (s >= 2 && out_col) {
        P y[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
          y[c] = O::add(O::add(c00[c], s_c[0][c][ty][tx - 1]), O::add(s_c[1][c][ty - 1][tx], s_c[2][c][ty - 1][tx - 1]));
#pragma unroll
        for (int l = 0; l < L; ++l) {
          const int zs = z0[l] + s - 1;
          if (zs < oend[l]) {
            const int p3 = 3 * ((zs + 1) * sz + colbase);
            const uint8_t m8 = mk[l];
            const T k0 = (m8 & 1) ? O::lane(y[0], l) : (T)0;
            const T k1 = (m8 & 2) ? O::lane(y[1], l) : (T)0;
            const T k2 = (m8 & 4) ? O::lane(y[2], l) : (T)0;
            if (EPI == EPI_APPLY) {
              out[p3] = k0; out[p3 + 1] = k1; out[p3 + 2] = k2;
              if (a.dot_partials) {
                const T u0 = O::lane(Sp.u[0][ty][tx], l), u1 = O::lane(Sp.u[1][ty][tx], l);
                const T u2 = O::lane(Sp.u[2][ty][tx], l);
                dot += (double)u0 * (double)k0 + (double)u1 * (double)k1 + (double)u2 * (double)k2;
              }
            } else {
              const int by = EPI != EPI_APPLY ? ty : 0;
              const T b0 = O::lane(Sp.b[0][by][tx], l), b1 = O::lane(Sp.b[1][by][tx], l);
              const T b2 = O::lane(Sp.b[2][by][tx], l);
              if (EPI == EPI_SMOOTH) {
                const int dy = EPI == EPI_SMOOTH ? ty : 0;
                const T u0 = O::lane(Sp.u[0][ty][tx], l), u1 = O::lane(Sp.u[1][ty][tx], l);
                const T u2 = O::lane(Sp.u[2][ty][tx], l);
                const T d0 = O::lane(Sp.d[0][dy][tx], l), d1 = O::lane(Sp.d[1][dy][tx], l);
                const T d2 = O::lane(Sp.d[2][dy][tx], l);
                T o0 = u0 + ((m8 & 1) ? w * (d0 * (b0 - k0)) : (T)0);
                T o1 = u1 + ((m8 & 2) ? w * (d1 * (b1 - k1)) : (T)0);
                T o2 = u2 + ((m8 & 4) ? w * (d2 * (b2 - k2)) : (T)0);
                if (dprev) { o0 += c1 * dprev[p3]; o1 += c1 * dprev[p3 + 1]; o2 += c1 * dprev[p3 + 2]; }
                out[p3] = o0; out[p3 + 1] = o1; out[p3 + 2] = o2;
                if (dout) { dout[p3] = o0 - u0; dout[p3 + 1] = o1 - u1; dout[p3 + 2] = o2 - u2; }
                if (a.dot_partials) dot += (double)b0 * (double)o0 + (double)b1 * (double)o1 + (double)b2 * (double)o2;
              } else {
                out[p3] = b0 - k0; out[p3 + 1] = b1 - k1; out[p3 + 2] = b2 - k2;
              }
            }
          }
        }
      }
    } else {
      __syncthreads();
    }
  };

  issue(0);
  cp_async_commit();
  if (1 < nsteps) issue(1);
  cp_async_commit();
  P Fa[3][4], Fb[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int m = 0; m < 4; ++m) { Fa[c][m] = O::zero(); Fb[c][m] = O::zero(); }
#pragma unroll 1
  for (int s = 0; s < nsteps; ++s) {
    step(s, Fa, Fb);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int m = 0; m < 4; ++m) Fb[c][m] = Fa[c][m];
  }
  cp_async_wait<0>();
  // APPLY: u.y (p.Ap); SMOOTH: b.u' (the V-cycle's last sweep: r.z)
  if ((EPI == EPI_APPLY || EPI == EPI_SMOOTH) && a.dot_partials && ks)
    reduce_and_finalize(dot, a.dot_partials, ks, a.dot_slot, nullptr);
}

template <typename T, int TY, bool LAME, int EPI>
constexpr size_t modal_smem_bytes() {
  using P = typename Pack<T>::P;
  return NSTAGE * sizeof(Stage<P, TY, LAME, EPI>) + sizeof(P) * 3 * 3 * TY * TX;
}

}  // namespace

ModalConst modal_constants(double nu, bool lame) {
  ModalConst m;
  for (int k = 0; k < 3; ++k) {
    const double wk = std::pow(3.0, -k) / 16.0;
    double cl, cm;
    if (lame) { cl = wk; cm = wk; }
    else { cl = wk * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)); cm = wk / (2.0 * (1.0 + nu)); }
    m.cLd[k] = cl; m.cMd[k] = cm; m.cLf[k] = (float)cl; m.cMf[k] = (float)cm;
  }
  return m;
}

// Launch geometry: (ceil((lx+1)/31), ceil((ly+1)/(TY-1)), ceil((lz+1)/zchunk)).
template <typename T>
void launch_modal_op(const Grid& g, int epi, const OpArgs& a, const ModalConst& mc, int ty, int zchunk,
                     cudaStream_t st) {
  const bool lame = a.mu != nullptr;
  if (zchunk < 1) zchunk = g.lz + 1;
  const int gz = (g.lz + 1 + zchunk - 1) / zchunk;
  (void)ty;
  constexpr int TYV = 8;
  const dim3 grid((g.lx + 1 + TX - 2) / (TX - 1), (g.ly + 1 + TYV - 2) / (TYV - 1), gz);
  const dim3 block(TX, TYV);
#define VF_MODAL_ONE(LM, EP)                                                                  \
  do {                                                                                        \
    auto kern = k_modal_op<T, LM, EP, TYV>;                                                   \
    constexpr size_t smem = modal_smem_bytes<T, TYV, LM, EP>();                               \
    static std::atomic<int> per_dev[kMaxDevices];                                             \
    kernel_prepare(per_dev, kern, smem, TX * TYV);                                            \
    launch_k(kern, grid, block, smem, st, g, a, mc, zchunk);                                  \
  } while (0)
  if (lame) {
    if (epi == EPI_APPLY) VF_MODAL_ONE(true, EPI_APPLY);
    else if (epi == EPI_SMOOTH) VF_MODAL_ONE(true, EPI_SMOOTH);
    else VF_MODAL_ONE(true, EPI_RESID);
  } else {
    if (epi == EPI_APPLY) VF_MODAL_ONE(false, EPI_APPLY);
    else if (epi == EPI_SMOOTH) VF_MODAL_ONE(false, EPI_SMOOTH);
    else VF_MODAL_ONE(false, EPI_RESID);
  }
#undef VF_MODAL_ONE
}

template void launch_modal_op<float>(const Grid&, int, const OpArgs&, const ModalConst&, int, int, cudaStream_t);
template void launch_modal_op<double>(const Grid&, int, const OpArgs&, const ModalConst&, int, int, cudaStream_t);

}  // namespace vf
