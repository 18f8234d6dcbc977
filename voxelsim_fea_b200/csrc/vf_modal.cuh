// Shared arithmetic of the modal hex8 operator kernels (vf_modal.cu,
// vf_modal_tma.cu): packed FP32x2 / FP64 helpers and the per-voxel modal
// physics (modal coefficients -> modal forces).
#pragma once

#include "vf_common.cuh"

namespace vf {
namespace modal {

template <typename T> struct Pack;

template <> struct Pack<float> {
  using P = float2;
  static constexpr int L = 2;
  __device__ __forceinline__ static P add(P a, P b) { return __fadd2_rn(a, b); }
  __device__ __forceinline__ static P sub(P a, P b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
  __device__ __forceinline__ static P mul(P a, P b) { return __fmul2_rn(a, b); }
  __device__ __forceinline__ static P fma(P a, P b, P c) { return __ffma2_rn(a, b, c); }
  __device__ __forceinline__ static P zero() { return make_float2(0.f, 0.f); }
  __device__ __forceinline__ static float lane(P a, int l) { return l ? a.y : a.x; }
};

template <> struct Pack<double> {
  using P = double;
  static constexpr int L = 1;
  __device__ __forceinline__ static P add(P a, P b) { return a + b; }
  __device__ __forceinline__ static P sub(P a, P b) { return a - b; }
  __device__ __forceinline__ static P mul(P a, P b) { return a * b; }
  __device__ __forceinline__ static P fma(P a, P b, P c) { return ::fma(a, b, c); }
  __device__ __forceinline__ static P zero() { return 0.0; }
  __device__ __forceinline__ static double lane(P a, int) { return a; }
};

// ModalConst (vf_common.cuh): non-LAME: Elam = Emu = E and cL/cM carry nu;
// LAME: Elam = lambda_e, Emu = mu_e and cL = cM = 3^-k / 16.  The 1/16 folds
// the two unnormalised Hadamard transforms (1/64) and the Jacobian factors (x4).

template <typename T> __device__ __forceinline__ T cL(const ModalConst& m, int k);
template <> __device__ __forceinline__ float cL<float>(const ModalConst& m, int k) { return m.cLf[k]; }
template <> __device__ __forceinline__ double cL<double>(const ModalConst& m, int k) { return m.cLd[k]; }
template <typename T> __device__ __forceinline__ T cM(const ModalConst& m, int k);
template <> __device__ __forceinline__ float cM<float>(const ModalConst& m, int k) { return m.cMf[k]; }
template <> __device__ __forceinline__ double cM<double>(const ModalConst& m, int k) { return m.cMd[k]; }

template <typename P> __device__ __forceinline__ P bc(double v);
template <> __device__ __forceinline__ float2 bc<float2>(double v) { return make_float2((float)v, (float)v); }
template <> __device__ __forceinline__ double bc<double>(double v) { return v; }

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// The per-voxel modal physics: A (modal coefficients, 3 comps x 8 modes) ->
// B (modal forces).  Mode index m = p + 2q + 4r for xi^p eta^q zeta^r.
template <typename O, typename P, typename T>
__device__ __forceinline__ void modal_physics(const P (&A)[3][8], P (&B)[3][8], const P El, const P Em,
                                              const ModalConst& mc) {
  const P L0 = O::mul(El, bc<P>(cL<T>(mc, 0))), L1 = O::mul(El, bc<P>(cL<T>(mc, 1)));
  const P L2 = O::mul(El, bc<P>(cL<T>(mc, 2)));
  const P M0 = O::mul(Em, bc<P>(cM<T>(mc, 0))), M1 = O::mul(Em, bc<P>(cM<T>(mc, 1)));
  const P M2 = O::mul(Em, bc<P>(cM<T>(mc, 2)));
  const P M0x2 = O::add(M0, M0), M1x2 = O::add(M1, M1);
  const P K2 = O::fma(M2, bc<P>(4.0), L2);
  {
    const P tr = O::add(O::add(A[0][1], A[1][2]), A[2][4]);
    const P Ltr = O::mul(L0, tr);
    B[0][1] = O::fma(M0x2, A[0][1], Ltr);
    B[1][2] = O::fma(M0x2, A[1][2], Ltr);
    B[2][4] = O::fma(M0x2, A[2][4], Ltr);
    const P sxy = O::mul(M0, O::add(A[0][2], A[1][1]));
    const P sxz = O::mul(M0, O::add(A[0][4], A[2][1]));
    const P syz = O::mul(M0, O::add(A[1][4], A[2][2]));
    B[0][2] = sxy; B[1][1] = sxy;
    B[0][4] = sxz; B[2][1] = sxz;
    B[1][4] = syz; B[2][2] = syz;
  }
  {
    const P Lx = O::mul(L1, O::add(A[1][3], A[2][5]));
    P by3 = O::fma(M1x2, A[1][3], Lx);
    P bz5 = O::fma(M1x2, A[2][5], Lx);
    P bx3 = O::mul(M1, A[0][3]);
    P bx5 = O::mul(M1, A[0][5]);
    const P syz = O::mul(M1, O::add(A[1][5], A[2][3]));
    P by5 = syz;
    P bz3 = syz;
    const P Ly = O::mul(L1, O::add(A[0][3], A[2][6]));
    bx3 = O::add(bx3, O::fma(M1x2, A[0][3], Ly));
    P bz6 = O::fma(M1x2, A[2][6], Ly);
    by3 = O::fma(M1, A[1][3], by3);
    P by6 = O::mul(M1, A[1][6]);
    const P sxz = O::mul(M1, O::add(A[0][6], A[2][3]));
    P bx6 = sxz;
    bz3 = O::add(bz3, sxz);
    const P Lz = O::mul(L1, O::add(A[0][5], A[1][6]));
    bx5 = O::add(bx5, O::fma(M1x2, A[0][5], Lz));
    by6 = O::add(by6, O::fma(M1x2, A[1][6], Lz));
    bz5 = O::fma(M1, A[2][5], bz5);
    bz6 = O::fma(M1, A[2][6], bz6);
    const P sxy = O::mul(M1, O::add(A[0][6], A[1][5]));
    bx6 = O::add(bx6, sxy);
    by5 = O::add(by5, sxy);
    B[0][3] = bx3; B[0][5] = bx5; B[0][6] = bx6;
    B[1][3] = by3; B[1][5] = by5; B[1][6] = by6;
    B[2][3] = bz3; B[2][5] = bz5; B[2][6] = bz6;
  }
  B[0][7] = O::mul(K2, A[0][7]);
  B[1][7] = O::mul(K2, A[1][7]);
  B[2][7] = O::mul(K2, A[2][7]);
}

}  // namespace modal
}  // namespace vf
