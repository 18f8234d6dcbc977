// 3x3x3 convolutions of the learned preconditioner stage: BF16 operands,
// FP32 accumulation on the tensor cores, implicit GEMM.
//
// Activations are channels-last BF16 tensors [Z][Y][X][C] (C = 16, 32 or 64),
// zero outside the box (the halo loads fill zeros: "same" padding).  Weights
// are [27][COUT][CIN] BF16 (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)), so the
// input-channel axis -- the GEMM K axis -- is contiguous.
//
// Forward and backward-data (the forward of dY with the weights transposed
// and the taps mirrored) run on tcgen05 with TMEM accumulators
// (vf_nn_tc.cu); this file keeps the dispatch and the weight gradient.
//
// Backward-weight: dW[tap][co][ci] = sum_v dY[v][co] X[v + off(tap)][ci] is a
// GEMM with M = co, N = ci and K = voxels (mma.m16n8k16).  A CTA takes a group
// of taps and a strided set of voxel tiles; both operands come out of shared
// memory through ldmatrix.trans.  Per-CTA partial sums are reduced in a fixed
// order (deterministic).
#include <cuda_bf16.h>

#include <atomic>

#include "vf_common.cuh"
#include "vf_nn.cuh"

namespace vf {

namespace {

using bf16 = __nv_bfloat16;

constexpr int OTX = 16, OTY = 8, OTZ = 2;                 // output tile
constexpr int HTX = OTX + 2, HTY = OTY + 2, HTZ = OTZ + 2;
constexpr int NHALO = HTX * HTY * HTZ;                     // 720
constexpr int NTHREADS = 256;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4_t(unsigned a, unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3) : "r"(a));
}
__device__ __forceinline__ void ldsm_x2_t(unsigned a, unsigned& r0, unsigned& r1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(a));
}
__device__ __forceinline__ void mma16816(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Load the (16 x 8 x 2 + halo) input box of a tile into shared memory,
// zero outside [0,X) x [0,Y) x [0,Z).  16-byte chunks.
template <int C, int CP>
__device__ __forceinline__ void load_halo(bf16* s, const bf16* __restrict__ g, int X, int Y, int Z, int X0, int Y0,
                                          int Z0) {
  constexpr int CH = C / 8;
  for (int i = threadIdx.x; i < NHALO * CH; i += NTHREADS) {
    const int v = i / CH, c = i - v * CH;
    const int hx = v % HTX, hy = (v / HTX) % HTY, hz = v / (HTX * HTY);
    const int x = X0 - 1 + hx, y = Y0 - 1 + hy, z = Z0 - 1 + hz;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (x >= 0 && x < X && y >= 0 && y < Y && z >= 0 && z < Z)
      val = __ldg(reinterpret_cast<const uint4*>(g + (((long long)z * Y + y) * X + x) * C) + c);
    *reinterpret_cast<uint4*>(s + v * CP + c * 8) = val;
  }
}

__device__ __forceinline__ int halo_index(int hx, int hy, int hz) { return (hz * HTY + hy) * HTX + hx; }

// ---------------------------------------------------------------------------
template <int CIN, int COUT>
struct WgradCfg {
  static constexpr int frags(int taps) { return taps * (COUT / 16) * (CIN / 8); }
  static constexpr int TAPS = frags(27) <= 128 ? 27 : (frags(9) <= 128 ? 9 : (frags(3) <= 128 ? 3 : 1));
  static constexpr int F = frags(TAPS);
  static constexpr int NF = (F + 7) / 8;   // fragments per warp
  static constexpr int DP = COUT + 8;      // smem stride of a dY voxel
  static constexpr size_t smem() {
    return sizeof(bf16) * ((size_t)NHALO * (CIN + 8) + (size_t)OTX * OTY * OTZ * DP);
  }
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(NTHREADS) k_conv3_wgrad(const bf16* __restrict__ x, const bf16* __restrict__ dy,
                                                           float* __restrict__ partial, int X, int Y, int Z) {
  using Cfg = WgradCfg<CIN, COUT>;
  constexpr int CP = CIN + 8, DP = Cfg::DP, NF = Cfg::NF, F = Cfg::F, TAPS = Cfg::TAPS;
  constexpr int MT = COUT / 16, NTI = CIN / 8;
  extern __shared__ __align__(16) unsigned char smem[];
  bf16* sX = reinterpret_cast<bf16*>(smem);
  bf16* sD = sX + NHALO * CP;   // [256 tile voxels][DP], voxel = (tz*8 + ty)*16 + tx
  const int tx = (X + OTX - 1) / OTX, ty = (Y + OTY - 1) / OTY, tz = (Z + OTZ - 1) / OTZ;
  const int ntiles = tx * ty * tz;
  const int tap0 = blockIdx.y * TAPS;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float acc[NF][4];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[f][k] = 0.f;
  // A = dY^T (m = co, k = voxel), from [voxel][co]: ldmatrix.trans, row = voxel
  const int a_v = (lane & 7) + ((lane >> 4) & 1) * 8;
  const int a_c = ((lane >> 3) & 1) * 8;
  // B = X shifted (k = voxel, n = ci), from [voxel][ci]: ldmatrix.trans, row = voxel (lanes 0..15)
  const int b_v = (lane & 7) + ((lane >> 3) & 1) * 8;

#pragma unroll 1
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int X0 = (t % tx) * OTX, Y0 = ((t / tx) % ty) * OTY, Z0 = (t / (tx * ty)) * OTZ;
    __syncthreads();
    load_halo<CIN, CP>(sX, x, X, Y, Z, X0, Y0, Z0);
    {
      constexpr int CH = COUT / 8;
      for (int i = threadIdx.x; i < OTX * OTY * OTZ * CH; i += NTHREADS) {
        const int v = i / CH, c = i - v * CH;
        const int vx = v % OTX, vy = (v / OTX) % OTY, vz = v / (OTX * OTY);
        const int gx = X0 + vx, gy = Y0 + vy, gz = Z0 + vz;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (gx < X && gy < Y && gz < Z)
          val = __ldg(reinterpret_cast<const uint4*>(dy + (((long long)gz * Y + gy) * X + gx) * COUT) + c);
        *reinterpret_cast<uint4*>(sD + v * DP + c * 8) = val;
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const int f = warp + 8 * j;
      if (f >= F) break;
      const int tap = f / (MT * NTI), rem = f % (MT * NTI), mt = rem / NTI, nt = rem % NTI;
      const int tg = tap0 + tap;
      const int ddz = tg / 9, ddy = (tg / 3) % 3, ddx = tg % 3;   // halo offsets (d + 1)
#pragma unroll 1
      for (int row = 0; row < OTY * OTZ; ++row) {
        const int ry = row % OTY, rz = row / OTY;
        unsigned a0, a1, a2, a3, b0, b1;
        ldsm_x4_t(smem_u32(sD + (row * OTX + a_v) * DP + mt * 16 + a_c), a0, a1, a2, a3);
        ldsm_x2_t(smem_u32(sX + halo_index((b_v & 15) + ddx, ry + ddy, rz + ddz) * CP + nt * 8), b0, b1);
        mma16816(acc[j], a0, a1, a2, a3, b0, b1);
      }
    }
  }
  // partial[block][tap][co][ci] for the taps of this group
  const int g = lane >> 2, tig = lane & 3;
  float* dst = partial + (long long)blockIdx.x * 27 * COUT * CIN;
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    const int f = warp + 8 * j;
    if (f >= F) break;
    const int tap = f / (MT * NTI), rem = f % (MT * NTI), mt = rem / NTI, nt = rem % NTI;
    const int tg = tap0 + tap;
    const int co = mt * 16 + g, ci = nt * 8 + 2 * tig;
    float* d = dst + ((long long)tg * COUT + co) * CIN + ci;
    d[0] = acc[j][0];
    d[1] = acc[j][1];
    d[8 * CIN] = acc[j][2];
    d[8 * CIN + 1] = acc[j][3];
  }
}

__global__ void k_reduce_partials(const float* __restrict__ partial, int nparts, long long n, float* __restrict__ out,
                                  int accumulate) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nparts; ++b) s += partial[(long long)b * n + i];
    out[i] = accumulate ? out[i] + s : s;
  }
}

template <int CIN, int COUT>
int conv_wgrad_t(const void* x, const void* dy, float* dw, float* work, size_t work_bytes, int X, int Y, int Z,
                 int accumulate, cudaStream_t st) {
  using Cfg = WgradCfg<CIN, COUT>;
  const size_t per = sizeof(float) * 27 * COUT * CIN;
  const long long tiles = (long long)((X + OTX - 1) / OTX) * ((Y + OTY - 1) / OTY) * ((Z + OTZ - 1) / OTZ);
  long long nb = std::min<long long>(tiles, 148);
  nb = std::min<long long>(nb, (long long)(work_bytes / per));
  if (nb < 1) return -1;
  constexpr size_t smem = Cfg::smem();
  static std::atomic<int> per_dev[kMaxDevices];
  kernel_prepare(per_dev, k_conv3_wgrad<CIN, COUT>, smem, NTHREADS);
  launch_k(k_conv3_wgrad<CIN, COUT>, dim3((unsigned)nb, 27 / Cfg::TAPS), dim3(NTHREADS), smem, st,
           (const bf16*)x, (const bf16*)dy, work, X, Y, Z);
  const long long n = 27LL * COUT * CIN;
  launch_k(k_reduce_partials, dim3((unsigned)((n + 255) / 256)), dim3(256), 0, st, (const float*)work, (int)nb, n,
           dw, accumulate);
  return 0;
}

}  // namespace

size_t nn_wgrad_work_bytes(int cin, int cout, int X, int Y, int Z) {
  const long long tiles = (long long)((X + OTX - 1) / OTX) * ((Y + OTY - 1) / OTY) * ((Z + OTZ - 1) / OTZ);
  return sizeof(float) * 27 * (size_t)cin * cout * (size_t)std::max<long long>(1, std::min<long long>(tiles, 148));
}

#define VF_NN_PAIRS(F) F(16, 16) F(16, 32) F(32, 16) F(32, 32) F(32, 64) F(64, 32) F(64, 64)

template <int CIN, int COUT> int conv_forward_tc(const NnConvArgs& a, cudaStream_t st);   // vf_nn_tc.cu

int nn_conv_forward(int cin, int cout, const NnConvArgs& a, cudaStream_t st) {
#define VF_NN_FWD(I, O) \
  if (cin == I && cout == O) return conv_forward_tc<I, O>(a, st);
  VF_NN_PAIRS(VF_NN_FWD)
#undef VF_NN_FWD
  return -1;
}

int nn_conv_wgrad(int cin, int cout, const void* x, const void* dy, float* dw, float* work, size_t work_bytes, int X,
                  int Y, int Z, int accumulate, cudaStream_t st) {
#define VF_NN_WG(I, O) \
  if (cin == I && cout == O) return conv_wgrad_t<I, O>(x, dy, dw, work, work_bytes, X, Y, Z, accumulate, st);
  VF_NN_PAIRS(VF_NN_WG)
#undef VF_NN_WG
  return -1;
}

}  // namespace vf

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
#include "../../include/voxfea.h"

extern "C" {

int vf_nn_conv3d_forward(const void* in, const void* w, const float* bias, const void* skip, int32_t relu, void* out,
                         float* out_f32, int32_t X, int32_t Y, int32_t Z, int32_t cin, int32_t cout, void* stream) {
  if (!in || !w || (!out && !out_f32) || X < 1 || Y < 1 || Z < 1) return VF_ERR_ARG;
  vf::NnConvArgs a{in, w, bias, skip, nullptr, out, out_f32, X, Y, Z, relu ? 1 : 0};
  if (vf::nn_conv_forward(cin, cout, a, (cudaStream_t)stream)) return VF_ERR_ARG;
  return cudaPeekAtLastError() == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

int vf_nn_conv3d_backward_data(const void* dy, const void* w_t, const void* gate, void* dx, int32_t X, int32_t Y,
                               int32_t Z, int32_t cin, int32_t cout, void* stream) {
  if (!dy || !w_t || !dx || X < 1 || Y < 1 || Z < 1) return VF_ERR_ARG;
  vf::NnConvArgs a{dy, w_t, nullptr, nullptr, gate, dx, nullptr, X, Y, Z, 0};
  if (vf::nn_conv_forward(cout, cin, a, (cudaStream_t)stream)) return VF_ERR_ARG;
  return cudaPeekAtLastError() == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

int vf_nn_conv3d_backward_weight(const void* x, const void* dy, float* dw, int32_t accumulate, float* work,
                                 size_t work_bytes, int32_t X, int32_t Y, int32_t Z, int32_t cin, int32_t cout,
                                 void* stream) {
  if (!x || !dy || !dw || !work || X < 1 || Y < 1 || Z < 1) return VF_ERR_ARG;
  if (vf::nn_conv_wgrad(cin, cout, x, dy, dw, work, work_bytes, X, Y, Z, accumulate, (cudaStream_t)stream))
    return VF_ERR_ARG;
  return cudaPeekAtLastError() == cudaSuccess ? VF_OK : VF_ERR_CUDA;
}

size_t vf_nn_wgrad_workspace(int32_t cin, int32_t cout, int32_t X, int32_t Y, int32_t Z) {
  return vf::nn_wgrad_work_bytes(cin, cout, X, Y, Z);
}

}  // extern "C"
