// 3x3x3 convolutions of the learned preconditioner stage on the 5th-generation
// tensor cores (tcgen05.mma, BF16 operands, FP32 accumulator in TMEM).
//
// Implicit GEMM per CTA: M = 128 output voxels (a tile of 8 x 16 voxels in
// x, y at one z), N = COUT output channels, K = CIN input channels x 27 taps.
// The input box of the tile -- 10 x 18 voxels on the three planes z-1..z+1 --
// is staged once in shared memory in the canonical no-swizzle K-major layout
// of the UMMA operands:
//     sIn[plane][k-chunk of 8 channels][y (18)][x (10)][8 channels]  (16 B per voxel)
// so the A operand of tap (dx, dy, dz) is the same array seen from another
// start address: 8 x-consecutive voxels form one core matrix (rows 16 B
// apart), the 16 y-rows of the tile follow at the row pitch (SBO = 160 B) and
// the second 8-channel chunk of a K = 16 step sits one chunk plane further
// (LBO = 2880 B).  No re-staging per tap, no swizzle to break by shifting.
// The weights of one dz plane (9 taps) are staged per phase as
//     sW[tap][k-chunk][COUT][8 channels]   (SBO = 128 B, LBO = COUT x 16 B).
// One thread issues the 27 x CIN/16 MMAs; tcgen05.commit arrives on an
// mbarrier per phase.  The epilogue: each warp reads its 32 TMEM lanes
// (tcgen05.ld 32x32b), one voxel per thread with its COUT channels in
// registers, adds bias / skip, applies ReLU or the ReLU gate of a saved
// activation, and stores BF16 (or FP32).
// Every wait is bounded (vf_wait.cuh): on expiry the kernel raises the error
// flag, waits (bounded) for its MMAs to finish, frees its TMEM and returns.
#include <cuda_bf16.h>

#include <atomic>
#include <cstdlib>
#include <cstring>

#include "vf_common.cuh"
#include "vf_nn.cuh"
#include "vf_wait.cuh"

namespace vf {

namespace {

using bf16 = __nv_bfloat16;

constexpr int TCX = 8, TCY = 16;            // output tile (x, y) at one z: 128 voxels = M
constexpr int HCX = TCX + 2, HCY = TCY + 2;  // halo box per plane
constexpr int kTcThreads = 128;              // 4 warps = the 128 TMEM lanes of M

__device__ __forceinline__ uint32_t s32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, canonical no-swizzle layout (version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, A and B K-major, M = 128, N.
template <int N>
__host__ __device__ constexpr uint32_t idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(s32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int CIN, int COUT>
struct TcLayout {
  static constexpr int KC = CIN / 8;                                  // 8-channel chunks
  static constexpr uint32_t ROW = HCX * 16;                           // y pitch of sIn (SBO of A)
  static constexpr uint32_t CHUNK_A = HCY * ROW;                      // k-chunk pitch of sIn (LBO of A)
  static constexpr uint32_t PLANE = KC * CHUNK_A;
  static constexpr uint32_t IN_BYTES = 3 * PLANE;
  static constexpr uint32_t CHUNK_B = COUT * 16;                      // LBO of B
  static constexpr uint32_t TAP_B = KC * CHUNK_B;
  static constexpr uint32_t W_BYTES = 9 * TAP_B;
  static constexpr int TCOLS = COUT < 32 ? 32 : COUT;                 // TMEM columns (power of two >= 32)
  static constexpr size_t smem() { return 1024 + (size_t)IN_BYTES + W_BYTES + 64; }
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kTcThreads) k_conv3_tc(NnConvArgs a) {
  using L = TcLayout<CIN, COUT>;
  static_assert(COUT % 16 == 0 && COUT >= 16 && COUT <= 256, "N of an M = 128 BF16 MMA");
  static_assert(CIN % 16 == 0, "K steps of 16 channels");
  if (a.skip_flag && *a.skip_flag) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sIn = base;
  unsigned char* sW = base + L::IN_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sW + L::W_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sW + L::W_BYTES + 16);

  const int X = a.X, Y = a.Y, Z = a.Z;
  const int ntx = (X + TCX - 1) / TCX, nty = (Y + TCY - 1) / TCY;
  const int X0 = (blockIdx.x % ntx) * TCX, Y0 = ((blockIdx.x / ntx) % nty) * TCY, z = blockIdx.x / (ntx * nty);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bf16* __restrict__ in = reinterpret_cast<const bf16*>(a.in);
  const bf16* __restrict__ w = reinterpret_cast<const bf16*>(a.w);

  // TMEM accumulator (warp 0 allocates; the permit is released for the next CTA)
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(s32(tslot)),
                 "r"((uint32_t)L::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(s32(bar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // input box of the three planes, zero outside the volume; consecutive
  // threads take consecutive voxels of one channel chunk (conflict-free stores)
  for (int i = threadIdx.x; i < 3 * L::KC * HCY * HCX; i += kTcThreads) {
    const int v = i % (HCY * HCX), rest = i / (HCY * HCX), kc = rest % L::KC, pl = rest / L::KC;
    const int hx = v % HCX, hy = v / HCX;
    const int x = X0 - 1 + hx, y = Y0 - 1 + hy, zz = z - 1 + pl;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (x >= 0 && x < X && y >= 0 && y < Y && zz >= 0 && zz < Z)
      val = __ldg(reinterpret_cast<const uint4*>(in + (((long long)zz * Y + y) * X + x) * CIN) + kc);
    *reinterpret_cast<uint4*>(sIn + pl * L::PLANE + kc * L::CHUNK_A + hy * L::ROW + hx * 16) = val;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = idesc_bf16<COUT>();
  bool failed = false;

#pragma unroll 1
  for (int dz = 0; dz < 3; ++dz) {
    // weights of the 9 taps of this plane: sW[t9][kc][n][8]
    for (int i = threadIdx.x; i < 9 * L::KC * COUT; i += kTcThreads) {
      const int n = i % COUT, rest = i / COUT, kc = rest % L::KC, t9 = rest / L::KC;
      const int tap = dz * 9 + t9;
      *reinterpret_cast<uint4*>(sW + t9 * L::TAP_B + kc * L::CHUNK_B + n * 16) =
          __ldg(reinterpret_cast<const uint4*>(w + ((long long)tap * COUT + n) * CIN) + kc);
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // generic stores -> MMA operand reads
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (threadIdx.x == 0) {
      const uint32_t a0 = s32(sIn) + dz * L::PLANE, b0 = s32(sW);
#pragma unroll 1
      for (int t9 = 0; t9 < 9; ++t9) {
        const int dy = t9 / 3, dx = t9 % 3;
#pragma unroll
        for (int kk = 0; kk < CIN / 16; ++kk) {
          const uint64_t ad = umma_desc(a0 + dy * L::ROW + dx * 16 + 2 * kk * L::CHUNK_A, L::CHUNK_A, L::ROW);
          const uint64_t bd = umma_desc(b0 + t9 * L::TAP_B + 2 * kk * L::CHUNK_B, L::CHUNK_B, 128);
          mma_bf16(tmem, ad, bd, idesc, (dz | t9 | kk) != 0 ? 1u : 0u);
        }
      }
      mma_commit(bar);
    }
    // the MMAs of this plane done (before sW is overwritten / the epilogue reads TMEM)
    const bool ok = mbar_wait_bounded(bar, (unsigned)(dz & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      if (threadIdx.x == 0 && a.err) atomicExch(a.err, 1);
      mbar_wait_bounded(bar, (unsigned)(dz & 1));   // let the issued MMAs land before TMEM is freed
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  }

  if (!failed) {
    // epilogue: warp w reads TMEM lanes 32w..32w+31 = voxels m = 32w + lane
    const int m = warp * 32 + lane;
    const int x = X0 + m % TCX, y = Y0 + m / TCX;
    const bool valid = x < X && y < Y;
    const long long vo = (((long long)z * Y + y) * X + x) * COUT;
    const bf16* __restrict__ skip = reinterpret_cast<const bf16*>(a.skip);
    const bf16* __restrict__ gate = reinterpret_cast<const bf16*>(a.gate);
    bf16* __restrict__ out = reinterpret_cast<bf16*>(a.out);
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (!valid) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        float t = v[j];
        if (a.bias) t += a.bias[c0 + j];
        if (skip) t += __bfloat162float(skip[vo + c0 + j]);
        if (a.relu) t = fmaxf(t, 0.f);
        if (gate) t = __bfloat162float(gate[vo + c0 + j]) > 0.f ? t : 0.f;
        v[j] = t;
      }
      if (a.out_f32) {
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(a.out_f32 + vo + c0 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
      } else {
        uint4 pk[2];
        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
        for (int j = 0; j < 8; ++j) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        *reinterpret_cast<uint4*>(out + vo + c0) = pk[0];
        *reinterpret_cast<uint4*>(out + vo + c0 + 8) = pk[1];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)L::TCOLS)
                 : "memory");
}

// The same GEMM marching a column of ZC output planes: all 27 weight taps stay
// resident, the input planes live in a 3-slot ring (plane p in slot p % 3),
// and each step stages one new plane before its 27 x CIN/16 MMAs.  For the
// channel pairs whose 27 taps fit in shared memory next to the ring.
template <int CIN, int COUT>
struct TczLayout {
  static constexpr int KC = CIN / 8;
  static constexpr uint32_t ROW = HCX * 16;
  static constexpr uint32_t CHUNK_A = HCY * ROW;
  static constexpr uint32_t PLANE = KC * CHUNK_A;
  static constexpr uint32_t IN_BYTES = 3 * PLANE;
  static constexpr uint32_t CHUNK_B = COUT * 16;
  static constexpr uint32_t TAP_B = KC * CHUNK_B;
  static constexpr uint32_t W_BYTES = 27 * TAP_B;
  static constexpr int TCOLS = COUT < 32 ? 32 : COUT;
  static constexpr size_t smem() { return 1024 + (size_t)IN_BYTES + W_BYTES + 64; }
  static constexpr bool fits() { return smem() <= 200 * 1024; }
  static_assert(TCOLS >= 32 && TCOLS <= 512, "TMEM columns");
};
constexpr int kZC = 8;   // output planes per CTA

template <int CIN, int COUT>
__device__ __forceinline__ void stage_plane(unsigned char* sIn, const bf16* __restrict__ in, int X, int Y, int Z,
                                            int X0, int Y0, int zz) {
  using L = TczLayout<CIN, COUT>;
  unsigned char* dst = sIn + ((zz + 3) % 3) * L::PLANE;
  for (int i = threadIdx.x; i < L::KC * HCY * HCX; i += kTcThreads) {
    const int v = i % (HCY * HCX), kc = i / (HCY * HCX);
    const int hx = v % HCX, hy = v / HCX;
    const int x = X0 - 1 + hx, y = Y0 - 1 + hy;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (x >= 0 && x < X && y >= 0 && y < Y && zz >= 0 && zz < Z)
      val = __ldg(reinterpret_cast<const uint4*>(in + (((long long)zz * Y + y) * X + x) * CIN) + kc);
    *reinterpret_cast<uint4*>(dst + kc * L::CHUNK_A + hy * L::ROW + hx * 16) = val;
  }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kTcThreads) k_conv3_tcz(NnConvArgs a) {
  using L = TczLayout<CIN, COUT>;
  static_assert(COUT % 16 == 0 && COUT >= 16 && COUT <= 256, "N of an M = 128 BF16 MMA");
  static_assert(CIN % 16 == 0, "K steps of 16 channels");
  if (a.skip_flag && *a.skip_flag) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sIn = base;
  unsigned char* sW = base + L::IN_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sW + L::W_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sW + L::W_BYTES + 16);

  const int X = a.X, Y = a.Y, Z = a.Z;
  const int ntx = (X + TCX - 1) / TCX, nty = (Y + TCY - 1) / TCY;
  const int X0 = (blockIdx.x % ntx) * TCX, Y0 = ((blockIdx.x / ntx) % nty) * TCY;
  const int zb = (blockIdx.x / (ntx * nty)) * kZC, ze = min(zb + kZC, Z);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bf16* __restrict__ in = reinterpret_cast<const bf16*>(a.in);
  const bf16* __restrict__ w = reinterpret_cast<const bf16*>(a.w);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(s32(tslot)),
                 "r"((uint32_t)L::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(s32(bar)), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // all 27 taps: sW[tap][kc][n][8]
  for (int i = threadIdx.x; i < 27 * L::KC * COUT; i += kTcThreads) {
    const int n = i % COUT, rest = i / COUT, kc = rest % L::KC, tap = rest / L::KC;
    *reinterpret_cast<uint4*>(sW + tap * L::TAP_B + kc * L::CHUNK_B + n * 16) =
        __ldg(reinterpret_cast<const uint4*>(w + ((long long)tap * COUT + n) * CIN) + kc);
  }
  stage_plane<CIN, COUT>(sIn, in, X, Y, Z, X0, Y0, zb - 1);
  stage_plane<CIN, COUT>(sIn, in, X, Y, Z, X0, Y0, zb);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = idesc_bf16<COUT>();
  const bf16* __restrict__ skip = reinterpret_cast<const bf16*>(a.skip);
  const bf16* __restrict__ gate = reinterpret_cast<const bf16*>(a.gate);
  bf16* __restrict__ out = reinterpret_cast<bf16*>(a.out);
  const int m = warp * 32 + lane;
  const int x = X0 + m % TCX, y = Y0 + m / TCX;
  const bool valid = x < X && y < Y;
  bool failed = false;

#pragma unroll 1
  for (int z = zb; z < ze; ++z) {
    // plane z+1 into the slot of plane z-2 (read by the previous step's MMAs,
    // which completed before that step's epilogue)
    stage_plane<CIN, COUT>(sIn, in, X, Y, Z, X0, Y0, z + 1);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (threadIdx.x == 0) {
      const uint32_t b0 = s32(sW);
#pragma unroll 1
      for (int tap = 0; tap < 27; ++tap) {
        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
        const uint32_t a0 = s32(sIn) + ((z - 1 + dz + 3) % 3) * L::PLANE;
#pragma unroll
        for (int kk = 0; kk < CIN / 16; ++kk) {
          const uint64_t ad = umma_desc(a0 + dy * L::ROW + dx * 16 + 2 * kk * L::CHUNK_A, L::CHUNK_A, L::ROW);
          const uint64_t bd = umma_desc(b0 + tap * L::TAP_B + 2 * kk * L::CHUNK_B, L::CHUNK_B, 128);
          mma_bf16(tmem, ad, bd, idesc, (tap | kk) != 0 ? 1u : 0u);
        }
      }
      mma_commit(bar);
    }
    const unsigned par = (unsigned)((z - zb) & 1);
    const bool ok = mbar_wait_bounded(bar, par);
    if (__syncthreads_or(!ok)) {
      failed = true;
      if (threadIdx.x == 0 && a.err) atomicExch(a.err, 1);
      mbar_wait_bounded(bar, par);   // let the issued MMAs land before TMEM is freed
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const long long vo = (((long long)z * Y + y) * X + x) * COUT;
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (!valid) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        float t = v[j];
        if (a.bias) t += a.bias[c0 + j];
        if (skip) t += __bfloat162float(skip[vo + c0 + j]);
        if (a.relu) t = fmaxf(t, 0.f);
        if (gate) t = __bfloat162float(gate[vo + c0 + j]) > 0.f ? t : 0.f;
        v[j] = t;
      }
      if (a.out_f32) {
#pragma unroll
        for (int j = 0; j < 16; j += 4)
          *reinterpret_cast<float4*>(a.out_f32 + vo + c0 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
      } else {
        uint4 pk[2];
        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
        for (int j = 0; j < 8; ++j) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        *reinterpret_cast<uint4*>(out + vo + c0) = pk[0];
        *reinterpret_cast<uint4*>(out + vo + c0 + 8) = pk[1];
      }
    }
    // every lane's TMEM reads of this step are done before the next MMAs overwrite D
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  }
  (void)failed;
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((uint32_t)L::TCOLS)
                 : "memory");
}

}  // namespace

// The z-marching form where its columns still give every SM a few CTAs (its
// steps are serial inside a CTA: on the U-Net's coarse boxes, 135 columns
// took 52 us where the one-plane form's 918 CTAs took 20 us); else one plane
// per CTA.
// VOXFEA_CONV_FORM=plane|column overrides the choice (the tests run both).
constexpr long long kTczMinColumns = 3LL * 148;

int conv_form_override() {
  const char* e = std::getenv("VOXFEA_CONV_FORM");
  if (!e) return 0;
  if (!std::strcmp(e, "plane")) return 1;
  if (!std::strcmp(e, "column")) return 2;
  return 0;
}

template <int CIN, int COUT>
int conv_forward_tc(const NnConvArgs& a, cudaStream_t st) {
  if constexpr (TczLayout<CIN, COUT>::fits()) {
    using LZ = TczLayout<CIN, COUT>;
    const long long cols = (long long)((a.X + TCX - 1) / TCX) * ((a.Y + TCY - 1) / TCY) * ((a.Z + kZC - 1) / kZC);
    const int ov = conv_form_override();
    if (ov == 2 || (ov == 0 && cols >= kTczMinColumns)) {
      static std::atomic<int> per_dev_z[kMaxDevices];
      kernel_prepare(per_dev_z, k_conv3_tcz<CIN, COUT>, LZ::smem(), kTcThreads);
      launch_k(k_conv3_tcz<CIN, COUT>, dim3((unsigned)cols), dim3(kTcThreads), LZ::smem(), st, a);
      return 0;
    }
  }
  using L = TcLayout<CIN, COUT>;
  static std::atomic<int> per_dev[kMaxDevices];
  kernel_prepare(per_dev, k_conv3_tc<CIN, COUT>, L::smem(), kTcThreads);
  const long long tiles = (long long)((a.X + TCX - 1) / TCX) * ((a.Y + TCY - 1) / TCY) * a.Z;
  if (tiles <= 0) return 0;
  launch_k(k_conv3_tc<CIN, COUT>, dim3((unsigned)tiles), dim3(kTcThreads), L::smem(), st, a);
  return 0;
}

#define VF_TC_INST(I, O) template int conv_forward_tc<I, O>(const NnConvArgs&, cudaStream_t);
VF_TC_INST(16, 16)
VF_TC_INST(16, 32)
VF_TC_INST(32, 16)
VF_TC_INST(32, 32)
VF_TC_INST(32, 64)
VF_TC_INST(64, 32)
VF_TC_INST(64, 64)
#undef VF_TC_INST

}  // namespace vf
