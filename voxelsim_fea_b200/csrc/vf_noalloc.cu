// vf_apply_noalloc: the fine-level hex8 operator y = mask(K u) with the fused
// dot product u.y, for callers that cannot allocate device memory.
//
// Who needs it: an application that owns every byte of device memory through
// its own allocator or a fixed arena (a solver embedded in a larger program
// with a hard memory budget), and code that must not trigger the implicit
// device synchronisation cudaMalloc/cudaFree can cause (real-time loops,
// work issued between other streams' kernels).  Such a caller passes its own
// device buffers; this entry point creates no solver handle and calls no
// allocator.  The only scratch -- one FP64 partial sum per thread block and a
// completion counter for the dot product -- lives in the fixed array below,
// which every GPU that loads the library keeps until the process exits.
//
// Limits and sharing:
//   * at most kMaxBlocks blocks of 256 threads, i.e. (nx+1)(ny+1)(nz+1) <=
//     kMaxNodes grid nodes; larger grids are rejected with VF_ERR_ARG;
//   * every call on a device shares the one array and it keeps the last call's
//     contents; the completion counter is cleared at the start of each call.
//     Calls whose kernels overlap on the GPU (different streams, no ordering)
//     race on the array and give wrong results: order them on one stream;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress with that device current) and keeps it for the
//     process; make that first call before any stream capture.  A
//     cudaDeviceReset tears the module down with the context, so the kept
//     address is stale afterwards: make no call on that device after a reset;
//   * u, y and u_dot_y must not overlap: threads read u at neighbouring nodes
//     while others write y, so an in-place call is rejected.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/voxfea.h"
#include "vf_common.cuh"
#include "vf_hex8.h"

namespace vf {
extern thread_local std::string g_last_error;
}

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 32768;
constexpr long long kMaxNodes = (long long)kMaxBlocks * kThreads;   // 8,388,608 nodes
constexpr int kMaxDevices = 64;
// [0, kMaxBlocks) doubles: per-block partials; then one unsigned counter.
constexpr size_t kScratchBytes = sizeof(double) * kMaxBlocks + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct KeParam { double k[576]; };

unsigned char* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of g_noalloc_scratch on the current device (set up once per device).
int scratch_for_device(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return VF_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      vf::g_last_error = std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e);
      return VF_ERR_CUDA;
    }
    g_scratch_addr[dev] = (unsigned char*)p;
  }
  *out = g_scratch_addr[dev];
  return VF_OK;
}

__global__ void __launch_bounds__(kThreads) k_apply_noalloc(int nx, int ny, int nz, const double* __restrict__ E,
                                                            const uint8_t* __restrict__ mask,
                                                            const double* __restrict__ u, double* __restrict__ y,
                                                            double* __restrict__ dot_out,
                                                            double* __restrict__ partials,
                                                            unsigned int* __restrict__ counter, const KeParam K) {
  const int nx1 = nx + 1, ny1 = ny + 1;
  const long long nn = (long long)nx1 * ny1 * (nz + 1);
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double dot = 0.0;
  if (r < nn) {
    const int x = (int)(r % nx1);
    const long long t = r / nx1;
    const int yy = (int)(t % ny1), z = (int)(t / ny1);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int ez = z - 1; ez <= z; ++ez) {
      if (ez < 0 || ez >= nz) continue;
      for (int ey = yy - 1; ey <= yy; ++ey) {
        if (ey < 0 || ey >= ny) continue;
        for (int ex = x - 1; ex <= x; ++ex) {
          if (ex < 0 || ex >= nx) continue;
          const double Ee = E[((long long)ex * ny + ey) * nz + ez];
          const int ka = vf::corner_k(x - ex, yy - ey, z - ez);
          double t0 = 0.0, t1 = 0.0, t2 = 0.0;
#pragma unroll
          for (int kb = 0; kb < 8; ++kb) {
            const int bx = (kb == 1 || kb == 2 || kb == 5 || kb == 6);
            const int by = (kb == 2 || kb == 3 || kb == 6 || kb == 7);
            const int bz = (kb >= 4);
            const long long m = 3 * ((ex + bx) + (long long)nx1 * ((ey + by) + (long long)ny1 * (ez + bz)));
            const double u0 = u[m], u1 = u[m + 1], u2 = u[m + 2];
            const int r0 = (3 * ka) * 24 + 3 * kb;
            t0 += K.k[r0] * u0 + K.k[r0 + 1] * u1 + K.k[r0 + 2] * u2;
            t1 += K.k[r0 + 24] * u0 + K.k[r0 + 25] * u1 + K.k[r0 + 26] * u2;
            t2 += K.k[r0 + 48] * u0 + K.k[r0 + 49] * u1 + K.k[r0 + 50] * u2;
          }
          a0 += Ee * t0; a1 += Ee * t1; a2 += Ee * t2;
        }
      }
    }
    const uint8_t mk = mask[r];
    a0 = (mk & 1) ? a0 : 0.0;
    a1 = (mk & 2) ? a1 : 0.0;
    a2 = (mk & 4) ? a2 : 0.0;
    y[3 * r] = a0; y[3 * r + 1] = a1; y[3 * r + 2] = a2;
    dot = u[3 * r] * a0 + u[3 * r + 1] * a1 + u[3 * r + 2] * a2;
  }
  // block sum in a fixed order, then the last block sums the partials in order
  __shared__ double s_w[kThreads / 32];
  __shared__ bool s_last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = dot;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) b += s_w[w];
    partials[blockIdx.x] = b;
    __threadfence();
    s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double s = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads) s += ((volatile double*)partials)[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) tot += s_w[w];
    *dot_out = tot;
    *counter = 0u;
  }
}

}  // namespace

extern "C" int vf_apply_noalloc(int32_t nx, int32_t ny, int32_t nz, double nu, const double* E,
                                const uint8_t* free_mask, const double* u, double* y, double* u_dot_y,
                                void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !E || !free_mask || !u || !y || !u_dot_y) {
    vf::g_last_error = "vf_apply_noalloc: invalid argument";
    return VF_ERR_ARG;
  }
  if (!(nu > -1.0 && nu < 0.5)) {
    vf::g_last_error = "vf_apply_noalloc: Poisson ratio must lie in (-1, 0.5)";
    return VF_ERR_ARG;
  }
  const long long nn = (long long)(nx + 1) * (ny + 1) * (nz + 1);
  if (nn > kMaxNodes) {
    vf::g_last_error = "vf_apply_noalloc: grid has " + std::to_string(nn) + " nodes; the fixed scratch array "
                       "supports at most " + std::to_string(kMaxNodes) + " ((nx+1)(ny+1)(nz+1) <= 8388608)";
    return VF_ERR_ARG;
  }
  {
    // [u, u + 3nn), [y, y + 3nn) and the one double at u_dot_y must be disjoint
    const uintptr_t bu = (uintptr_t)u, by = (uintptr_t)y, bd = (uintptr_t)u_dot_y;
    const uintptr_t len = (uintptr_t)(3 * nn) * sizeof(double);
    auto overlap = [](uintptr_t a0, uintptr_t a1, uintptr_t b0, uintptr_t b1) { return a0 < b1 && b0 < a1; };
    if (overlap(bu, bu + len, by, by + len) || overlap(bd, bd + sizeof(double), bu, bu + len) ||
        overlap(bd, bd + sizeof(double), by, by + len)) {
      vf::g_last_error = "vf_apply_noalloc: u, y and u_dot_y must not overlap";
      return VF_ERR_ARG;
    }
  }
  unsigned char* base = nullptr;
  int rc = scratch_for_device(&base);
  if (rc) return rc;
  double* partials = (double*)base;
  unsigned int* counter = (unsigned int*)(base + sizeof(double) * kMaxBlocks);
  cudaStream_t st = (cudaStream_t)stream;
  KeParam K;
  double tab[1728], b0[144];
  vf::hex8_tables(nu, tab, b0);
  for (int i = 0; i < 576; ++i) K.k[i] = tab[i];
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) {
    vf::g_last_error = std::string("vf_apply_noalloc: ") + cudaGetErrorString(e);
    return VF_ERR_CUDA;
  }
  const int blocks = (int)((nn + kThreads - 1) / kThreads);
  vf::launch_k(k_apply_noalloc, blocks, kThreads, 0, st, nx, ny, nz, E, free_mask, u, y, u_dot_y, partials,
               counter, K);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    vf::g_last_error = std::string("vf_apply_noalloc launch: ") + cudaGetErrorString(e);
    return VF_ERR_CUDA;
  }
  return VF_OK;
}
