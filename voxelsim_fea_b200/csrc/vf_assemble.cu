// Grid assembly of a solve job on the device (core/solve_worker.py:242-287):
// role masks -> active voxels, per-node fixed-DOF bits and the nodal force
// vector, and the island pre-step on those bits.
//
// Roles, in the job's order (the reference's semantics):
//   build    (per voxel)  the active set is the LAST build mask;
//   exclude  (per voxel)  removed from the active set (OR over the roles);
//   bearing  (per node)   the DOFs of the axes flagged in meta[3i..3i+2] are
//                         fixed (OR over the roles);
//   load     (per node)   the force meta[3i..3i+2] (N) is spread evenly over
//                         the role's nodes: f[3n+c] += meta[c] / count, role
//                         by role in job order, so the sums are the
//                         reference's bit for bit.
// Counts are integer reductions (atomics on integers are order-independent).
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/voxfea.h"
#include "vf_common.cuh"

namespace vf {
extern thread_local std::string g_last_error;
int flood_fill_islands(int nx, int ny, int nz, const uint8_t* d_active, const uint8_t* d_fixed_node, uint8_t* d_kept,
                       int* d_changed, cudaStream_t st);
}

namespace {

constexpr int kT = 256;
inline int grid_for(long long n) {
  long long b = (n + kT - 1) / kT;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

__global__ void k_copy_bool(long long n, const uint8_t* __restrict__ src, uint8_t* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src ? (uint8_t)(src[i] != 0) : (uint8_t)0;
}

__global__ void k_and_not(long long n, uint8_t* __restrict__ act, const uint8_t* __restrict__ excl) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (excl[i]) act[i] = 0;
}

__global__ void k_or_bits(long long n, uint8_t* __restrict__ bits, const uint8_t* __restrict__ mask, uint8_t axes) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (mask[i]) bits[i] |= axes;
}

__global__ void k_count(long long n, const uint8_t* __restrict__ mask, unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += mask[i] != 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// f[3n + c] += F[c] / count for the role's nodes (count from the device)
__global__ void k_add_force(long long n, const uint8_t* __restrict__ mask, const unsigned long long* __restrict__ count,
                            double f0, double f1, double f2, double* __restrict__ force) {
  const unsigned long long cnt = *count;
  if (cnt == 0) return;
  const double d = (double)cnt;
  const double v0 = f0 / d, v1 = f1 / d, v2 = f2 / d;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (mask[i]) {
      force[3 * i] += v0;
      force[3 * i + 1] += v1;
      force[3 * i + 2] += v2;
    }
}

__global__ void k_popcount_bits(long long n, const uint8_t* __restrict__ bits, unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    c += __popc((unsigned)(bits[i] & 7));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Device buffers of one call, released on every exit path.
struct Scratch {
  std::vector<void*> p;
  cudaStream_t st = nullptr;
  ~Scratch() {
    if (st) cudaStreamSynchronize(st);
    for (void* q : p) cudaFree(q);
    if (st) cudaStreamDestroy(st);
  }
  template <typename T> bool alloc(T** out, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T) + 16) != cudaSuccess) return false;
    p.push_back(q);
    *out = (T*)q;
    return true;
  }
};

int fail(const std::string& msg, int code) {
  vf::g_last_error = msg;
  return code;
}

}  // namespace

extern "C" {

int vf_assemble_grid(int32_t nx, int32_t ny, int32_t nz, int32_t n_roles, const int32_t* roles,
                     const uint8_t* const* masks, const double* meta, uint32_t flags, uint8_t* active_out,
                     uint8_t* fixed_bits_out, double* force_out, int64_t* n_active_out, int64_t* n_fixed_out) {
  if (nx < 1 || ny < 1 || nz < 1 || n_roles < 0 || (n_roles > 0 && (!roles || !masks || !meta)) || !active_out ||
      !fixed_bits_out || !force_out)
    return fail("vf_assemble_grid: invalid argument", VF_ERR_ARG);
  for (int i = 0; i < n_roles; ++i) {
    if (roles[i] < VF_ROLE_BUILD || roles[i] > VF_ROLE_LOAD) return fail("vf_assemble_grid: unknown role", VF_ERR_ARG);
    if (!masks[i]) return fail("vf_assemble_grid: null mask", VF_ERR_ARG);
  }
  const bool dev = (flags & VF_SOLVE_DEVICE_PTRS) != 0;
  const long long ne = (long long)nx * ny * nz;
  const long long nn = (long long)(nx + 1) * (ny + 1) * (nz + 1);
  Scratch sc;
  if (cudaStreamCreateWithFlags(&sc.st, cudaStreamNonBlocking) != cudaSuccess)
    return fail("vf_assemble_grid: no CUDA stream", VF_ERR_CUDA);
  cudaStream_t st = sc.st;
  uint8_t *d_act = nullptr, *d_bits = nullptr, *d_mask = nullptr;
  double* d_f = nullptr;
  unsigned long long* d_cnt = nullptr;
  if (dev) {
    d_act = active_out;
    d_bits = fixed_bits_out;
    d_f = force_out;
  } else if (!sc.alloc(&d_act, ne) || !sc.alloc(&d_bits, nn) || !sc.alloc(&d_f, 3 * nn)) {
    return fail("vf_assemble_grid: device allocation failed", VF_ERR_NOMEM);
  }
  if (!sc.alloc(&d_cnt, 2 * (size_t)(n_roles + 1)) || (!dev && !sc.alloc(&d_mask, nn > ne ? nn : ne)))
    return fail("vf_assemble_grid: device allocation failed", VF_ERR_NOMEM);
  cudaMemsetAsync(d_bits, 0, nn, st);
  cudaMemsetAsync(d_f, 0, sizeof(double) * 3 * nn, st);
  cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 2 * (n_roles + 1), st);
  // the mask of role i on the device (host masks go through one staging buffer,
  // stream-ordered with the kernels that read it)
  auto mask_of = [&](int i, long long n) -> const uint8_t* {
    if (dev) return masks[i];
    cudaMemcpyAsync(d_mask, masks[i], (size_t)n, cudaMemcpyHostToDevice, st);
    return d_mask;
  };
  int last_build = -1;
  for (int i = 0; i < n_roles; ++i)
    if (roles[i] == VF_ROLE_BUILD) last_build = i;
  vf::launch_k(k_copy_bool, grid_for(ne), kT, 0, st, ne, last_build >= 0 ? mask_of(last_build, ne) : nullptr, d_act);
  for (int i = 0; i < n_roles; ++i) {
    switch (roles[i]) {
      case VF_ROLE_EXCLUDE:
        vf::launch_k(k_and_not, grid_for(ne), kT, 0, st, ne, d_act, mask_of(i, ne));
        break;
      case VF_ROLE_BEARING: {
        const uint8_t axes = (uint8_t)((meta[3 * i] != 0.0 ? 1 : 0) | (meta[3 * i + 1] != 0.0 ? 2 : 0) |
                                       (meta[3 * i + 2] != 0.0 ? 4 : 0));
        if (axes) vf::launch_k(k_or_bits, grid_for(nn), kT, 0, st, nn, d_bits, mask_of(i, nn), axes);
        break;
      }
      case VF_ROLE_LOAD: {
        const uint8_t* m = mask_of(i, nn);
        vf::launch_k(k_count, grid_for(nn), kT, 0, st, nn, m, d_cnt + i);
        vf::launch_k(k_add_force, grid_for(nn), kT, 0, st, nn, m, (const unsigned long long*)(d_cnt + i),
                     meta[3 * i], meta[3 * i + 1], meta[3 * i + 2], d_f);
        break;
      }
      default:
        break;
    }
  }
  unsigned long long* d_tot = d_cnt + 2 * n_roles;
  vf::launch_k(k_count, grid_for(ne), kT, 0, st, ne, (const uint8_t*)d_act, d_tot);
  vf::launch_k(k_popcount_bits, grid_for(nn), kT, 0, st, nn, (const uint8_t*)d_bits, d_tot + 1);
  if (cudaGetLastError() != cudaSuccess) return fail("vf_assemble_grid: kernel launch failed", VF_ERR_CUDA);
  unsigned long long tot[2] = {0, 0};
  if (!dev) {
    cudaMemcpyAsync(active_out, d_act, (size_t)ne, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(fixed_bits_out, d_bits, (size_t)nn, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(force_out, d_f, sizeof(double) * 3 * nn, cudaMemcpyDeviceToHost, st);
  }
  cudaMemcpyAsync(tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return fail("vf_assemble_grid: CUDA error", VF_ERR_CUDA);
  if (n_active_out) *n_active_out = (int64_t)tot[0];
  if (n_fixed_out) *n_fixed_out = (int64_t)tot[1];
  return VF_OK;
}

int vf_drop_unsupported_islands_mask(int32_t nx, int32_t ny, int32_t nz, const uint8_t* active,
                                     const uint8_t* fixed_bits, uint32_t flags, uint8_t* kept_out,
                                     int64_t* n_removed) {
  if (nx < 1 || ny < 1 || nz < 1 || !active || !fixed_bits || !kept_out || !n_removed)
    return fail("vf_drop_unsupported_islands_mask: invalid argument", VF_ERR_ARG);
  const bool dev = (flags & VF_SOLVE_DEVICE_PTRS) != 0;
  const long long ne = (long long)nx * ny * nz;
  const long long nn = (long long)(nx + 1) * (ny + 1) * (nz + 1);
  Scratch sc;
  if (cudaStreamCreateWithFlags(&sc.st, cudaStreamNonBlocking) != cudaSuccess)
    return fail("vf_drop_unsupported_islands_mask: no CUDA stream", VF_ERR_CUDA);
  cudaStream_t st = sc.st;
  uint8_t *d_act = nullptr, *d_fix = nullptr, *d_kept = nullptr, *d_in = nullptr, *d_bits = nullptr;
  int* d_changed = nullptr;
  unsigned long long* d_cnt = nullptr;
  if (!sc.alloc(&d_act, ne) || !sc.alloc(&d_fix, nn) || !sc.alloc(&d_kept, ne) || !sc.alloc(&d_changed, 1) ||
      !sc.alloc(&d_cnt, 2))
    return fail("vf_drop_unsupported_islands_mask: device allocation failed", VF_ERR_NOMEM);
  if (dev) {
    d_in = (uint8_t*)active;
    d_bits = (uint8_t*)fixed_bits;
  } else {
    if (!sc.alloc(&d_in, ne) || !sc.alloc(&d_bits, nn))
      return fail("vf_drop_unsupported_islands_mask: device allocation failed", VF_ERR_NOMEM);
    cudaMemcpyAsync(d_in, active, (size_t)ne, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_bits, fixed_bits, (size_t)nn, cudaMemcpyHostToDevice, st);
  }
  cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), st);
  vf::launch_k(k_copy_bool, grid_for(ne), kT, 0, st, ne, (const uint8_t*)d_in, d_act);
  // a node carries a support when any of its DOFs is fixed
  vf::launch_k(k_copy_bool, grid_for(nn), kT, 0, st, nn, (const uint8_t*)d_bits, d_fix);
  if (vf::flood_fill_islands(nx, ny, nz, d_act, d_fix, d_kept, d_changed, st) < 0)
    return fail("vf_drop_unsupported_islands_mask: CUDA error in the flood fill", VF_ERR_CUDA);
  vf::launch_k(k_count, grid_for(ne), kT, 0, st, ne, (const uint8_t*)d_act, d_cnt);
  vf::launch_k(k_count, grid_for(ne), kT, 0, st, ne, (const uint8_t*)d_kept, d_cnt + 1);
  unsigned long long cnt[2] = {0, 0};
  cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return fail("vf_drop_unsupported_islands_mask: CUDA error", VF_ERR_CUDA);
  // core/fea.py:220-225: nothing reached from a support -> unchanged
  const uint8_t* res = cnt[1] == 0 ? d_act : d_kept;
  *n_removed = cnt[1] == 0 ? 0 : (int64_t)(cnt[0] - cnt[1]);
  if (cudaMemcpyAsync(kept_out, res, (size_t)ne, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return fail("vf_drop_unsupported_islands_mask: CUDA error", VF_ERR_CUDA);
  return VF_OK;
}

}  // extern "C"
