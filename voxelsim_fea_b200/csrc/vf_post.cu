// Post-processing on the device, next to the solution already in HBM:
//   * centroid von Mises stress  (core/fea.py:604-626)
//   * element strain energy u_e^T KE u_e  (core/fea.py:595-602)
// and the pre-step that drops voxel islands not connected to a support
// (core/fea.py:165-227) as an in-place 6-connected flood fill.
#include "../../include/voxfea.h"
#include "vf_common.cuh"

namespace vf {

namespace {

struct B0Tab { double b[6 * 24]; };
struct KETab { double k[576]; };

__device__ __forceinline__ void gather_ue(const Grid& g, const double* __restrict__ u, int ix, int iy, int iz,
                                          double ue[24]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int ox = (k == 1 || k == 2 || k == 5 || k == 6);
    const int oy = (k == 2 || k == 3 || k == 6 || k == 7);
    const int oz = (k >= 4);
    const long long p = 3 * (long long)g.idx(ix + ox, iy + oy, iz + oz);
    ue[3 * k] = u[p]; ue[3 * k + 1] = u[p + 1]; ue[3 * k + 2] = u[p + 2];
  }
}

__global__ void k_von_mises(Grid g, const double* __restrict__ u, const double* __restrict__ Es,
                            const double* __restrict__ nu_ref, double nu, const uint8_t* __restrict__ active,
                            const B0Tab B, double* __restrict__ vm) {
  const long long ne = (long long)g.lx * g.ly * g.lz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
    if (active && !active[e]) { vm[e] = 0.0; continue; }
    const int iz = (int)(e % g.lz);
    const long long t = e / g.lz;
    const int iy = (int)(t % g.ly), ix = (int)(t / g.ly);
    double ue[24];
    gather_ue(g, u, ix, iy, iz, ue);
    double eps[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < 24; ++j) s += B.b[r * 24 + j] * ue[j];
      eps[r] = s;
    }
    const double n = nu_ref ? nu_ref[e] : nu;
    const double c = 1.0 / ((1.0 + n) * (1.0 - 2.0 * n));
    const double gsh = c * (1.0 - 2.0 * n) / 2.0;
    const double E = Es[e];
    const double sx = E * c * ((1.0 - n) * eps[0] + n * eps[1] + n * eps[2]);
    const double sy = E * c * (n * eps[0] + (1.0 - n) * eps[1] + n * eps[2]);
    const double sz = E * c * (n * eps[0] + n * eps[1] + (1.0 - n) * eps[2]);
    const double txy = E * gsh * eps[3], tyz = E * gsh * eps[4], tzx = E * gsh * eps[5];
    const double v = 0.5 * ((sx - sy) * (sx - sy) + (sy - sz) * (sy - sz) + (sz - sx) * (sz - sx)) +
                     3.0 * (txy * txy + tyz * tyz + tzx * tzx);
    vm[e] = sqrt(v > 0.0 ? v : 0.0);
  }
}

__global__ void k_strain_energy(Grid g, const double* __restrict__ u, const uint8_t* __restrict__ active,
                                const KETab K, double* __restrict__ se) {
  const long long ne = (long long)g.lx * g.ly * g.lz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
    if (active && !active[e]) { se[e] = 0.0; continue; }
    const int iz = (int)(e % g.lz);
    const long long t = e / g.lz;
    const int iy = (int)(t % g.ly), ix = (int)(t / g.ly);
    double ue[24];
    gather_ue(g, u, ix, iy, iz, ue);
    double s = 0.0;
    for (int i = 0; i < 24; ++i) {
      double ki = 0.0;
#pragma unroll
      for (int j = 0; j < 24; ++j) ki += K.k[i * 24 + j] * ue[j];
      s += ue[i] * ki;
    }
    se[e] = s;
  }
}

// seed[e] = active[e] && an element node is fixed (fea.py:165-177)
__global__ void k_island_seed(int nx, int ny, int nz, const uint8_t* __restrict__ active,
                              const uint8_t* __restrict__ fixed_node, uint8_t* __restrict__ kept) {
  const long long ne = (long long)nx * ny * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(e % nz);
    const long long t = e / nz;
    const int iy = (int)(t % ny), ix = (int)(t / ny);
    uint8_t s = 0;
    if (active[e]) {
      for (int k = 0; k < 8 && !s; ++k) {
        const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
        const long long nid = (ix + ox) + (long long)(nx + 1) * ((iy + oy) + (long long)(ny + 1) * (iz + oz));
        s = fixed_node[nid];
      }
    }
    kept[e] = s ? 1 : 0;
  }
}

// One in-place dilation pass (monotone: kept only grows, so any visiting
// order reaches the same fixed point as fea.py:193-204's synchronous passes).
__global__ void k_island_grow(int nx, int ny, int nz, const uint8_t* __restrict__ active, uint8_t* kept,
                              int* changed) {
  const long long ne = (long long)nx * ny * nz;
  int any = 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
    if (!active[e] || kept[e]) continue;
    const int iz = (int)(e % nz);
    const long long t = e / nz;
    const int iy = (int)(t % ny), ix = (int)(t / ny);
    const long long sx = (long long)ny * nz, sy = nz;
    uint8_t g = 0;
    if (ix > 0) g |= ((volatile uint8_t*)kept)[e - sx];
    if (ix + 1 < nx) g |= ((volatile uint8_t*)kept)[e + sx];
    if (iy > 0) g |= ((volatile uint8_t*)kept)[e - sy];
    if (iy + 1 < ny) g |= ((volatile uint8_t*)kept)[e + sy];
    if (iz > 0) g |= ((volatile uint8_t*)kept)[e - 1];
    if (iz + 1 < nz) g |= ((volatile uint8_t*)kept)[e + 1];
    if (g) { kept[e] = 1; any = 1; }
  }
  if (any) *changed = 1;
}

}  // namespace

void launch_von_mises(const Grid& g, const double* u_pad, const double* Es_ref, const double* nu_ref, double nu,
                      const uint8_t* active_ref, const double* B0, double* vm_ref, cudaStream_t st) {
  B0Tab B;
  for (int i = 0; i < 144; ++i) B.b[i] = B0[i];
  const long long ne = (long long)g.lx * g.ly * g.lz;
  int blocks = (int)((ne + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  launch_k(k_von_mises, blocks, 256, 0, st, g, u_pad, Es_ref, nu_ref, nu, active_ref, B, vm_ref);
}

void launch_strain_energy_tab(const Grid& g, const double* u_pad, const uint8_t* active_ref, const double* KE,
                              double* se_ref, cudaStream_t st) {
  KETab K;
  for (int i = 0; i < 576; ++i) K.k[i] = KE[i];
  const long long ne = (long long)g.lx * g.ly * g.lz;
  int blocks = (int)((ne + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  launch_k(k_strain_energy, blocks, 256, 0, st, g, u_pad, active_ref, K, se_ref);
}

// Returns the number of dilation passes run.  d_changed: one device int.
int flood_fill_islands(int nx, int ny, int nz, const uint8_t* d_active, const uint8_t* d_fixed_node,
                       uint8_t* d_kept, int* d_changed, cudaStream_t st) {
  const long long ne = (long long)nx * ny * nz;
  int blocks = (int)((ne + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  launch_k(k_island_seed, blocks, 256, 0, st, nx, ny, nz, d_active, d_fixed_node, d_kept);
  int passes = 0;
  const long long max_passes = 4 * ((long long)nx + ny + nz) + ne;   // monotone: ends long before
  for (;;) {
    int h_changed = 0;
    cudaMemsetAsync(d_changed, 0, sizeof(int), st);
    for (int k = 0; k < 8; ++k) launch_k(k_island_grow, blocks, 256, 0, st, nx, ny, nz, d_active, d_kept, d_changed);
    passes += 8;
    cudaMemcpyAsync(&h_changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
    if (!h_changed || passes > max_passes) break;
  }
  return passes;
}

}  // namespace vf

// ---------------------------------------------------------------------------
// Per-element displacement field of the result views (solve_worker.py:374-388):
// each voxel gets the mean of its 8 corner nodes' displacement magnitude.
// Reference node / element orders; host arrays in, FP32 field out.
// ---------------------------------------------------------------------------
namespace vf {
namespace {
__global__ void k_elem_disp(int nx, int ny, int nz, const double* __restrict__ u, float* __restrict__ out) {
  const long long ne = (long long)nx * ny * nz;
  const int nx1 = nx + 1, ny1 = ny + 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(e % nz), iy = (int)((e / nz) % ny), ix = (int)(e / ((long long)nz * ny));
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {   // corner order of build_edof (fea.py:33-36)
      const int ox = (k == 1 || k == 2 || k == 5 || k == 6), oy = (k == 2 || k == 3 || k == 6 || k == 7), oz = k >= 4;
      const long long n = (ix + ox) + (long long)nx1 * ((iy + oy) + (long long)ny1 * (iz + oz));
      const double a = u[3 * n], b = u[3 * n + 1], c = u[3 * n + 2];
      s += sqrt(a * a + b * b + c * c);
    }
    out[e] = (float)(s / 8.0);
  }
}
}  // namespace
}  // namespace vf

extern "C" int vf_element_displacement(int32_t nx, int32_t ny, int32_t nz, const double* u, float* disp_out) {
  if (nx < 1 || ny < 1 || nz < 1 || !u || !disp_out) return VF_ERR_ARG;
  const size_t ndof = 3 * (size_t)(nx + 1) * (ny + 1) * (nz + 1), ne = (size_t)nx * ny * nz;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return VF_ERR_CUDA;
  double* d_u = nullptr;
  float* d_o = nullptr;
  int rc = VF_OK;
  if (cudaMalloc(&d_u, sizeof(double) * ndof) != cudaSuccess || cudaMalloc(&d_o, sizeof(float) * ne) != cudaSuccess) {
    rc = VF_ERR_NOMEM;
  } else {
    cudaMemcpyAsync(d_u, u, sizeof(double) * ndof, cudaMemcpyHostToDevice, st);
    const long long b = ((long long)ne + 255) / 256;
    vf::launch_k(vf::k_elem_disp, (int)(b < 148 * 16 ? b : 148 * 16), 256, 0, st, nx, ny, nz, (const double*)d_u, d_o);
    cudaMemcpyAsync(disp_out, d_o, sizeof(float) * ne, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = VF_ERR_CUDA;
  }
  cudaFree(d_u);
  cudaFree(d_o);
  cudaStreamDestroy(st);
  return rc;
}
