// Point-in-mesh inside test (voxelization), the step before grid assembly
// (the reference's core/inside_worker.py:_inside_mask_numpy, lines 105-147).
//
// One fixed ray direction d per query; a point is inside a closed triangle
// mesh when the ray from it crosses an odd number of triangles
// (Moeller-Trumbore: u >= -1e-7, v >= -1e-7, u + v <= 1 + 1e-7, t > 1e-7,
// triangles with |det| < 1e-9 skipped).  One thread per point; triangles are
// streamed through shared memory in tiles, pre-transformed once (v0, e1, e2,
// p = d x e2, 1/det).  Every product and sum is an explicitly rounded FP64
// operation in the reference's evaluation order (no contraction into FMAs),
// so the inside/outside decisions are the reference's bit for bit.
// The points are either given, or generated on the fly for a voxel grid
// (voxel centers in element order iz-fastest, or nodes in node order
// x-fastest: inside_worker.py:voxel_centers / node_coords).
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/voxfea.h"
#include "vf_common.cuh"

namespace vf {

namespace {

constexpr int kTile = 128;   // triangles per shared-memory tile
constexpr int kTriVals = 13; // v0 (3), e1 (3), e2 (3), pvec (3), inv_det (1)

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
// a.b = (a0 b0 + a1 b1) + a2 b2
__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return add(add(mul(a[0], b[0]), mul(a[1], b[1])), mul(a[2], b[2]));
}
// a x b, component-wise a1 b2 - a2 b1, ...
__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = sub(mul(a[1], b[2]), mul(a[2], b[1]));
  c[1] = sub(mul(a[2], b[0]), mul(a[0], b[2]));
  c[2] = sub(mul(a[0], b[1]), mul(a[1], b[0]));
}

struct Dir { double d[3]; };

__global__ void k_prepare_tris(const double* __restrict__ verts, const int64_t* __restrict__ faces, int64_t nf,
                               Dir dir, double* __restrict__ tri) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nf; t += (int64_t)gridDim.x * blockDim.x) {
    double v0[3], v1[3], v2[3], e1[3], e2[3], pv[3];
    for (int c = 0; c < 3; ++c) {
      v0[c] = verts[3 * faces[3 * t] + c];
      v1[c] = verts[3 * faces[3 * t + 1] + c];
      v2[c] = verts[3 * faces[3 * t + 2] + c];
      e1[c] = sub(v1[c], v0[c]);
      e2[c] = sub(v2[c], v0[c]);
    }
    cross3(dir.d, e2, pv);
    const double det = dot3(e1, pv);
    const bool parallel = fabs(det) < 1e-9;
    double* o = tri + kTriVals * t;
    for (int c = 0; c < 3; ++c) { o[c] = v0[c]; o[3 + c] = e1[c]; o[6 + c] = e2[c]; o[9 + c] = pv[c]; }
    o[12] = parallel ? 0.0 : 1.0 / det;   // 0 marks a skipped triangle
  }
}

// mode 0: explicit points (x, y, z) triples; 1: voxel centers; 2: grid nodes
__global__ void k_inside(int mode, const double* __restrict__ pts, int64_t npts, int nx, int ny, int nz,
                         double ox, double oy, double oz, double vs, const double* __restrict__ tri, int64_t nf,
                         Dir dir, uint8_t* __restrict__ out) {
  __shared__ double s_tri[kTile * kTriVals];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double p[3] = {0.0, 0.0, 0.0};
  const bool live = i < npts;
  if (live) {
    if (mode == 0) {
      p[0] = pts[3 * i]; p[1] = pts[3 * i + 1]; p[2] = pts[3 * i + 2];
    } else if (mode == 1) {   // element order: (ix * ny + iy) * nz + iz
      const int iz = (int)(i % nz), iy = (int)((i / nz) % ny), ix = (int)(i / ((int64_t)nz * ny));
      p[0] = add(mul(ix + 0.5, vs), ox);
      p[1] = add(mul(iy + 0.5, vs), oy);
      p[2] = add(mul(iz + 0.5, vs), oz);
    } else {                  // node order: ix + (nx+1) (iy + (ny+1) iz)
      const int nxp = nx + 1, nyp = ny + 1;
      const int ix = (int)(i % nxp), iy = (int)((i / nxp) % nyp), iz = (int)(i / ((int64_t)nxp * nyp));
      p[0] = add(mul((double)ix, vs), ox);
      p[1] = add(mul((double)iy, vs), oy);
      p[2] = add(mul((double)iz, vs), oz);
    }
  }
  int hits = 0;
  for (int64_t t0 = 0; t0 < nf; t0 += kTile) {
    const int nt = (int)((nf - t0 < kTile) ? (nf - t0) : kTile);
    __syncthreads();
    for (int k = threadIdx.x; k < nt * kTriVals; k += blockDim.x) s_tri[k] = tri[kTriVals * t0 + k];
    __syncthreads();
    if (!live) continue;
    for (int k = 0; k < nt; ++k) {
      const double* T = s_tri + kTriVals * k;
      const double inv = T[12];
      if (inv == 0.0) continue;   // |det| < 1e-9
      const double tv[3] = {sub(p[0], T[0]), sub(p[1], T[1]), sub(p[2], T[2])};
      const double u = mul(dot3(tv, T + 9), inv);
      double q[3];
      cross3(tv, T + 3, q);
      const double v = mul(dot3(dir.d, q), inv);
      const double t = mul(dot3(T + 6, q), inv);
      hits += (u >= -1e-7 && v >= -1e-7 && add(u, v) <= 1.0 + 1e-7 && t > 1e-7) ? 1 : 0;
    }
  }
  if (live) out[i] = (uint8_t)(hits & 1);
}

int inside_run(int mode, const double* verts, int64_t nv, const int64_t* faces, int64_t nf, const double* pts,
               int64_t npts, const int32_t* dims, const double* origin, double vsize, const double* dir3,
               uint8_t* out) {
  if (npts <= 0) return VF_OK;
  for (int64_t k = 0; k < 3 * nf; ++k)   // the kernels index verts by these: check them here
    if (faces[k] < 0 || faces[k] >= nv) return VF_ERR_ARG;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return VF_ERR_CUDA;
  double *d_v = nullptr, *d_tri = nullptr, *d_p = nullptr;
  int64_t* d_f = nullptr;
  uint8_t* d_o = nullptr;
  int rc = VF_OK;
  const size_t nfs = (size_t)(nf > 0 ? nf : 1);
  if (cudaMalloc(&d_v, sizeof(double) * 3 * (size_t)(nv > 0 ? nv : 1)) != cudaSuccess ||
      cudaMalloc(&d_f, sizeof(int64_t) * 3 * nfs) != cudaSuccess ||
      cudaMalloc(&d_tri, sizeof(double) * kTriVals * nfs) != cudaSuccess ||
      cudaMalloc(&d_o, (size_t)npts) != cudaSuccess ||
      (mode == 0 && cudaMalloc(&d_p, sizeof(double) * 3 * (size_t)npts) != cudaSuccess)) {
    rc = VF_ERR_NOMEM;
  }
  Dir d;
  for (int c = 0; c < 3; ++c) d.d[c] = dir3[c];
  if (rc == VF_OK) {
    if (nf > 0) {
      cudaMemcpyAsync(d_v, verts, sizeof(double) * 3 * (size_t)nv, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(d_f, faces, sizeof(int64_t) * 3 * (size_t)nf, cudaMemcpyHostToDevice, st);
      launch_k(k_prepare_tris, (int)((nf + 255) / 256 < 4096 ? (nf + 255) / 256 : 4096), 256, 0, st,
               (const double*)d_v, (const int64_t*)d_f, nf, d, d_tri);
    }
    if (mode == 0) cudaMemcpyAsync(d_p, pts, sizeof(double) * 3 * (size_t)npts, cudaMemcpyHostToDevice, st);
    const int nx = dims ? dims[0] : 0, ny = dims ? dims[1] : 0, nz = dims ? dims[2] : 0;
    const double ox = origin ? origin[0] : 0.0, oy = origin ? origin[1] : 0.0, oz = origin ? origin[2] : 0.0;
    launch_k(k_inside, (unsigned)((npts + 255) / 256), 256, 0, st, mode, (const double*)d_p, npts, nx, ny, nz, ox, oy,
             oz, vsize, (const double*)d_tri, nf, d, d_o);
    cudaMemcpyAsync(out, d_o, (size_t)npts, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = VF_ERR_CUDA;
  }
  cudaFree(d_v); cudaFree(d_f); cudaFree(d_tri); cudaFree(d_o); cudaFree(d_p);
  cudaStreamDestroy(st);
  return rc;
}

}  // namespace

}  // namespace vf

extern "C" {

int vf_inside_points(const double* verts, int64_t nv, const int64_t* faces, int64_t nf, const double* points,
                     int64_t npts, const double* dir3, uint8_t* out) {
  if (npts < 0 || nf < 0 || nv < 0 || !dir3 || (npts > 0 && (!points || !out)) || (nf > 0 && (!verts || !faces)))
    return VF_ERR_ARG;
  return vf::inside_run(0, verts, nv, faces, nf, points, npts, nullptr, nullptr, 0.0, dir3, out);
}

int vf_inside_grid(const double* verts, int64_t nv, const int64_t* faces, int64_t nf, const int32_t* dims3,
                   const double* origin3, double vsize, int32_t target, const double* dir3, uint8_t* out) {
  if (!dims3 || !origin3 || !dir3 || !out || nf < 0 || nv < 0 || (nf > 0 && (!verts || !faces)) ||
      (target != 0 && target != 1) || dims3[0] < 1 || dims3[1] < 1 || dims3[2] < 1)
    return VF_ERR_ARG;
  const int64_t n = target == 0 ? (int64_t)dims3[0] * dims3[1] * dims3[2]
                                : (int64_t)(dims3[0] + 1) * (dims3[1] + 1) * (dims3[2] + 1);
  return vf::inside_run(target == 0 ? 1 : 2, verts, nv, faces, nf, nullptr, n, dims3, origin3, vsize, dir3, out);
}

}  // extern "C"
