// The learned preconditioner stage: U-Net inference on one level of the
// multigrid hierarchy, entirely on the device (capturable in the PCG graphs).
//
// Network (3 levels, 16/32/64 channels, 3x3x3 convolutions of vf_nn.cu):
//   in(16: r/s x3, occupancy, log-modulus, 0...)
//   a0 = relu(c0(in))            16 -> 16   U-Net level 0
//   s0 = relu(c1(a0))            16 -> 16
//   p1 = avgpool2(s0)
//   a1 = relu(c2(p1))            16 -> 32   level 1
//   s1 = relu(c3(a1))            32 -> 32
//   p2 = avgpool2(s1)
//   a2 = relu(c4(p2))            32 -> 64   level 2
//   b2 = relu(c5(a2))            64 -> 64
//   u1 = up2(b2)
//   c1o = relu(c6(u1) + s1)      64 -> 32
//   d1 = relu(c7(c1o))           32 -> 32
//   u0 = up2(d1)
//   c0o = relu(c8(u0) + s0)      32 -> 16
//   y  = c9(c0o)                 16 -> 16 (channels 0..2 used), FP32
// The U-Net grid is the node grid of hierarchy level L padded to multiples of
// 4; the correction on level L is e = mask * y[0..2] * s / Eref (s = RMS of
// the input residual, Eref = the largest voxel modulus), prolongated to the
// fine grid by the V-cycle's own P.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "vf_common.cuh"
#include "vf_nn.cuh"

namespace vf {

namespace {

using bf16 = __nv_bfloat16;

constexpr int kLayers = 10;
constexpr int kCin[kLayers] = {16, 16, 16, 32, 32, 64, 64, 32, 32, 16};
constexpr int kCout[kLayers] = {16, 16, 32, 32, 64, 64, 32, 32, 16, 16};

__global__ void k_nn_features(Grid g0, const double* __restrict__ E0, int L, const double* __restrict__ eref_dev,
                              int nx1, int ny1, int nz1, int X, int Y, int Z, float2* __restrict__ feat) {
  const long long n = (long long)X * Y * Z;
  const int h = 1 << L;
  const double eref = *eref_dev > 0.0 ? *eref_dev : 1.0;
  const double thr = 1e-6 * eref;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long long)X * Y));
    float2 f = make_float2(0.f, 0.f);
    if (x < nx1 && y < ny1 && z < nz1) {
      int cnt = 0, act = 0;
      double lsum = 0.0;
      for (int ez = z * h - h; ez < z * h + h; ++ez)
        for (int ey = y * h - h; ey < y * h + h; ++ey)
          for (int ex = x * h - h; ex < x * h + h; ++ex) {
            ++cnt;
            if (ex < 0 || ey < 0 || ez < 0 || ex >= g0.lx || ey >= g0.ly || ez >= g0.lz) continue;
            const double e = E0[g0.idx(ex, ey, ez)];
            if (e > thr) {
              ++act;
              lsum += log10(e / eref);
            }
          }
      f.x = (float)act / (float)cnt;
      f.y = act ? (float)(lsum / act / 6.0 + 1.0) : 0.f;
    }
    feat[i] = f;
  }
}

// sum of r^2 over the level's padded vector -> partials (fixed grid), then scale
template <typename T>
__global__ void k_nn_sumsq(long long n3, const T* __restrict__ r, double* __restrict__ part, const int* skip) {
  if (skip && *skip) return;
  __shared__ double sh[256];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)r[i];
    s += v * v;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_nn_scale(const double* __restrict__ part, int nb, double nnodes, float* __restrict__ scale,
                           const int* skip) {
  if (skip && *skip) return;
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < nb; ++i) s += part[i];
  const double rms = sqrt(s / (3.0 * nnodes));
  scale[0] = rms > 0.0 ? (float)rms : 1.f;
}

template <typename T>
__global__ void k_nn_input(Grid gL, const T* __restrict__ r, const float2* __restrict__ feat,
                           const float* __restrict__ scale, int X, int Y, int Z, bf16* __restrict__ in,
                           const int* skip) {
  if (skip && *skip) return;
  const long long n = (long long)X * Y * Z;
  const float inv = 1.f / scale[0];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long long)X * Y));
    float v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = 0.f;
    if (x <= gL.lx && y <= gL.ly && z <= gL.lz) {
      const long long p3 = 3LL * gL.idx(x, y, z);
      v[0] = (float)r[p3] * inv;
      v[1] = (float)r[p3 + 1] * inv;
      v[2] = (float)r[p3 + 2] * inv;
      const float2 f = feat[i];
      v[3] = f.x;
      v[4] = f.y;
    }
    __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(in + i * 16);
#pragma unroll
    for (int c = 0; c < 8; ++c) o[c] = __floats2bfloat162_rn(v[2 * c], v[2 * c + 1]);
  }
}

// e (level vector, every padded node written) = mask * y[0..2] * s / Eref
template <typename T>
__global__ void k_nn_output(Grid gL, const float* __restrict__ y, const float* __restrict__ scale,
                            const double* __restrict__ eref_dev, int X, int Y, const uint8_t* __restrict__ mask,
                            T* __restrict__ e, const int* skip) {
  if (skip && *skip) return;
  const double eref = *eref_dev > 0.0 ? *eref_dev : 1.0;
  const double s = (double)scale[0] / eref;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < gL.n; p += gridDim.x * blockDim.x) {
    const int x = p % gL.px - 1, y0 = (p / gL.px) % gL.py - 1, z = p / (gL.px * gL.py) - 1;
    const uint8_t m = mask[p];
    T o0 = 0, o1 = 0, o2 = 0;
    if (m && x >= 0 && y0 >= 0 && z >= 0 && x <= gL.lx && y0 <= gL.ly && z <= gL.lz) {
      const float* yv = y + (((long long)z * Y + y0) * X + x) * 16;
      if (m & 1) o0 = (T)(yv[0] * s);
      if (m & 2) o1 = (T)(yv[1] * s);
      if (m & 4) o2 = (T)(yv[2] * s);
    }
    e[3LL * p] = o0;
    e[3LL * p + 1] = o1;
    e[3LL * p + 2] = o2;
  }
}

// 2x2x2 average pool, channels-last, C = 16 or 32 (8-channel chunks)
__global__ void k_nn_pool(const bf16* __restrict__ a, int X, int Y, int Z, int C, bf16* __restrict__ o,
                          const int* skip) {
  if (skip && *skip) return;
  const int Xo = X / 2, Yo = Y / 2, Zo = Z / 2, CH = C / 8;
  const long long n = (long long)Xo * Yo * Zo * CH;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % CH);
    const long long v = i / CH;
    const int x = (int)(v % Xo), y = (int)((v / Xo) % Yo), z = (int)(v / ((long long)Xo * Yo));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const bf16* src = a + ((((long long)(2 * z + dz) * Y + (2 * y + dy)) * X + (2 * x + dx)) * C) + c * 8;
          const uint4 w = *reinterpret_cast<const uint4*>(src);
          const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&w);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const float2 f = __bfloat1622float2(h[k]);
            acc[2 * k] += f.x;
            acc[2 * k + 1] += f.y;
          }
        }
    uint4 w;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&w);
#pragma unroll
    for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(acc[2 * k] * 0.125f, acc[2 * k + 1] * 0.125f);
    *reinterpret_cast<uint4*>(o + v * C + c * 8) = w;
  }
}

// nearest-neighbour 2x upsampling, channels-last (8-channel chunks)
__global__ void k_nn_up(const bf16* __restrict__ a, int Xc, int Yc, int Zc, int C, bf16* __restrict__ o,
                        const int* skip) {
  if (skip && *skip) return;
  const int X = 2 * Xc, Y = 2 * Yc, Z = 2 * Zc, CH = C / 8;
  const long long n = (long long)X * Y * Z * CH;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % CH);
    const long long v = i / CH;
    const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
    const long long s = (((long long)(z / 2) * Yc + (y / 2)) * Xc + (x / 2)) * C + c * 8;
    *reinterpret_cast<uint4*>(o + v * C + c * 8) = *reinterpret_cast<const uint4*>(a + s);
  }
}

// max of a non-negative array: fixed grid of partial maxima, one finalizing block
__global__ void k_max_part(const double* __restrict__ v, long long n, double* __restrict__ part) {
  __shared__ double sh[256];
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, v[i]);
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_max_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double m = 0.0;
  for (int i = 0; i < nb; ++i) m = fmax(m, part[i]);
  out[0] = m;
}

__global__ void k_f32_to_bf16(const float* __restrict__ a, long long n, bf16* __restrict__ o) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    o[i] = __float2bfloat16_rn(a[i]);
}

int grid_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

long long nn_param_count() {
  long long n = 0;
  for (int k = 0; k < kLayers; ++k) n += 27LL * kCin[k] * kCout[k] + kCout[k];
  return n;
}

struct NnStage {
  int level = 1;
  int X[3] = {0, 0, 0}, Y[3] = {0, 0, 0}, Z[3] = {0, 0, 0};
  int nx1 = 0, ny1 = 0, nz1 = 0;
  const double* eref_dev = nullptr;   // device max modulus (set with the features)
  bool have_weights = false;
  bf16* w[kLayers] = {};
  float* b[kLayers] = {};
  float2* feat = nullptr;
  bf16 *in = nullptr, *a0 = nullptr, *s0 = nullptr, *p1 = nullptr, *a1 = nullptr, *s1 = nullptr, *p2 = nullptr;
  bf16 *a2 = nullptr, *b2 = nullptr, *u1 = nullptr, *c1 = nullptr, *d1 = nullptr, *u0 = nullptr, *c0 = nullptr;
  float* y = nullptr;
  float* wstage = nullptr;   // FP32 staging of the uploaded parameters
  double* part = nullptr;    // sum-of-squares partials
  float* scale = nullptr;
  std::vector<void*> allocs;
  int* err = nullptr;        // the solver's error flag (expired bounded waits of the convolutions)
};

namespace {
template <typename P>
cudaError_t nn_alloc(NnStage* s, P** p, size_t count, cudaStream_t st) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(P));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(P), st);   // ordered with the solver stream
  s->allocs.push_back(q);
  *p = (P*)q;
  return e;
}
constexpr int kPartBlocks = 148 * 4;
}  // namespace

void nn_destroy(NnStage* s) {
  if (!s) return;
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

// gL: grid of hierarchy level `level` (lx, ly, lz voxels).
NnStage* nn_create(const Grid& gL, int level, cudaStream_t st, cudaError_t* err) {
  NnStage* s = new NnStage();
  s->level = level;
  s->nx1 = gL.lx + 1; s->ny1 = gL.ly + 1; s->nz1 = gL.lz + 1;
  s->X[0] = (s->nx1 + 3) / 4 * 4; s->Y[0] = (s->ny1 + 3) / 4 * 4; s->Z[0] = (s->nz1 + 3) / 4 * 4;
  for (int k = 1; k < 3; ++k) { s->X[k] = s->X[k - 1] / 2; s->Y[k] = s->Y[k - 1] / 2; s->Z[k] = s->Z[k - 1] / 2; }
  const size_t v0 = (size_t)s->X[0] * s->Y[0] * s->Z[0], v1 = v0 / 8, v2 = v0 / 64;
  cudaError_t e = cudaSuccess;
  auto A = [&](auto** p, size_t cnt) { if (e == cudaSuccess) e = nn_alloc(s, p, cnt, st); };
  for (int k = 0; k < kLayers; ++k) {
    A(&s->w[k], 27 * (size_t)kCin[k] * kCout[k]);
    A(&s->b[k], (size_t)kCout[k]);
  }
  A(&s->feat, v0);
  A(&s->in, v0 * 16); A(&s->a0, v0 * 16); A(&s->s0, v0 * 16);
  A(&s->p1, v1 * 16); A(&s->a1, v1 * 32); A(&s->s1, v1 * 32);
  A(&s->p2, v2 * 32); A(&s->a2, v2 * 64); A(&s->b2, v2 * 64);
  A(&s->u1, v1 * 64); A(&s->c1, v1 * 32); A(&s->d1, v1 * 32);
  A(&s->u0, v0 * 32); A(&s->c0, v0 * 16);
  A(&s->y, v0 * 16);
  A(&s->wstage, (size_t)nn_param_count());
  A(&s->part, (size_t)kPartBlocks);
  A(&s->scale, 1);
  if (err) *err = e;
  if (e != cudaSuccess) { nn_destroy(s); return nullptr; }
  return s;
}

void nn_dims(const NnStage* s, int* xyz) { xyz[0] = s->X[0]; xyz[1] = s->Y[0]; xyz[2] = s->Z[0]; }

// Parameters: per layer W[27][cout][cin] then b[cout], FP32, in layer order.
cudaError_t nn_set_weights(NnStage* s, const float* host, cudaStream_t st) {
  const long long n = nn_param_count();
  cudaError_t e = cudaMemcpyAsync(s->wstage, host, sizeof(float) * n, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  long long off = 0;
  for (int k = 0; k < kLayers; ++k) {
    const long long nw = 27LL * kCin[k] * kCout[k];
    launch_k(k_f32_to_bf16, grid_for(nw), 256, 0, st, (const float*)(s->wstage + off), nw, s->w[k]);
    off += nw;
    e = cudaMemcpyAsync(s->b[k], s->wstage + off, sizeof(float) * kCout[k], cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    off += kCout[k];
  }
  s->have_weights = true;
  return cudaGetLastError();
}

bool nn_has_weights(const NnStage* s) { return s && s->have_weights; }

// Static per-geometry features from the fine modulus (padded voxel layout).
void nn_set_features(NnStage* s, const Grid& g0, const double* E0, const double* eref_dev, cudaStream_t st) {
  s->eref_dev = eref_dev;
  const long long n = (long long)s->X[0] * s->Y[0] * s->Z[0];
  launch_k(k_nn_features, grid_for(n), 256, 0, st, g0, E0, s->level, eref_dev, s->nx1, s->ny1, s->nz1, s->X[0],
           s->Y[0], s->Z[0], s->feat);
}

void launch_max_f64(const double* v, long long n, double* out, cudaStream_t st) {
  // out[1 .. kPartBlocks] is scratch for the partial maxima
  launch_k(k_max_part, kPartBlocks, 256, 0, st, v, n, out + 1);
  launch_k(k_max_final, 1, 32, 0, st, (const double*)(out + 1), kPartBlocks, out);
}

// U-Net input from a level-L residual (padded layout of gL): BF16 [Z][Y][X][16].
template <typename T>
void nn_make_input(NnStage* s, const Grid& gL, const T* r, const int* skip, cudaStream_t st) {
  const long long n3 = 3LL * gL.n;
  launch_k(k_nn_sumsq<T>, kPartBlocks, 256, 0, st, n3, r, s->part, skip);
  launch_k(k_nn_scale, 1, 32, 0, st, (const double*)s->part, kPartBlocks,
           (double)s->nx1 * s->ny1 * s->nz1, s->scale, skip);
  const long long nv = (long long)s->X[0] * s->Y[0] * s->Z[0];
  launch_k(k_nn_input<T>, grid_for(nv), 256, 0, st, gL, r, (const float2*)s->feat, (const float*)s->scale, s->X[0],
           s->Y[0], s->Z[0], s->in, skip);
}

void nn_set_error_flag(NnStage* s, int* err) { s->err = err; }

void nn_forward(NnStage* s, const int* skip, cudaStream_t st) {
  auto conv = [&](int k, int lv, const bf16* in, bf16* out, const bf16* sk, bool relu, float* of32) {
    NnConvArgs a{in, s->w[k], s->b[k], sk, nullptr, out, of32, s->X[lv], s->Y[lv], s->Z[lv], relu ? 1 : 0};
    a.skip_flag = skip;
    a.err = s->err;
    nn_conv_forward(kCin[k], kCout[k], a, st);
  };
  const long long v1 = (long long)s->X[1] * s->Y[1] * s->Z[1], v0 = v1 * 8, v2 = v1 / 8;
  conv(0, 0, s->in, s->a0, nullptr, true, nullptr);
  conv(1, 0, s->a0, s->s0, nullptr, true, nullptr);
  launch_k(k_nn_pool, grid_for(v1 * 2), 256, 0, st, (const bf16*)s->s0, s->X[0], s->Y[0], s->Z[0], 16, s->p1, skip);
  conv(2, 1, s->p1, s->a1, nullptr, true, nullptr);
  conv(3, 1, s->a1, s->s1, nullptr, true, nullptr);
  launch_k(k_nn_pool, grid_for(v2 * 4), 256, 0, st, (const bf16*)s->s1, s->X[1], s->Y[1], s->Z[1], 32, s->p2, skip);
  conv(4, 2, s->p2, s->a2, nullptr, true, nullptr);
  conv(5, 2, s->a2, s->b2, nullptr, true, nullptr);
  launch_k(k_nn_up, grid_for(v1 * 8), 256, 0, st, (const bf16*)s->b2, s->X[2], s->Y[2], s->Z[2], 64, s->u1, skip);
  conv(6, 1, s->u1, s->c1, s->s1, true, nullptr);
  conv(7, 1, s->c1, s->d1, nullptr, true, nullptr);
  launch_k(k_nn_up, grid_for(v0 * 4), 256, 0, st, (const bf16*)s->d1, s->X[1], s->Y[1], s->Z[1], 32, s->u0, skip);
  conv(8, 0, s->u0, s->c0, s->s0, true, nullptr);
  conv(9, 0, s->c0, nullptr, nullptr, false, s->y);
}

template <typename T>
void nn_make_output(NnStage* s, const Grid& gL, const uint8_t* maskL, T* e, const int* skip, cudaStream_t st) {
  launch_k(k_nn_output<T>, grid_for(gL.n), 256, 0, st, gL, (const float*)s->y, (const float*)s->scale,
           s->eref_dev, s->X[0], s->Y[0], maskL, e, skip);
}

const void* nn_input_buffer(const NnStage* s) { return s->in; }
const float* nn_scale_buffer(const NnStage* s) { return s->scale; }

template void nn_make_input<float>(NnStage*, const Grid&, const float*, const int*, cudaStream_t);
template void nn_make_input<double>(NnStage*, const Grid&, const double*, const int*, cudaStream_t);
template void nn_make_output<float>(NnStage*, const Grid&, const uint8_t*, float*, const int*, cudaStream_t);
template void nn_make_output<double>(NnStage*, const Grid&, const uint8_t*, double*, const int*, cudaStream_t);

}  // namespace vf
