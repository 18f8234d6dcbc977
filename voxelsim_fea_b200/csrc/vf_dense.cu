// Coarsest-level direct solve in FP64: the assembled coarsest operator (with
// identity rows on non-free DOFs) is factored A = L L^T by a blocked
// right-looking Cholesky, inverted as A^{-1} = Y^T Y with Y = L^{-1}, and each
// V-cycle applies the explicit inverse with one GEMV.  All kernels are plain
// CUDA-core FP64 (the coarsest level holds a few thousand DOFs at most);
// the factorization runs once per set_material, outside the iteration.
// Replaces the reference's 30-sweep Jacobi "coarse solve" (core/multigrid.py:428-429)
// when VF_COARSEST_CHOLESKY is selected.
#include <algorithm>

#include "vf_common.cuh"

namespace vf {

namespace {

constexpr int NB = 32;

// Dense row-major A from the coarsest stencil; node order = reference order
// of the level's nodes, DOF 3*node + c.
__global__ void k_dense_assemble(Grid c, const double* __restrict__ st, const uint8_t* __restrict__ cm,
                                 double* __restrict__ A, int n) {
  const int nx1 = c.lx + 1, ny1 = c.ly + 1, nint = nx1 * ny1 * (c.lz + 1);
  const long long ns = c.n;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nint * 27; t += gridDim.x * blockDim.x) {
    const int r = t / 27, s = t % 27;
    const int x = r % nx1, rr = r / nx1, y = rr % ny1, z = rr / ny1;
    const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
    const int X = x + dx, Y = y + dy, Z = z + dz;
    if (X < 0 || X > c.lx || Y < 0 || Y > c.ly || Z < 0 || Z > c.lz) continue;
    const int q = X + nx1 * (Y + ny1 * Z);
    const int p = c.idx(x, y, z);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        A[(long long)(3 * r + a) * n + 3 * q + b] = st[((long long)s * 9 + a * 3 + b) * ns + p];
    if (s == 13) {
      const uint8_t m = cm[p];
      for (int a = 0; a < 3; ++a)
        if (!((m >> a) & 1)) A[(long long)(3 * r + a) * n + 3 * r + a] = 1.0;
    }
  }
}

// Factor the nb x nb diagonal block at (k, k) (rows already updated) and
// invert it: L_kk -> A's lower block, L_kk^-1 -> linv (NB x NB, zero padded).
// 1024 threads, one per (row t, column c) of the block; the panel solve and
// the block-row solve of the inverse phase then multiply by linv instead of
// substituting row by row.
__global__ void __launch_bounds__(NB * NB, 1) k_potrf_diag(double* A, int n, int k, int nb, int* info, double* linv) {
  // L: the block being reduced (column j is read, columns > j updated in step
  // j); F: the factor, each entry written once -- so one barrier per column:
  // every thread takes the pivot's square root itself, and nothing reads
  // what step j writes until step j + 1
  __shared__ double L[NB][NB + 1], F[NB][NB + 1], X[NB][NB + 1];
  const int c = threadIdx.x % NB, t = threadIdx.x / NB;
  L[t][c] = (t < nb && c <= t) ? A[(long long)(k + t) * n + k + c] : 0.0;
  F[t][c] = 0.0;
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const double d = L[j][j];
    const bool bad = !(d > 0.0);
    const double piv = bad ? 1.0 : sqrt(d);
    const double rinv = 1.0 / piv;
    if (t == j && c == j) {
      F[j][j] = piv;
      if (bad && *info == 0) *info = k + j + 1;
    }
    if (t > j && t < nb) {
      const double lt = L[t][j] * rinv;
      if (c == j) F[t][j] = lt;
      else if (c > j && c <= t) L[t][c] -= lt * (L[c][j] * rinv);
    }
    __syncthreads();
  }
  // X = F^-1 by right-looking substitution: thread (t, c) keeps X[t][c] in a
  // register; step r finalises row r and every lower row subtracts its
  // multiple of it -- one FMA and one barrier per step
  double xv = (t == c) ? 1.0 : 0.0;
  for (int r = 0; r < nb; ++r) {
    if (t == r) {
      xv = xv / F[r][r];
      X[r][c] = xv;
    }
    __syncthreads();
    if (t > r && t < nb) xv = fma(-F[t][r], X[r][c], xv);
  }
  if (t < nb && c <= t) A[(long long)(k + t) * n + k + c] = F[t][c];
  linv[t * NB + c] = (t < nb && c < nb) ? X[t][c] : 0.0;
}

// Rows i >= k+nb: A[i, k:k+nb] <- A[i, k:k+nb] L_kk^-T, i.e.
// X[i][j] = sum_{l <= j} A[i][k+l] linv[j][l].  64 rows per CTA.
__global__ void __launch_bounds__(256) k_trsm_panel(double* A, int n, int k, int nb, const double* linv) {
  __shared__ double P[64][NB + 1], Li[NB][NB + 1];
  const int tid = threadIdx.x;
  const int i0 = k + nb + blockIdx.x * 64;
  for (int e = tid; e < NB * NB; e += 256) Li[e / NB][e % NB] = linv[e];
  for (int e = tid; e < 64 * NB; e += 256) {
    const int r = e / NB, l = e % NB;
    P[r][l] = (i0 + r < n && l < nb) ? A[(long long)(i0 + r) * n + k + l] : 0.0;
  }
  __syncthreads();
  const int c = tid % NB, r0 = tid / NB;
  for (int a = 0; a < 8; ++a) {
    const int r = r0 + 8 * a;
    double v = 0.0;
    for (int l = 0; l <= c; ++l) v = fma(P[r][l], Li[c][l], v);
    if (i0 + r < n && c < nb) A[(long long)(i0 + r) * n + k + c] = v;
  }
}

// The three O(n^3) phases (trailing update, the update of Y = L^-1, Y^T Y)
// run on 64 x 64 output tiles per CTA of 256 threads, each thread holding a
// 4 x 4 register block (rows ty + 16a, columns tx + 16b): per inner index one
// shared-memory load of 4 + 4 values feeds 16 FMAs.
constexpr int TB = 64;

// Trailing update (lower triangle): A[i][j] -= sum_l A[i][k+l] A[j][k+l].
// Grid: one CTA per 64 x 64 tile pair bi >= bj of the trailing matrix.
__global__ void __launch_bounds__(256) k_syrk_update(double* A, int n, int k, int nb) {
  const int t0 = k + nb;
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi) return;
  const int i0 = t0 + bi * TB, j0 = t0 + bj * TB;
  __shared__ double Pi[TB][NB + 1], Pj[TB][NB + 1];
  const int tid = threadIdx.x;
  for (int e = tid; e < TB * NB; e += 256) {
    const int r = e / NB, l = e % NB;
    Pi[r][l] = (i0 + r < n && l < nb) ? A[(long long)(i0 + r) * n + k + l] : 0.0;
    Pj[r][l] = (j0 + r < n && l < nb) ? A[(long long)(j0 + r) * n + k + l] : 0.0;
  }
  __syncthreads();
  const int tx = tid % 16, ty = tid / 16;
  double acc[4][4] = {};
  for (int l = 0; l < nb; ++l) {
    double pi[4], pj[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) pi[a] = Pi[ty + 16 * a][l];
#pragma unroll
    for (int b = 0; b < 4; ++b) pj[b] = Pj[tx + 16 * b][l];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(pi[a], pj[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      if (i < n && j <= i) A[(long long)i * n + j] -= acc[a][b];
    }
}

// Y = L^-1 by recursive doubling over the 32-row block structure (the
// blocked triangular inversion): with both halves of a block pair already
// inverted,
//     [L11 0; L21 L22]^-1 = [Y11 0; -Y22 L21 Y11  Y22],
// so each level is two batched products over all pairs of the level:
// T = L21 Y11, then Y21 = -Y22 T.  8 levels for n = 4,131 (16 launches
// instead of a 130-step substitution whose products had K = 32).
struct GemmJob {
  const double* A; const double* B; double* C;   // C (M x N) = alpha A (M x K) B (K x N), row-major
  int lda, ldb, ldc, M, N, K;
};
constexpr int kMaxJobs = 128;
struct GemmBatch {
  GemmJob job[kMaxJobs];
  int count;
  double alpha;
  int a_lower, b_lower;   // A / B lower triangular (square): skip the zero part of the K range
  // a_bw > 0: A is a block L21 of a band matrix, its row 0 K rows below its
  // column 0, so A[i][k] = 0 for k < i + K - a_bw
  int a_bw;
};

// One 64 x 64 output tile per CTA (blockIdx.x: tile of job blockIdx.y),
// 4 x 4 register blocks, K in chunks of 32 through shared memory.
__global__ void __launch_bounds__(256) k_gemm_batched(const __grid_constant__ GemmBatch bt) {
  const GemmJob& jb = bt.job[blockIdx.y];
  const int tn = (jb.N + TB - 1) / TB, tm = (jb.M + TB - 1) / TB;
  if ((int)blockIdx.x >= tn * tm) return;
  const int i0 = ((int)blockIdx.x / tn) * TB, j0 = ((int)blockIdx.x % tn) * TB;
  int kb = 0, ke = jb.K;
  if (bt.b_lower) kb = j0;                        // B[k][j] = 0 for k < j
  if (bt.a_lower) ke = min(ke, i0 + TB);          // A[i][k] = 0 for k > i
  if (bt.a_bw > 0) kb = max(kb, i0 + jb.K - bt.a_bw);
  constexpr int LC = 32;
  __shared__ double As[TB][LC + 1], Bs[LC][TB + 1];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  double acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += LC) {
    for (int e = tid; e < TB * LC; e += 256) {
      const int r = e / LC, l = e % LC;
      const int gi = i0 + r, gk = k0 + l;
      As[r][l] = (gi < jb.M && gk < ke) ? jb.A[(long long)gi * jb.lda + gk] : 0.0;
      const int lr = e / TB, c = e % TB;
      const int gk2 = k0 + lr, gj = j0 + c;
      Bs[lr][c] = (gk2 < ke && gj < jb.N) ? jb.B[(long long)gk2 * jb.ldb + gj] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int l = 0; l < LC; ++l) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] = As[ty + 16 * q][l];
#pragma unroll
      for (int q = 0; q < 4; ++q) b[q] = Bs[l][tx + 16 * q];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int w = 0; w < 4; ++w) acc[q][w] = fma(a[q], b[w], acc[q][w]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const int i = i0 + ty + 16 * q, j = j0 + tx + 16 * w;
      if (i < jb.M && j < jb.N) jb.C[(long long)i * jb.ldc + j] = bt.alpha * acc[q][w];
    }
}

// Y = 0 with the inverted diagonal blocks L_kk^-1 on the diagonal.
__global__ void k_y_init(double* Y, int n, const double* linv_all) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    double v = 0.0;
    if (i / NB == j / NB) {
      const int k = i / NB;
      v = linv_all[(size_t)k * NB * NB + (i - k * NB) * NB + (j - k * NB)];
    }
    Y[e] = v;
  }
}

// Ainv = Y^T Y (Y lower triangular): Ainv[i][j] = sum_{l >= max(i,j)} Y[l][i] Y[l][j].
// A^-1 = Y^T Y is symmetric: one CTA per 64x64 tile of the lower triangle
// (blockIdx.x enumerates the pairs bi >= bj), written to both triangles.
__global__ void __launch_bounds__(256) k_yty(const double* Y, double* Ainv, int n) {
  int bi = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);
  while ((bi + 1) * (bi + 2) / 2 <= (int)blockIdx.x) ++bi;
  while (bi * (bi + 1) / 2 > (int)blockIdx.x) --bi;
  const int bj = (int)blockIdx.x - bi * (bi + 1) / 2;
  const int i0 = bi * TB, j0 = bj * TB;
  constexpr int LC = 32;   // inner-index chunk
  __shared__ double Yi[LC][TB + 1], Yj[LC][TB + 1];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  double acc[4][4] = {};
  const int lstart = (i0 > j0 ? i0 : j0);
  for (int l0 = lstart; l0 < n; l0 += LC) {
    for (int e = tid; e < LC * TB; e += 256) {
      const int r = e / TB, c = e % TB;
      const int l = l0 + r;
      Yi[r][c] = (l < n && i0 + c < n) ? Y[(long long)l * n + i0 + c] : 0.0;
      Yj[r][c] = (l < n && j0 + c < n) ? Y[(long long)l * n + j0 + c] : 0.0;
    }
    __syncthreads();
    for (int l = 0; l < LC; ++l) {
      double yi[4], yj[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) yi[a] = Yi[l][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) yj[b] = Yj[l][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(yi[a], yj[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      if (i < n && j < n) {
        Ainv[(long long)i * n + j] = acc[a][b];
        Ainv[(long long)j * n + i] = acc[a][b];
      }
    }
}

// Padded-storage vector index of each coarsest DOF (reference node order,
// DOF 3 * node + c): the GEMVs gather b and scatter x through it instead of
// decoding node coordinates in every CTA.
__global__ void k_dense_perm(Grid c, int* __restrict__ perm, int n) {
  const int nx1 = c.lx + 1, ny1 = c.ly + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = i / 3, comp = i - 3 * r;
    const int xx = r % nx1, rr = r / nx1, yy = rr % ny1, zz = rr / ny1;
    perm[i] = 3 * c.idx(xx, yy, zz) + comp;
  }
}

// FP32 copy of the FP64 inverse with rows padded to ld (a multiple of 4)
// floats, the padding zero: every row starts on a 16-byte boundary.
__global__ void k_convert_pad(const double* __restrict__ A, float* __restrict__ B, int n, int ld) {
  const long long total = (long long)n * ld;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / ld), j = (int)(e - (long long)i * ld);
    B[e] = j < n ? (float)A[(long long)i * n + j] : 0.0f;
  }
}

// x = Ainv b on the coarsest level; b gathered into shared memory in FP64,
// products accumulated in FP64 (Ainv in FP64; the FP32 V-cycle reads the
// padded FP32 copy in k_dense_solve_f32).
template <typename T>
__global__ void k_dense_solve(const double* __restrict__ Ainv, int n, const int* __restrict__ perm,
                              const T* __restrict__ b, T* __restrict__ x, const KrylovState* ks) {
  if (ks && ks->done) return;
  extern __shared__ double sb[];
  for (int i = threadIdx.x; i < n; i += blockDim.x) sb[i] = (double)b[__ldg(perm + i)];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int i = blockIdx.x * wpb + warp; i < n; i += gridDim.x * wpb) {
    const double* row = Ainv + (long long)i * n;
    // eight independent partial sums keep eight 256-byte row segments in
    // flight per warp (the GEMV streams n^2 doubles per call)
    double part[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int j = lane;
    for (; j + 7 * 32 < n; j += 8 * 32) {
#pragma unroll
      for (int k = 0; k < 8; ++k) part[k] += __ldg(row + j + 32 * k) * sb[j + 32 * k];
    }
    for (; j < n; j += 32) part[7] += __ldg(row + j) * sb[j];
    double s = ((part[0] + part[1]) + (part[2] + part[3])) + ((part[4] + part[5]) + (part[6] + part[7]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) x[__ldg(perm + i)] = (T)s;
  }
}

// The FP32 V-cycle's coarsest GEMV: rows of ld floats (16-byte aligned,
// zero-padded past n), each lane streaming float4s, eight in flight per lane
// (4 KB per warp: enough bytes in flight to approach the HBM rate with one
// row per warp), products accumulated in FP64.
template <typename T>
__global__ void k_dense_solve_f32(const float* __restrict__ Ainv, int n, int ld, const int* __restrict__ perm,
                                  const T* __restrict__ b, T* __restrict__ x, const KrylovState* ks) {
  if (ks && ks->done) return;
  extern __shared__ double sb[];   // ld values, zero past n
  for (int i = threadIdx.x; i < ld; i += blockDim.x) sb[i] = i < n ? (double)b[__ldg(perm + i)] : 0.0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const int n4 = ld >> 2;
  for (int i = blockIdx.x * wpb + warp; i < n; i += gridDim.x * wpb) {
    const float4* row = reinterpret_cast<const float4*>(Ainv + (long long)i * ld);
    double part[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int j = lane;
    for (; j + 7 * 32 < n4; j += 8 * 32) {
      float4 v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = __ldg(row + j + 32 * k);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const double* bb = sb + 4 * (j + 32 * k);
        part[k] += (double)v[k].x * bb[0] + (double)v[k].y * bb[1] + (double)v[k].z * bb[2] +
                   (double)v[k].w * bb[3];
      }
    }
    for (; j < n4; j += 32) {
      const float4 v = __ldg(row + j);
      const double* bb = sb + 4 * j;
      part[7] += (double)v.x * bb[0] + (double)v.y * bb[1] + (double)v.z * bb[2] + (double)v.w * bb[3];
    }
    double s = ((part[0] + part[1]) + (part[2] + part[3])) + ((part[4] + part[5]) + (part[6] + part[7]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) x[__ldg(perm + i)] = (T)s;
  }
}

}  // namespace

int dense_assemble(const Grid& c, const double* stencil, const uint8_t* cmask, double* A, int n, cudaStream_t st) {
  cudaMemsetAsync(A, 0, sizeof(double) * (size_t)n * n, st);
  const long long work = (long long)(c.lx + 1) * (c.ly + 1) * (c.lz + 1) * 27;
  int blocks = (int)((work + 255) / 256);
  launch_k(k_dense_assemble, blocks, 256, 0, st, c, stencil, cmask, A, n);
  return 0;
}

// Doubles of the work buffer: Y = L^-1 (n x n) and the inverted diagonal
// blocks (NB x NB each).
size_t dense_work_count(int n) {
  return (size_t)n * n + (size_t)((n + NB - 1) / NB) * NB * NB + (size_t)n * n / 2 + (size_t)NB * n;
}

// A (n x n, lower part) is overwritten by L; work (dense_work_count(n))
// receives Y = L^-1 and the inverted diagonal blocks; A <- Y^T Y = A^-1.
// d_info > 0 flags a non-positive pivot.  bw: A[i][j] == 0 for |i - j| > bw
// (a stencil operator in lexicographic node order is banded).  A Cholesky
// factor keeps the band, so the panel solve and the trailing update of block
// column k only touch the rows below it that lie within the band: the rows
// they skip would receive exact zeros (the factor is the same bit for bit).
int dense_cholesky_inverse(double* A, double* work, int n, int bw, int* d_info, cudaStream_t st) {
  cudaMemsetAsync(d_info, 0, sizeof(int), st);
  double* linv_all = work + (size_t)n * n;
  if (bw < 0 || bw > n) bw = n;
  for (int k = 0; k < n; k += NB) {
    const int nb = (n - k < NB) ? (n - k) : NB;
    double* linv = linv_all + (size_t)(k / NB) * NB * NB;
    launch_k(k_potrf_diag, 1, NB * NB, 0, st, A, n, k, nb, d_info, linv);
    // rows > k + nb - 1 + bw of columns k .. k + nb - 1 are zero
    const int rest = std::min(n, k + nb + bw) - (k + nb);
    if (rest > 0) {
      launch_k(k_trsm_panel, (rest + 63) / 64, 256, 0, st, A, n, k, nb, (const double*)linv);
      const int tiles = (rest + TB - 1) / TB;
      launch_k(k_syrk_update, dim3(tiles, tiles), 256, 0, st, A, n, k, nb);
    }
  }
  // Y = L^{-1} into work: diagonal blocks from the factorization, then the
  // off-diagonal blocks level by level (T in the scratch after linv_all)
  launch_k(k_y_init, 148 * 4, 256, 0, st, work, n, (const double*)linv_all);
  double* tbuf = linv_all + (size_t)((n + NB - 1) / NB) * NB * NB;
  const int nbk = (n + NB - 1) / NB;
  for (int g = 1; g < nbk; g *= 2) {
    GemmBatch b1{}, b2{};
    b1.alpha = 1.0; b1.b_lower = 1;     // T = L21 Y11
    b1.a_bw = bw;
    b2.alpha = -1.0; b2.a_lower = 1;    // Y21 = -Y22 T
    int max_tiles = 0;
    size_t toff = 0;
    auto flush = [&]() {
      if (b1.count == 0) return;
      launch_k(k_gemm_batched, dim3(max_tiles, b1.count), 256, 0, st, b1);
      launch_k(k_gemm_batched, dim3(max_tiles, b2.count), 256, 0, st, b2);
      b1.count = b2.count = 0;
      max_tiles = 0;
    };
    for (int p0 = 0; p0 < nbk; p0 += 2 * g) {
      const int r0 = p0 * NB, r1 = std::min((p0 + g) * NB, n), r2 = std::min((p0 + 2 * g) * NB, n);
      if (r1 >= r2) continue;
      const int m = r2 - r1, h = r1 - r0;
      double* T = tbuf + toff;   // distinct per pair within a level (sum of m h <= n^2 / 4)
      toff += (size_t)m * h;
      // L21 = L[r1:r2, r0:r1] is zero below its row bw (the band), and so
      // is T: only its first mb rows are formed, and only they enter Y21
      const int mb = std::min(m, bw);
      b1.job[b1.count++] = GemmJob{A + (size_t)r1 * n + r0, work + (size_t)r0 * n + r0, T, n, n, h, mb, h, h};
      b2.job[b2.count++] = GemmJob{work + (size_t)r1 * n + r1, T, work + (size_t)r1 * n + r0, n, h, n, m, h, mb};
      max_tiles = std::max(max_tiles, ((m + TB - 1) / TB) * ((h + TB - 1) / TB));
      if (b1.count == kMaxJobs) flush();
    }
    flush();
  }
  // A <- Y^T Y (lower-triangle tiles, mirrored)
  const int tiles = (n + TB - 1) / TB;
  launch_k(k_yty, dim3(tiles * (tiles + 1) / 2), 256, 0, st, work, A, n);
  return 0;
}

// b is staged in dynamic shared memory (n doubles, n <= 16384).  The limit is
// a per-function attribute shared by every solver of the process (solvers of
// different sizes run concurrently in batch solves): always the maximum.
void dense_prepare_smem(int n) {
  (void)n;
  const int bytes = (int)sizeof(double) * 16384;
  cudaFuncSetAttribute(k_dense_solve<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_dense_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_dense_solve_f32<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

int dense_ld32(int n) { return (n + 3) / 4 * 4; }

void launch_dense_perm(const Grid& c, int* perm, int n, cudaStream_t st) {
  launch_k(k_dense_perm, (n + 255) / 256, 256, 0, st, c, perm, n);
}

void launch_dense_convert_pad(const double* A, float* B, int n, cudaStream_t st) {
  const int ld = dense_ld32(n);
  const long long total = (long long)n * ld;
  launch_k(k_convert_pad, (int)std::min<long long>((total + 255) / 256, 148LL * 32), 256, 0, st, A, B, n, ld);
}

template <typename T>
void launch_dense_solve(const double* Ainv, int n, const int* perm, const T* b, T* x, const KrylovState* ks,
                        cudaStream_t st) {
  const int blocks = (n + 7) / 8;   // one row per warp: every row's stream in flight at once
  launch_k(k_dense_solve<T>, blocks, 256, sizeof(double) * n, st, Ainv, n, perm, b, x, ks);
}
template void launch_dense_solve<double>(const double*, int, const int*, const double*, double*,
                                         const KrylovState*, cudaStream_t);
template void launch_dense_solve<float>(const double*, int, const int*, const float*, float*,
                                        const KrylovState*, cudaStream_t);

void launch_dense_solve_f32(const float* Ainv32, int n, const int* perm, const float* b, float* x,
                            const KrylovState* ks, cudaStream_t st) {
  const int ld = dense_ld32(n);
  const int blocks = (n + 7) / 8;
  launch_k(k_dense_solve_f32<float>, blocks, 256, sizeof(double) * ld, st, Ainv32, n, ld, perm, b, x, ks);
}

}  // namespace vf
