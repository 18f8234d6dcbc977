// Fine-level hex8 operator, modal z-marching form with TMA staging (default).
//
// Same arithmetic and tile bookkeeping as vf_modal.cu (a CTA of 32 x 8
// threads marches a 31 x 7 output tile along z; two independent z-ranges are
// packed in float2 for FP32), but every streamed input plane -- the halo plane
// of u, the voxel modulus (and mu), the rhs and the inverse diagonal -- is
// brought into shared memory by one elected thread with cp.async.bulk.tensor
// (one box per array, plane and z-range), completing on a per-stage mbarrier.
// The 4-byte cp.async copies of the first form (about 26 per thread and plane,
// with their address arithmetic and bank conflicts) saturated the
// shared-memory / LSU pipe; the bulk copies take that traffic off the threads.
//
// TMA boxes are rows of the AoS arrays: the x origin is rounded down to a
// 16-byte boundary (the rule for tiled bulk copies) and the box is widened by
// up to 3 elements; threads index from the remainder.  Out-of-range planes
// and columns read zeros (the tensor maps' fill), like the ghost shell.
// Every wait on an mbarrier is bounded (vf_wait.cuh: about 1 s): on expiry
// the CTA stops marching, raises the error flag (the host turns it into a
// status), waits -- again bounded -- for the copies it still has in flight
// and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

#include "vf_common.cuh"
#include "vf_modal.cuh"
#include "vf_reduce.cuh"
#include "vf_wait.cuh"

namespace vf {

namespace {

using namespace modal;

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int NSTAGE = 4;

// widths (elements) of the boxes: u / rhs / diagonal rows cover the 33 nodes
// of the halo tile (3 values each), modulus rows the 32 voxel columns; plus
// the alignment remainder
template <typename T> struct Box;
template <> struct Box<float> { static constexpr int W = 104, WE = 36, A = 4; };
template <> struct Box<double> { static constexpr int W = 100, WE = 34, A = 2; };

constexpr int rup128(int b) { return (b + 127) / 128 * 128; }

template <typename T, bool LAME, int EPI>
struct Layout {
  static constexpr int L = Pack<T>::L;
  static constexpr int U = rup128((TY + 1) * Box<T>::W * (int)sizeof(T));   // one lane
  static constexpr int E = rup128(TY * Box<T>::WE * (int)sizeof(T));
  static constexpr int B = rup128(TY * Box<T>::W * (int)sizeof(T));
  static constexpr int NB = (EPI != EPI_APPLY ? 1 : 0) + (EPI == EPI_SMOOTH ? 1 : 0);
  static constexpr int LANE = U + E * (LAME ? 2 : 1) + B * NB;
  static constexpr int STAGE = LANE * L;
  // bytes the TMA delivers per stage (boxes without the 128-byte padding)
  static constexpr unsigned TXB = (unsigned)(L * ((TY + 1) * Box<T>::W + TY * Box<T>::WE * (LAME ? 2 : 1) +
                                                  TY * Box<T>::W * NB) *
                                             (int)sizeof(T));
  static constexpr int offU = 0, offE = U, offM = U + E, offB = U + E * (LAME ? 2 : 1), offD = offB + B;
  static constexpr size_t total() {
    return 128 + (size_t)NSTAGE * STAGE + sizeof(typename Pack<T>::P) * 3 * 3 * TY * TX + 8 * NSTAGE;
  }
};

__device__ __forceinline__ unsigned su32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(su32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(su32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load3(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(su32(bar))
      : "memory");
}

template <typename T, bool LAME, int EPI>
__global__ void __launch_bounds__(TX * TY, 2)
    k_modal_tma(Grid g, OpArgs a, ModalConst mc, int zchunk, const __grid_constant__ CUtensorMap tm_u,
                const __grid_constant__ CUtensorMap tm_e, const __grid_constant__ CUtensorMap tm_m,
                const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tm_d) {
  using O = Pack<T>;
  using P = typename O::P;
  using Lay = Layout<T, LAME, EPI>;
  constexpr int L = O::L;
  constexpr int W = Box<T>::W, WE = Box<T>::WE, AL = Box<T>::A;
  KrylovState* ks = a.ks;
  if (ks && ks->done) return;

  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  P (*s_c)[3][TY][TX] = reinterpret_cast<P (*)[3][TY][TX]>(smem + NSTAGE * Lay::STAGE);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NSTAGE * Lay::STAGE + sizeof(P) * 3 * 3 * TY * TX);

  T* __restrict__ out = (T*)a.out;
  const uint8_t* __restrict__ mask = a.mask;
  const T w = a.omega_dev ? (T)(*a.omega_dev) : (T)a.omega;
  const T* dprev = (const T*)a.dprev;
  T* dout = (T*)a.dout;
  const T c1 = a.c1_dev ? (T)(*a.c1_dev) : (T)0;

  const int tx = threadIdx.x, ty = threadIdx.y;
  const bool leader = (tx == 0 && ty == 0);
  // Work of this CTA: a range [ub, ue) of (tile, output plane) units, tile-
  // major, NP planes per tile.  zchunk > 0: one tile and z-chunk per CTA
  // (x tiles fastest, then y tiles, then chunks); zchunk <= 0: the units split
  // evenly over the grid (one resident wave), a range crossing into the next
  // tile marched as a second segment.
  const int ntx = (g.lx + TX - 1) / (TX - 1), nty = (g.ly + TY - 1) / (TY - 1);
  const int NP = g.lz + 1;
  long long ub, ue;
  if (zchunk > 0) {
    const int ntile = ntx * nty;
    const int tile = (int)(blockIdx.x % ntile), ch = (int)(blockIdx.x / ntile);
    ub = (long long)tile * NP + (long long)ch * zchunk;
    ue = (long long)tile * NP + min((long long)(ch + 1) * zchunk, (long long)NP);
  } else {
    const long long U = (long long)ntx * nty * NP;
    ub = U * blockIdx.x / gridDim.x;
    ue = U * (blockIdx.x + 1) / gridDim.x;
  }
  const int sz = g.px * g.py;
  // per-segment geometry (set at the top of each segment)
  int X0 = 0, Y0 = 0, Xc = 0, Yc = 0, colbase = 0, xu = 0, ou = 0, xe = 0, oe = 0, nsteps = 0, gbase = 0;
  int issued_hi = -1;   // leader: running index of the last step whose copies were issued
  bool out_col = false;
  int z0[L], oend[L];

  if (leader) {
#pragma unroll
    for (int k = 0; k < NSTAGE; ++k) mbar_init(&bar[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  // stages and mbarrier phases follow the CTA's running step count gbase + s
  auto issue = [&](int s) {   // leader only
    const int st = (gbase + s) % NSTAGE;
    unsigned char* base = smem + st * Lay::STAGE;
    issued_hi = gbase + s;
    mbar_expect_tx(&bar[st], Lay::TXB);
#pragma unroll
    for (int l = 0; l < L; ++l) {
      unsigned char* lb = base + l * Lay::LANE;
      const int plane = z0[l] + 1 + s;   // storage plane (beyond pz: zero fill)
      tma_load3(lb + Lay::offU, &tm_u, &bar[st], xu, Y0, plane);
      tma_load3(lb + Lay::offE, &tm_e, &bar[st], xe, Y0, plane);
      if (LAME) tma_load3(lb + Lay::offM, &tm_m, &bar[st], xe, Y0, plane);
      if (EPI != EPI_APPLY) tma_load3(lb + Lay::offB, &tm_b, &bar[st], xu, Y0, plane);
      if (EPI == EPI_SMOOTH) tma_load3(lb + Lay::offD, &tm_d, &bar[st], xu, Y0, plane);
    }
  };
  // element accessors of stage st, lane l
  auto uval = [&](int st, int l, int c, int j, int i) -> T {
    const T* r = reinterpret_cast<const T*>(smem + st * Lay::STAGE + l * Lay::LANE + Lay::offU);
    return r[j * W + ou + 3 * i + c];
  };
  auto bval = [&](int st, int l, int off, int c) -> T {
    const T* r = reinterpret_cast<const T*>(smem + st * Lay::STAGE + l * Lay::LANE + off);
    return r[ty * W + ou + 3 * tx + c];
  };
  auto eval_ = [&](int st, int l, int off) -> T {
    const T* r = reinterpret_cast<const T*>(smem + st * Lay::STAGE + l * Lay::LANE + off);
    return r[ty * WE + oe + tx];
  };
  auto pk = [&](auto f) -> P {
    if constexpr (L == 2) return make_float2(f(0), f(1));
    else return f(0);
  };

  P hiPrev[3][4];
  double dot = 0.0;
  uint8_t mk_next[L];

  // false: this step's copies did not arrive in time (every thread agrees)
  auto step = [&](const int s, P (&Fc)[3][4], const P (&Fp)[3][4]) -> bool {
    const int gs = gbase + s;
    const int st = gs % NSTAGE, sp = (gs + NSTAGE - 1) % NSTAGE;
    const bool arrived = mbar_wait_bounded(&bar[st], (unsigned)((gs / NSTAGE) & 1));
    // the barrier also marks step s-1 done everywhere: stage (s+2) is free
    if (__syncthreads_or(!arrived)) return false;
    if (leader && s + 2 < nsteps) issue(s + 2);
    // free-mask bytes: this step's were loaded one step ahead (mk_next),
    // the next step's are requested now, far from their use
    uint8_t mk[L];
#pragma unroll
    for (int l = 0; l < L; ++l) {
      mk[l] = mk_next[l];
      const int zs = z0[l] + s;   // output plane of step s + 1
      mk_next[l] = (s + 1 >= 2 && s + 1 < nsteps && out_col && zs < oend[l]) ? __ldg(mask + (zs + 1) * sz + colbase)
                                                                             : (uint8_t)0;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const P u00 = pk([&](int l) { return uval(st, l, c, ty, tx); });
      const P u10 = pk([&](int l) { return uval(st, l, c, ty, tx + 1); });
      const P u01 = pk([&](int l) { return uval(st, l, c, ty + 1, tx); });
      const P u11 = pk([&](int l) { return uval(st, l, c, ty + 1, tx + 1); });
      const P e0 = O::add(u10, u00), e1 = O::sub(u10, u00);
      const P e2 = O::add(u11, u01), e3 = O::sub(u11, u01);
      Fc[c][0] = O::add(e0, e2);
      Fc[c][1] = O::add(e1, e3);
      Fc[c][2] = O::sub(e2, e0);
      Fc[c][3] = O::sub(e3, e1);
    }
    if (s >= 1) {
      P A[3][8];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          A[c][m] = O::add(Fp[c][m], Fc[c][m]);
          A[c][m + 4] = O::sub(Fc[c][m], Fp[c][m]);
        }
      const P El = pk([&](int l) { return eval_(sp, l, Lay::offE); });
      const P Em = LAME ? pk([&](int l) { return eval_(sp, l, Lay::offM); }) : El;
      P B[3][8];
      modal_physics<O, P, T>(A, B, El, Em, mc);
      P acc[3][4];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc[c][0] = O::sub(hiPrev[c][0], B[c][4]);
        const P hi0 = B[c][4];
#pragma unroll
        for (int m = 1; m < 4; ++m) {
          acc[c][m] = O::add(hiPrev[c][m], O::sub(B[c][m], B[c][m + 4]));
          hiPrev[c][m] = O::add(B[c][m], B[c][m + 4]);
        }
        hiPrev[c][0] = hi0;
      }
      P c00[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const P t0 = O::sub(acc[c][0], acc[c][2]), t1 = O::sub(acc[c][1], acc[c][3]);
        const P t2 = O::add(acc[c][0], acc[c][2]), t3 = O::add(acc[c][1], acc[c][3]);
        c00[c] = O::sub(t0, t1);
        s_c[0][c][ty][tx] = O::add(t0, t1);
        s_c[1][c][ty][tx] = O::sub(t2, t3);
        s_c[2][c][ty][tx] = O::add(t2, t3);
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
                const T u0 = uval(sp, l, 0, ty, tx), u1 = uval(sp, l, 1, ty, tx), u2 = uval(sp, l, 2, ty, tx);
                dot += (double)u0 * (double)k0 + (double)u1 * (double)k1 + (double)u2 * (double)k2;
              }
            } else {
              const T b0 = bval(sp, l, Lay::offB, 0), b1 = bval(sp, l, Lay::offB, 1), b2 = bval(sp, l, Lay::offB, 2);
              if (EPI == EPI_SMOOTH) {
                const T u0 = uval(sp, l, 0, ty, tx), u1 = uval(sp, l, 1, ty, tx), u2 = uval(sp, l, 2, ty, tx);
                const T d0 = bval(sp, l, Lay::offD, 0), d1 = bval(sp, l, Lay::offD, 1);
                const T d2 = bval(sp, l, Lay::offD, 2);
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
    return true;
  };

  P Fa[3][4], Fb[3][4];
  int failed_at = -1;   // running index of the step whose copies did not arrive
  // Segments: a new segment's first two loads go to the stages of steps
  // gbase-4 and gbase-3, whose last readers (steps gbase-3 and gbase-2) every
  // thread has left once the leader is past step gbase-1's first barrier.
#pragma unroll 1
  for (long long u0 = ub; u0 < ue;) {
    const int tile = (int)(u0 / NP);
    const int zb = (int)(u0 - (long long)tile * NP);
    const int ze = (int)min((long long)NP, (long long)zb + (ue - u0));
    u0 = (long long)tile * NP + ze;
    X0 = (tile % ntx) * (TX - 1);
    Y0 = (tile / ntx) * (TY - 1);
    Xc = X0 - 1 + tx;
    Yc = Y0 - 1 + ty;
    const bool col_in = (Xc + 1 < g.px) && (Yc + 1 < g.py);
    colbase = col_in ? (Yc + 1) * g.px + (Xc + 1) : 0;
    out_col = tx >= 1 && ty >= 1 && Xc <= g.lx && Yc <= g.ly;
    // box origins (storage coordinates; x rounded down to 16 bytes) and remainders
    xu = (3 * X0) & ~(AL - 1);
    ou = 3 * X0 - xu;
    xe = X0 & ~(AL - 1);
    oe = X0 - xe;
    const int H = (ze - zb + L - 1) / L;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      z0[l] = zb + l * H - 1;
      oend[l] = min(min(zb + l * H + H, ze), g.lz + 1);
    }
    nsteps = H + 2;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int m = 0; m < 4; ++m) { hiPrev[c][m] = O::zero(); Fa[c][m] = O::zero(); Fb[c][m] = O::zero(); }
    if (leader) {
      issue(0);
      issue(1);
    }
#pragma unroll
    for (int l = 0; l < L; ++l) mk_next[l] = 0;   // steps 0 and 1 write no output
#pragma unroll 1
    for (int s = 0; s < nsteps; ++s) {
      if (!step(s, Fa, Fb)) {
        failed_at = gbase + s;
        break;
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int m = 0; m < 4; ++m) Fb[c][m] = Fa[c][m];
    }
    if (failed_at >= 0) break;
    gbase += nsteps;
  }
  if (failed_at >= 0) {
    // expired wait: flag it, then let the copies still in flight (steps
    // failed_at .. issued_hi, at most three) land before the CTA exits --
    // each wait bounded like the first
    if (leader) {
      if (a.err) atomicExch(a.err, 1);
      for (int k = failed_at; k <= issued_hi; ++k) mbar_wait_bounded(&bar[k % NSTAGE], (unsigned)((k / NSTAGE) & 1));
    }
    __syncthreads();
  }
  // APPLY: u.y (p.Ap); SMOOTH: b.u' (the V-cycle's last sweep: r.z)
  if ((EPI == EPI_APPLY || EPI == EPI_SMOOTH) && a.dot_partials && ks)
    reduce_and_finalize(dot, a.dot_partials, ks, a.dot_slot, nullptr);
}

// ---- tensor maps ----------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_tm_mu;
std::map<std::tuple<const void*, int, int, int, int, int>, CUtensorMap> g_tm_cache;

bool encode_fn() {
  if (g_encode) return true;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn)
    return false;
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return true;
}

// kind 0: AoS node vector, box rows TY+1 (u); 1: AoS node vector, box rows TY
// (rhs, diagonal); 2: per-voxel scalar, box rows TY (modulus, mu)
template <typename T>
bool tensor_map(const void* ptr, const Grid& g, int kind, CUtensorMap* out) {
  if (!ptr || (reinterpret_cast<uintptr_t>(ptr) & 15)) return false;
  const auto key = std::make_tuple(ptr, kind, g.px, g.py, g.pz, (int)sizeof(T));
  std::lock_guard<std::mutex> lk(g_tm_mu);
  auto it = g_tm_cache.find(key);
  if (it != g_tm_cache.end()) { *out = it->second; return true; }
  if (!encode_fn()) return false;
  const int per = (kind == 2) ? 1 : 3;
  const cuuint64_t dims[3] = {(cuuint64_t)per * g.px, (cuuint64_t)g.py, (cuuint64_t)g.pz};
  const cuuint64_t strides[2] = {(cuuint64_t)per * g.px * sizeof(T), (cuuint64_t)per * g.px * g.py * sizeof(T)};
  if ((strides[0] & 15) || (strides[1] & 15)) return false;
  const cuuint32_t box[3] = {(cuuint32_t)(kind == 2 ? Box<T>::WE : Box<T>::W), (cuuint32_t)(kind == 0 ? TY + 1 : TY), 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  CUtensorMap m;
  const CUresult r = g_encode(&m, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                              3, const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  g_tm_cache[key] = m;
  *out = m;
  return true;
}

}  // namespace

bool modal_tma_supported() { return encode_fn(); }

// Launch geometry: zchunk > 0 (0: the whole column): one CTA per 31 x 7 tile
// and z-chunk, ceil((lx+1)/31) * ceil((ly+1)/7) * ceil((lz+1)/zchunk) CTAs;
// zchunk < 0: one resident wave (SMs x CTAs per SM, at most one per unit)
// sharing the (tile, plane) units evenly.
// Returns false (nothing launched) when a tensor map cannot be built.
template <typename T>
bool launch_modal_tma(const Grid& g, int epi, const OpArgs& a, const ModalConst& mc, int zchunk, cudaStream_t st) {
  const bool lame = a.mu != nullptr;
  if (zchunk == 0) zchunk = g.lz + 1;
  CUtensorMap mu, me, mm, mb, md;
  if (!tensor_map<T>(a.u, g, 0, &mu) || !tensor_map<T>(a.E, g, 2, &me)) return false;
  mm = me;
  mb = mu;
  md = mu;
  if (lame && !tensor_map<T>(a.mu, g, 2, &mm)) return false;
  if (epi != EPI_APPLY && !tensor_map<T>(a.b, g, 1, &mb)) return false;
  if (epi == EPI_SMOOTH && !tensor_map<T>(a.minv, g, 1, &md)) return false;
  const long long tiles = (long long)((g.lx + TX - 1) / (TX - 1)) * ((g.ly + TY - 1) / (TY - 1));
  const long long units = tiles * (g.lz + 1);
  const dim3 block(TX, TY);
#define VF_TMA_ONE(LM, EP)                                                                    \
  do {                                                                                        \
    auto kern = k_modal_tma<T, LM, EP>;                                                       \
    constexpr size_t smem = Layout<T, LM, EP>::total();                                       \
    static std::atomic<int> per_dev[kMaxDevices];                                             \
    const int per_sm = kernel_prepare(per_dev, kern, smem, TX * TY);                          \
    long long nb;                                                                             \
    if (zchunk > 0) {                                                                         \
      nb = tiles * ((g.lz + 1 + zchunk - 1) / zchunk);                                        \
    } else {                                                                                  \
      int dev = 0, sms = 148;                                                                 \
      cudaGetDevice(&dev);                                                                    \
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);                      \
      nb = std::min<long long>((long long)sms * per_sm, units);                               \
    }                                                                                         \
    launch_k(kern, dim3((unsigned)nb), block, smem, st, g, a, mc, zchunk, mu, me, mm, mb, md); \
  } while (0)
  if (lame) {
    if (epi == EPI_APPLY) VF_TMA_ONE(true, EPI_APPLY);
    else if (epi == EPI_SMOOTH) VF_TMA_ONE(true, EPI_SMOOTH);
    else VF_TMA_ONE(true, EPI_RESID);
  } else {
    if (epi == EPI_APPLY) VF_TMA_ONE(false, EPI_APPLY);
    else if (epi == EPI_SMOOTH) VF_TMA_ONE(false, EPI_SMOOTH);
    else VF_TMA_ONE(false, EPI_RESID);
  }
#undef VF_TMA_ONE
  return true;
}

template bool launch_modal_tma<float>(const Grid&, int, const OpArgs&, const ModalConst&, int, cudaStream_t);
template bool launch_modal_tma<double>(const Grid&, int, const OpArgs&, const ModalConst&, int, cudaStream_t);

}  // namespace vf
