// Deterministic FP64 reductions with a last-block-done finalize, and the
// scalar logic of the PCG recurrences that runs on the device so that no
// host round-trip is needed inside an iteration (the reference blocks on a
// float() per dot: core/multigrid.py:471, 499, 516, 533).
//
// Every reduction kernel runs a FIXED grid over a grid-stride loop; each CTA
// writes one partial, and the last CTA to finish sums the partials in index
// order.  The result therefore depends only on the problem size, never on
// scheduling: two runs are bitwise identical.
#pragma once

#include "vf_common.cuh"

namespace vf {

// Reduction slots: what the finalize does with the sum.
enum RedSlot {
  SLOT_PAP = 0,      // p.Ap      -> alpha (or stop on pAp == 0, multigrid.py:500-511)
  SLOT_RR = 1,       // r.r       -> ratio, history, tol / stall / max_it (multigrid.py:516-531)
  SLOT_RZ = 2,       // r.z       -> beta or restart (multigrid.py:533-546)
  SLOT_RZ_INIT = 3,  // r.z before the loop (multigrid.py:476)
  SLOT_FNORM = 4,    // ||f||^2   -> fnorm (multigrid.py:471)
  SLOT_OUTER = 5,    // ||r64||^2 -> outer (refinement) residual
  SLOT_PLAIN = 6,    // sum stored in ks->rr only
  SLOT_FCG = 7,      // (r.z, z.Ap) -> flexible-CG beta = -z.Ap / p.Ap (Notay's FCG(1))
  SLOT_GNUM = 8,     // c.r1  -> learned-stage step numerator
  SLOT_GDEN = 9      // c.Ac  -> learned-stage step denominator
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Linear thread / block indices (kernels may use 2-D blocks and 3-D grids).
__device__ __forceinline__ int lin_tid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
__device__ __forceinline__ int lin_nthreads() { return blockDim.x * blockDim.y * blockDim.z; }
__device__ __forceinline__ unsigned lin_bid() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ __forceinline__ unsigned lin_nblocks() { return gridDim.x * gridDim.y * gridDim.z; }

// Block-wide sum in a fixed order; valid in thread 0.  <= 1024 threads, whole warps.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s_warp[32];
  v = warp_sum(v);
  const int t0 = lin_tid();
  const int lane = t0 & 31, w = t0 >> 5;
  __syncthreads();
  if (lane == 0) s_warp[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = (lane < ((lin_nthreads() + 31) >> 5)) ? s_warp[lane] : 0.0;
    t = warp_sum(t);
  }
  return t;
}

__device__ inline void finalize_slot(KrylovState* ks, int slot, double total, double* hist) {
  switch (slot) {
    case SLOT_PAP: {
      ks->pAp = total;
      if (!(total == total) || total == INFINITY || total == -INFINITY) {
        ks->done = 1; ks->status = KS_NONFINITE;
      } else if (total == 0.0) {
        ks->done = 1;
        ks->status = (ks->resid < ks->tol) ? KS_CONVERGED : KS_BREAKDOWN;
      } else {
        ks->alpha = ks->rz / total;
      }
      break;
    }
    case SLOT_RR: {
      ks->rr = total;
      const int it = ks->it + 1;
      ks->it = it;
      const double ratio = sqrt(total) / ks->fnorm;
      ks->resid = ratio;
      if (hist) hist[ks->it_base + it - 1] = ratio * ks->hist_scale;
      if (!(ratio == ratio)) { ks->done = 1; ks->status = KS_NONFINITE; break; }
      if (ratio < ks->tol) { ks->done = 1; ks->status = KS_CONVERGED; break; }
      if (ratio < ks->best) ks->best = ratio;
      if (ks->stall_guard && it >= 10 && ratio > 5.0 * ks->best) {
        ks->done = 1; ks->status = KS_STALLED; break;
      }
      if (total < ks->rr_trigger) { ks->done = 1; ks->status = KS_RELIABLE; break; }
      if (ks->it_trigger > 0 && it >= ks->it_trigger) { ks->done = 1; ks->status = KS_RELIABLE; break; }
      if (it >= ks->max_it) { ks->done = 1; ks->status = KS_MAXIT; }
      break;
    }
    case SLOT_RZ: {
      ks->rz_new = total;
      if (ks->rz == 0.0) { ks->restart = 1; ks->beta = 0.0; }
      else { ks->restart = 0; ks->beta = total / ks->rz; }
      ks->rz = total;
      break;
    }
    case SLOT_RZ_INIT: ks->rz = total; ks->restart = 0; break;
    case SLOT_FNORM: ks->fnorm = sqrt(total); break;
    case SLOT_OUTER: ks->rr = total; ks->resid = sqrt(total) / ks->fnorm; break;
    case SLOT_GNUM: ks->gnum = total; break;
    case SLOT_GDEN: ks->gden = total; break;
    default: ks->rr = total; break;
  }
}

// Two sums in one pass (partials hold 2 doubles per CTA); the last CTA finalizes
// both together.  Used by the flexible-CG beta.
__device__ inline void reduce2_and_finalize(double a, double b, double* partials, KrylovState* ks, int slot) {
  __shared__ bool s_last2;
  const double sa = block_sum(a);
  const double sb = block_sum(b);
  const int tid = lin_tid();
  const unsigned nb = lin_nblocks();
  if (tid == 0) {
    partials[2 * lin_bid()] = sa;
    partials[2 * lin_bid() + 1] = sb;
    __threadfence();
    unsigned int prev = atomicAdd(&ks->counter[slot], 1u);
    s_last2 = (prev == nb - 1);
  }
  __syncthreads();
  if (!s_last2) return;
  __threadfence();
  double ta = 0.0, tb = 0.0;
  for (int i = tid; i < (int)nb; i += lin_nthreads()) {
    ta += ((volatile double*)partials)[2 * i];
    tb += ((volatile double*)partials)[2 * i + 1];
  }
  ta = block_sum(ta);
  tb = block_sum(tb);
  if (tid == 0) {
    // FCG(1): p_new = z - (z.Ap / p.Ap) p; alpha next = (r.z) / (p_new.Ap_new)
    ks->rz_new = ta;
    ks->zap = tb;
    if (ks->pAp != 0.0) { ks->restart = 0; ks->beta = -tb / ks->pAp; }
    else { ks->restart = 1; ks->beta = 0.0; }
    ks->rz = ta;
    ks->counter[slot] = 0u;
    __threadfence();
  }
}

// Called by every thread of every CTA with its own partial `v`.  The CTA sum
// goes to partials[linear block id]; the last CTA finalizes.
__device__ inline void reduce_and_finalize(double v, double* partials, KrylovState* ks, int slot,
                                           double* hist) {
  __shared__ bool s_last;
  double bsum = block_sum(v);
  const int tid = lin_tid();
  const unsigned nb = lin_nblocks();
  if (tid == 0) {
    partials[lin_bid()] = bsum;
    __threadfence();
    unsigned int prev = atomicAdd(&ks->counter[slot], 1u);
    s_last = (prev == nb - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double t = 0.0;
  for (int i = tid; i < (int)nb; i += lin_nthreads()) t += ((volatile double*)partials)[i];
  t = block_sum(t);
  if (tid == 0) {
    finalize_slot(ks, slot, t, hist);
    ks->counter[slot] = 0u;
    __threadfence();
  }
}

}  // namespace vf
