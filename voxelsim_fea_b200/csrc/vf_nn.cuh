// Convolution kernels of the learned preconditioner stage (vf_nn.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace vf {

// One 3x3x3 "same" convolution over a channels-last BF16 box [Z][Y][X][C].
//   out = act(conv(in, w) + bias + skip),  act = ReLU if relu;
//   then, if gate: out *= (gate > 0)  (the ReLU derivative of a saved activation)
// w: [27][cout][cin] BF16.  out_f32 (optional) replaces the BF16 output.
struct NnConvArgs {
  const void* in;
  const void* w;
  const float* bias;
  const void* skip;
  const void* gate;
  void* out;
  float* out_f32;
  int X, Y, Z;
  int relu;
};

// Supported (cin, cout): (16,16) (16,32) (32,16) (32,32) (32,64) (64,32) (64,64).
int nn_conv_forward(int cin, int cout, const NnConvArgs& a, cudaStream_t st);
// dw[27][cout][cin] (FP32) = sum_v dy[v][co] x[v + off(tap)][ci]; work: per-CTA partials.
int nn_conv_wgrad(int cin, int cout, const void* x, const void* dy, float* dw, float* work, size_t work_bytes, int X,
                  int Y, int Z, int accumulate, cudaStream_t st);
size_t nn_wgrad_work_bytes(int cin, int cout, int X, int Y, int Z);

}  // namespace vf
