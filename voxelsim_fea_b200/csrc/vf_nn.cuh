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
  const int* skip_flag = nullptr;   // device flag: the launch is a no-op while *skip_flag != 0
  int* err = nullptr;               // device flag raised when a bounded wait of the kernel expires
};

// Supported (cin, cout): (16,16) (16,32) (32,16) (32,32) (32,64) (64,32) (64,64).
int nn_conv_forward(int cin, int cout, const NnConvArgs& a, cudaStream_t st);
// dw[27][cout][cin] (FP32) = sum_v dy[v][co] x[v + off(tap)][ci]; work: per-CTA partials.
int nn_conv_wgrad(int cin, int cout, const void* x, const void* dy, float* dw, float* work, size_t work_bytes, int X,
                  int Y, int Z, int accumulate, cudaStream_t st);
size_t nn_wgrad_work_bytes(int cin, int cout, int X, int Y, int Z);

// ---- U-Net inference stage (vf_learned.cu) ----
struct Grid;
struct NnStage;
long long nn_param_count();
NnStage* nn_create(const Grid& gL, int level, cudaStream_t st, cudaError_t* err);
void nn_destroy(NnStage* s);
void nn_dims(const NnStage* s, int* xyz);
cudaError_t nn_set_weights(NnStage* s, const float* host, cudaStream_t st);
bool nn_has_weights(const NnStage* s);
// static features from the fine modulus (padded voxel layout of g0); eref_dev: device max modulus
void nn_set_features(NnStage* s, const Grid& g0, const double* E0, const double* eref_dev, cudaStream_t st);
template <typename T> void nn_make_input(NnStage* s, const Grid& gL, const T* r, const int* skip, cudaStream_t st);
void nn_forward(NnStage* s, const int* skip, cudaStream_t st);
void nn_set_error_flag(NnStage* s, int* err);
template <typename T> void nn_make_output(NnStage* s, const Grid& gL, const uint8_t* maskL, T* e, const int* skip,
                                          cudaStream_t st);
const void* nn_input_buffer(const NnStage* s);
const float* nn_scale_buffer(const NnStage* s);
void launch_max_f64(const double* v, long long n, double* out, cudaStream_t st);

}  // namespace vf
