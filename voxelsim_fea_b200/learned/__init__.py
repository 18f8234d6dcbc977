"""Learned preconditioner stage: a 3-level 3-D U-Net (16/32/64 channels,
3x3x3 BF16 convolutions with FP32 accumulation) that maps a residual plus the
occupancy / log-modulus fields to a displacement correction, used as a stage
of the flexible-CG preconditioner.

The convolutions -- forward, data gradient and weight gradient -- are this
package's own tensor-core kernels (libvoxfea, vf_nn.cu); PyTorch holds the
buffers and runs the glue (pooling, upsampling, ReLU, optimizer) during
training.  Inference inside the solver runs entirely in libvoxfea.
"""
