"""3x3x3 "same" convolution on channels-last BF16 boxes through libvoxfea.

Layout: activations are (Z, Y, X, C) BF16 CUDA tensors, C in {16, 32, 64};
weights (27, Cout, Cin) FP32 masters, cast to BF16 for the kernel, with
tap = (dz+1)*9 + (dy+1)*3 + (dx+1) -- the cross-correlation of
``torch.nn.functional.conv3d`` (weight[co, ci, kz, ky, kx] == W[tap, co, ci]).
"""

import ctypes

import torch

from .. import _lib

PAIRS = {(16, 16), (16, 32), (32, 16), (32, 32), (32, 64), (64, 32), (64, 64)}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(rc, what):
    if rc != _lib.VF_OK:
        raise RuntimeError(f"{what} failed: {_lib.load().vf_status_string(rc).decode()}")


def conv3d_forward(x, w_bf16, bias=None, skip=None, relu=False, out_f32=False):
    """y = relu?(conv(x, w) + bias + skip); x (Z,Y,X,Cin) BF16, w (27,Cout,Cin) BF16."""
    Z, Y, X, cin = x.shape
    cout = w_bf16.shape[1]
    if (cin, cout) not in PAIRS:
        raise ValueError(f"unsupported channel pair {(cin, cout)}")
    assert x.is_contiguous() and w_bf16.is_contiguous() and x.dtype == torch.bfloat16
    if out_f32:
        y = torch.empty((Z, Y, X, cout), device=x.device, dtype=torch.float32)
        yb, yf = None, y
    else:
        y = torch.empty((Z, Y, X, cout), device=x.device, dtype=torch.bfloat16)
        yb, yf = y, None
    b = None if bias is None else bias.float().contiguous()
    rc = _lib.load().vf_nn_conv3d_forward(_ptr(x), _ptr(w_bf16), _ptr(b), _ptr(skip), int(bool(relu)), _ptr(yb),
                                          _ptr(yf), X, Y, Z, cin, cout, _stream())
    _check(rc, "vf_nn_conv3d_forward")
    return y


def mirror_transpose(w):
    """(27, Cout, Cin) -> (27, Cin, Cout) with the taps mirrored: the weights of
    the data-gradient convolution."""
    return w.flip(0).transpose(1, 2).contiguous()


def conv3d_backward_data(dy, w_bf16, gate=None):
    Z, Y, X, cout = dy.shape
    cin = w_bf16.shape[2]
    dx = torch.empty((Z, Y, X, cin), device=dy.device, dtype=torch.bfloat16)
    wt = mirror_transpose(w_bf16)
    rc = _lib.load().vf_nn_conv3d_backward_data(_ptr(dy.contiguous()), _ptr(wt), _ptr(gate), _ptr(dx), X, Y, Z,
                                                cin, cout, _stream())
    _check(rc, "vf_nn_conv3d_backward_data")
    return dx


def conv3d_backward_weight(x, dy):
    Z, Y, X, cin = x.shape
    cout = dy.shape[3]
    L = _lib.load()
    nbytes = L.vf_nn_wgrad_workspace(cin, cout, X, Y, Z)
    work = torch.empty(nbytes // 4, device=x.device, dtype=torch.float32)
    dw = torch.empty((27, cout, cin), device=x.device, dtype=torch.float32)
    rc = L.vf_nn_conv3d_backward_weight(_ptr(x), _ptr(dy.contiguous()), _ptr(dw), 0, _ptr(work), nbytes, X, Y, Z,
                                        cin, cout, _stream())
    _check(rc, "vf_nn_conv3d_backward_weight")
    return dw


class Conv3dFn(torch.autograd.Function):
    """y = conv(x, w) + b with the libvoxfea kernels in both directions
    (BF16 output, or FP32 with ``out_f32``)."""

    @staticmethod
    def forward(ctx, x, w, b, out_f32=False):
        wb = w.to(torch.bfloat16).contiguous()
        ctx.save_for_backward(x, wb)
        return conv3d_forward(x.contiguous(), wb, bias=b, out_f32=out_f32)

    @staticmethod
    def backward(ctx, dy):
        x, wb = ctx.saved_tensors
        dy = dy.to(torch.bfloat16).contiguous()
        dx = conv3d_backward_data(dy, wb) if ctx.needs_input_grad[0] else None
        dw = conv3d_backward_weight(x, dy) if ctx.needs_input_grad[1] else None
        db = dy.float().sum(dim=(0, 1, 2)) if ctx.needs_input_grad[2] else None
        return dx, dw, db, None


def conv3d(x, w, b, out_f32=False):
    return Conv3dFn.apply(x, w, b, out_f32)
