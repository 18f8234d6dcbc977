"""The BF16 tensor-core convolutions of the learned stage against a CPU FP64
oracle (torch.nn.functional.conv3d in float64 on the same BF16-rounded
operands): forward with every epilogue, data gradient, weight gradient, for
every channel pair the U-Net uses, on a box with partial tiles in x, y and z."""

import numpy as np
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu

PAIRS = [(16, 16), (16, 32), (32, 16), (32, 32), (32, 64), (64, 32), (64, 64)]
SHAPE = (5, 11, 21)    # Z, Y, X: 16x8x2 tiles cut in every axis


def _to_ncdhw(t):       # (Z,Y,X,C) -> (1,C,Z,Y,X), float64 on the CPU
    return t.detach().cpu().double().permute(3, 0, 1, 2).unsqueeze(0)


def _from_ncdhw(t):
    return t.squeeze(0).permute(1, 2, 3, 0)


def _w_torch(w):        # (27,Cout,Cin) -> (Cout,Cin,3,3,3)
    co, ci = w.shape[1], w.shape[2]
    return w.detach().cpu().double().view(3, 3, 3, co, ci).permute(3, 4, 0, 1, 2)


def _rel(a, b):
    a = a.detach().cpu().double()
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("cin,cout", PAIRS)
def test_conv_forward_and_gradients(gpu, cin, cout):
    from voxelsim_fea_b200.learned import conv
    torch.manual_seed(cin * 100 + cout)
    dev = "cuda"
    x = torch.randn(*SHAPE, cin, device=dev).to(torch.bfloat16)
    w = (torch.randn(27, cout, cin, device=dev) / (27 * cin) ** 0.5).to(torch.bfloat16)
    b = torch.randn(cout, device=dev)
    g = torch.randn(*SHAPE, cout, device=dev).to(torch.bfloat16)

    xr = _to_ncdhw(x).requires_grad_(True)
    wr = _w_torch(w).requires_grad_(True)
    yr = F.conv3d(xr, wr, b.cpu().double(), padding=1)
    yr.backward(_to_ncdhw(g))
    y_ref = _from_ncdhw(yr.detach())

    y32 = conv.conv3d_forward(x, w, bias=b, out_f32=True)
    assert _rel(y32, y_ref) < 1e-5                        # FP32 accumulation
    y16 = conv.conv3d_forward(x, w, bias=b)
    assert _rel(y16, y_ref) < 8e-3                        # + one BF16 rounding

    dx = conv.conv3d_backward_data(g, w)
    assert _rel(dx, _from_ncdhw(xr.grad)) < 8e-3
    dw = conv.conv3d_backward_weight(x, g)
    dw_ref = wr.grad.permute(2, 3, 4, 0, 1).reshape(27, cout, cin)
    assert _rel(dw, dw_ref) < 1e-5


@pytest.mark.parametrize("form", ["column", "plane"])
@pytest.mark.parametrize("cin,cout", PAIRS)
def test_conv_forward_z_columns(gpu, monkeypatch, cin, cout, form):
    """Both forward forms (VOXFEA_CONV_FORM: one output plane per CTA, or a
    column of 8 planes marched with the taps resident -- on its own only on
    boxes large enough to fill the GPU with columns) over 19 planes = two
    full columns and one of 3, with the epilogue's skip input and ReLU."""
    from voxelsim_fea_b200.learned import conv
    monkeypatch.setenv("VOXFEA_CONV_FORM", form)
    torch.manual_seed(cin * 7 + cout)
    shape = (19, 13, 10)
    x = torch.randn(*shape, cin, device="cuda").to(torch.bfloat16)
    w = (torch.randn(27, cout, cin, device="cuda") / (27 * cin) ** 0.5).to(torch.bfloat16)
    b = torch.randn(cout, device="cuda")
    skip = torch.randn(*shape, cout, device="cuda").to(torch.bfloat16)
    y = conv.conv3d_forward(x, w, bias=b, skip=skip, relu=True, out_f32=True)
    ref = torch.relu(_from_ncdhw(F.conv3d(_to_ncdhw(x), _w_torch(w), b.cpu().double(), padding=1))
                     + skip.cpu().double())
    assert _rel(y, ref) < 1e-5


def test_conv_epilogues(gpu):
    """bias + skip + ReLU in the forward epilogue; the ReLU gate in backward."""
    from voxelsim_fea_b200.learned import conv
    torch.manual_seed(3)
    x = torch.randn(*SHAPE, 32, device="cuda").to(torch.bfloat16)
    w = (torch.randn(27, 16, 32, device="cuda") / 30).to(torch.bfloat16)
    b = torch.randn(16, device="cuda")
    skip = torch.randn(*SHAPE, 16, device="cuda").to(torch.bfloat16)
    y = conv.conv3d_forward(x, w, bias=b, skip=skip, relu=True, out_f32=True)
    ref = torch.relu(_from_ncdhw(F.conv3d(_to_ncdhw(x), _w_torch(w), b.cpu().double(), padding=1))
                     + skip.cpu().double())
    assert _rel(y, ref) < 1e-5
    g = torch.randn(*SHAPE, 16, device="cuda").to(torch.bfloat16)
    gate = torch.relu(torch.randn(*SHAPE, 32, device="cuda")).to(torch.bfloat16)
    dx = conv.conv3d_backward_data(g, w, gate=gate)
    dx_ref = conv.conv3d_backward_data(g, w).double() * (gate > 0).double()
    assert torch.equal(dx.double(), dx_ref)


def test_conv_autograd_function(gpu):
    """Conv3dFn inside torch autograd: gradients of a two-layer net match FP64."""
    from voxelsim_fea_b200.learned import conv
    torch.manual_seed(5)
    x = torch.randn(7, 9, 17, 16, device="cuda").to(torch.bfloat16)
    w1 = (torch.randn(27, 32, 16, device="cuda") / 20).requires_grad_(True)
    b1 = torch.zeros(32, device="cuda", requires_grad=True)
    w2 = (torch.randn(27, 16, 32, device="cuda") / 30).requires_grad_(True)
    b2 = torch.zeros(16, device="cuda", requires_grad=True)
    y = conv.conv3d(torch.relu(conv.conv3d(x, w1, b1)), w2, b2)
    y.float().square().sum().backward()
    xr = _to_ncdhw(x)
    w1r = _w_torch(w1.to(torch.bfloat16)).requires_grad_(True)
    w2r = _w_torch(w2.to(torch.bfloat16)).requires_grad_(True)
    yr = F.conv3d(torch.relu(F.conv3d(xr, w1r, padding=1)), w2r, padding=1)
    yr.square().sum().backward()
    g1 = w1r.grad.permute(2, 3, 4, 0, 1).reshape(27, 32, 16)
    g2 = w2r.grad.permute(2, 3, 4, 0, 1).reshape(27, 16, 32)
    # BF16 storage of the hidden activation and of dY bounds the agreement
    assert _rel(w2.grad, g2) < 3e-2
    assert _rel(w1.grad, g1) < 3e-2
