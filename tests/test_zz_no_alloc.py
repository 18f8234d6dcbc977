"""vf_apply_noalloc: the fine hex8 operator (+ u.y) for callers that cannot
allocate device memory -- programs whose device memory all comes from their
own allocator or a fixed arena, or that must avoid the device synchronisation
cudaMalloc/cudaFree can cause.  The entry point takes the caller's device
buffers and uses only the library's fixed static scratch array.

Checked through the C-ABI against the existing vf_apply (MGSolver._apply at
level 0) with the FP64 operator tolerance of the other parity tests, on two
calls in a row with different inputs (the shared scratch is reused), and for
the size limit of that scratch.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-13


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_apply_noalloc_matches_vf_apply(gpu):
    import torch
    from voxelsim_fea_b200 import _lib
    from voxelsim_fea_b200.multigrid import MGSolver

    g = golden("mg_ops_16x8x8.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    nu = float(g["nu"])
    m = MGSolver(nx, ny, nz, g["fixed"], nu=nu)
    m.set_density(g["E"])
    ndof = m.ndof
    free = np.ones(ndof, dtype=bool)
    free[g["fixed"]] = False
    mask = (free.reshape(-1, 3) * np.array([1, 2, 4])).sum(axis=1).astype(np.uint8)

    dev = torch.device("cuda", 0)
    E_d = torch.from_numpy(np.ascontiguousarray(g["E"], dtype=np.float64)).to(dev)
    mask_d = torch.from_numpy(mask).to(dev)
    u_d = torch.empty(ndof, dtype=torch.float64, device=dev)
    y_d = torch.empty(ndof, dtype=torch.float64, device=dev)
    dot_d = torch.empty(1, dtype=torch.float64, device=dev)
    L = _lib.load()
    rng = np.random.default_rng(2024)
    for call in range(2):
        u = rng.standard_normal(ndof) * (1.0 + call)
        ref = m._apply(0, u)                       # existing entry point (vf_apply)
        u_d.copy_(torch.from_numpy(u))
        y_d.fill_(float("nan"))
        dot_d.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.vf_apply_noalloc(nx, ny, nz, nu, _ptr(E_d), _ptr(mask_d), _ptr(u_d), _ptr(y_d), _ptr(dot_d),
                                None)
        assert rc == _lib.VF_OK, L.vf_global_last_error()
        torch.cuda.synchronize()
        y = y_d.cpu().numpy()
        scale = np.abs(ref).max()
        assert np.abs(y - ref).max() <= FP64_RTOL * scale, (call, np.abs(y - ref).max() / scale)
        dot_ref = float(u @ ref)
        assert abs(dot_d.item() - dot_ref) <= FP64_RTOL * np.abs(u).sum() * scale, (call, dot_d.item(), dot_ref)
    m.close()


def test_apply_noalloc_many_blocks_on_a_stream(gpu):
    """A 48x24x24 grid (about 120 blocks of the last-block reduction) on a
    non-default stream, two calls back to back on that stream before one
    synchronisation: both results against vf_apply."""
    import torch
    from voxelsim_fea_b200 import _lib
    from voxelsim_fea_b200.multigrid import MGSolver

    nx, ny, nz, nu = 48, 24, 24, 0.3
    rng = np.random.default_rng(77)
    E = np.exp(rng.standard_normal(nx * ny * nz))
    nn = (nx + 1) * (ny + 1) * (nz + 1)
    fixed = np.arange(0, 3 * nn, 3 * (nx + 1))          # x DOF of every x=0 node
    m = MGSolver(nx, ny, nz, fixed, nu=nu)
    m.set_density(E)
    free = np.ones(3 * nn, dtype=bool)
    free[fixed] = False
    mask = (free.reshape(-1, 3) * np.array([1, 2, 4])).sum(axis=1).astype(np.uint8)
    us = [rng.standard_normal(3 * nn), rng.standard_normal(3 * nn) * 3.0]
    refs = [m._apply(0, u) for u in us]
    m.close()

    dev = torch.device("cuda", 0)
    E_d = torch.from_numpy(E).to(dev)
    mask_d = torch.from_numpy(mask).to(dev)
    u_d = [torch.from_numpy(u).to(dev) for u in us]
    y_d = [torch.full((3 * nn,), float("nan"), dtype=torch.float64, device=dev) for _ in us]
    dot_d = [torch.full((1,), float("nan"), dtype=torch.float64, device=dev) for _ in us]
    torch.cuda.synchronize()
    L = _lib.load()
    st = torch.cuda.Stream(device=dev)
    for k in range(2):
        rc = L.vf_apply_noalloc(nx, ny, nz, nu, _ptr(E_d), _ptr(mask_d), _ptr(u_d[k]), _ptr(y_d[k]),
                                _ptr(dot_d[k]), ctypes.c_void_p(st.cuda_stream))
        assert rc == _lib.VF_OK, L.vf_global_last_error()
    st.synchronize()
    for k in range(2):
        y = y_d[k].cpu().numpy()
        scale = np.abs(refs[k]).max()
        assert np.abs(y - refs[k]).max() <= FP64_RTOL * scale, (k, np.abs(y - refs[k]).max() / scale)
        dot_ref = float(us[k] @ refs[k])
        assert abs(dot_d[k].item() - dot_ref) <= FP64_RTOL * np.abs(us[k]).sum() * scale, (k, dot_d[k].item())


def test_apply_noalloc_rejects_aliasing(gpu):
    import torch
    from voxelsim_fea_b200 import _lib
    L = _lib.load()
    nx, ny, nz = 4, 4, 4
    t = torch.zeros(3 * 125 + 8, dtype=torch.float64, device="cuda")
    m = torch.zeros(125, dtype=torch.uint8, device="cuda")
    d = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.vf_apply_noalloc(nx, ny, nz, 0.3, _ptr(t), _ptr(m), _ptr(t), _ptr(t), _ptr(d), None)
    assert rc == _lib.VF_ERR_ARG
    assert b"overlap" in L.vf_global_last_error()


def test_apply_noalloc_rejects_oversized_grid(gpu):
    import torch
    from voxelsim_fea_b200 import _lib
    L = _lib.load()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    # (257)^3 nodes exceed the fixed scratch (8,388,608 nodes): rejected before any launch
    rc = L.vf_apply_noalloc(256, 256, 256, 0.3, _ptr(t), _ptr(t), _ptr(t), _ptr(t), _ptr(t), None)
    assert rc == _lib.VF_ERR_ARG
    assert b"8388608" in L.vf_global_last_error()
