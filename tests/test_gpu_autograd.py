"""GPU tests of the differentiable path (forward, d/dvalues, d/dqueries)."""
import numpy as np
import pytest
import scipy.sparse
import torch

import natinterp3d_b200 as ni
from natinterp3d_b200 import autograd as nag

pytestmark = pytest.mark.gpu


def setup(nk, nq, seed, lo=0.1, hi=0.9, dim=4, vdtype=torch.float32, device=None):
    rng = np.random.default_rng(seed)
    keys = rng.uniform(0, 1, (nk, 3))
    interp = ni.Interpolator(keys, device=device)
    q = torch.from_numpy(rng.uniform(lo, hi, (nq, 3))).to(device).requires_grad_(True)
    v = torch.from_numpy(rng.standard_normal((nk, dim))).to(device, vdtype).requires_grad_(True)
    g = torch.from_numpy(rng.standard_normal((nq, dim))).to(device, torch.float64)
    return interp, q, v, g


def test_forward_and_values_gradient_match_scipy(cuda_device):
    interp, q, v, g = setup(5000, 20000, 0, device=cuda_device)
    out = nag.interpolate(interp, q, v)
    fused = interp.interpolate_device(q.detach(), v.detach())
    assert out.dtype == torch.float64
    assert torch.equal(out, fused)
    (out * g).sum().backward()
    W = interp.get_weights(q.detach().cpu().numpy())
    expect = (W.T @ g.cpu().numpy()).astype(np.float32)   # scipy: column sums in ascending row order
    assert v.grad.dtype == torch.float32
    assert np.array_equal(v.grad.cpu().numpy(), expect)


def test_values_gradient_f64_bitwise(cuda_device):
    interp, q, v, g = setup(3000, 10000, 1, vdtype=torch.float64, device=cuda_device)
    out = nag.interpolate(interp, q, v)
    (out * g).sum().backward()
    W = interp.get_weights(q.detach().cpu().numpy())
    assert np.array_equal(v.grad.cpu().numpy(), W.T @ g.cpu().numpy())


def _pattern(W, i):
    return tuple(sorted(W.indices[W.indptr[i]:W.indptr[i + 1]]))


def test_query_gradient_matches_central_differences(cuda_device):
    # 1,000 queries, FP64 central differences with h = 1e-6, away from degenerate
    # configurations: rows whose natural-neighbour set changes within +-h are skipped
    interp, q, v, g = setup(20000, 1000, 2, dim=3, vdtype=torch.float64, device=cuda_device)
    out = nag.interpolate(interp, q, v)
    (out * g).sum().backward()
    gq = q.grad.cpu().numpy()
    qn = q.detach().cpu().numpy()
    vn = v.detach().cpu().numpy()
    gn = g.cpu().numpy()
    h = 1e-6
    W0 = interp.get_weights(qn)
    fd = np.zeros_like(qn)
    keep = np.ones(qn.shape[0], bool)
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        Wp, Wm = interp.get_weights(qn + e), interp.get_weights(qn - e)
        lp = ((Wp @ vn) * gn).sum(axis=1)
        lm = ((Wm @ vn) * gn).sum(axis=1)
        fd[:, d] = (lp - lm) / (2 * h)
        for i in range(qn.shape[0]):
            if keep[i] and not (_pattern(Wp, i) == _pattern(W0, i) == _pattern(Wm, i)):
                keep[i] = False
    assert keep.sum() >= 950
    rel = np.linalg.norm(gq - fd, axis=1) / np.maximum(np.linalg.norm(fd, axis=1), 1e-12)
    assert np.all(rel[keep] < 1e-5), (rel[keep].max(), np.argmax(rel * keep))
    assert np.median(rel[keep]) < 1e-8


def test_query_gradient_of_linear_field_is_the_slope(cuda_device):
    # interpolating an affine function reproduces it inside the hull, so
    # d/dq of a.out = a.A exactly (up to rounding) away from the hull
    rng = np.random.default_rng(3)
    keys = rng.uniform(0, 1, (8000, 3))
    interp = ni.Interpolator(keys, device=cuda_device)
    vx = interp.mesh_arrays[0][:8000] + interp.centroid
    A = np.array([[1.0, -2.0, 0.5], [0.3, 0.7, -1.1]])  # values = vx @ A.T + b
    vals = torch.from_numpy(vx @ A.T + np.array([0.2, -0.4])).to(cuda_device)
    q = torch.from_numpy(rng.uniform(0.2, 0.8, (500, 3))).to(cuda_device).requires_grad_(True)
    out = nag.interpolate(interp, q, vals)
    wgt = torch.tensor([[1.5, -0.5]], dtype=torch.float64, device=cuda_device)
    (out * wgt).sum().backward()
    expect = (wgt.cpu().numpy() @ A).ravel()
    assert np.abs(q.grad.cpu().numpy() - expect).max() < 1e-9


def test_float32_inputs_and_module(cuda_device):
    rng = np.random.default_rng(4)
    keys = rng.uniform(0, 1, (2000, 3))
    mod = nag.SibsonInterpolation(keys, device=cuda_device)
    q = torch.from_numpy(rng.uniform(0.2, 0.8, (300, 3)).astype(np.float32)).to(cuda_device)
    q.requires_grad_(True)
    v = torch.from_numpy(rng.standard_normal(2000).astype(np.float32)).to(cuda_device)
    v.requires_grad_(True)
    out = mod(q, v)
    assert out.shape == (300,) and out.dtype == torch.float32
    out.sum().backward()
    assert q.grad.dtype == torch.float32 and torch.isfinite(q.grad).all()
    assert v.grad.shape == (2000,) and v.grad.dtype == torch.float32


def test_ordered_transpose_product_is_bit_identical(cuda_device):
    # the transpose product with the columns visited in a caller-given order
    # (the mesh's spatial key order, or any permutation) equals the plain one
    # and scipy's W.T @ x bit for bit
    import ctypes
    from natinterp3d_b200 import _native as N
    from natinterp3d_b200.device import _vp, _stream_ptr
    rng = np.random.default_rng(17)
    M, Ncol, D = 5000, 3000, 5
    W = scipy.sparse.random(M, Ncol, density=0.004, format='csr', random_state=3, dtype=np.float64)
    x = rng.standard_normal((M, D))
    dev = cuda_device
    rowptr = torch.from_numpy(W.indptr.astype(np.int32)).to(dev)
    cols = torch.from_numpy(W.indices.astype(np.int32)).to(dev)
    vals = torch.from_numpy(W.data).to(dev)
    xd = torch.from_numpy(x).to(dev)
    rank = torch.from_numpy(rng.permutation(Ncol).astype(np.int32)).to(dev)
    lib = N.cuda_lib()
    nb = ctypes.c_size_t()
    N.check(lib.nif_spmm_t_workspace_bytes(M, Ncol, W.nnz, ctypes.byref(nb)), 'ws')
    ws = torch.empty(int(nb.value), dtype=torch.uint8, device=dev)
    outs = []
    for ordered in (False, True):
        y = torch.empty((Ncol, D), dtype=torch.float64, device=dev)
        args = [M, Ncol, W.nnz, _vp(rowptr), _vp(cols), _vp(vals), N.NIF_F64, _vp(xd), N.NIF_F64, D,
                _vp(y), N.NIF_F64]
        if ordered:
            rc = lib.nif_spmm_t_ordered(*args, _vp(rank), _vp(ws), ws.numel(), _stream_ptr(dev))
        else:
            rc = lib.nif_spmm_t(*args, _vp(ws), ws.numel(), _stream_ptr(dev))
        N.check(rc, 'spmm_t')
        outs.append(y.cpu().numpy())
    assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8))
    ref = W.T.tocsr() @ x
    assert np.abs(outs[1] - ref).max() < 1e-12
