"""The query gradient from the forward's kept cavity records
(nif_weights_count_records + nif_query_grad_records) against the gradient
that locates and floods every cavity again (nif_query_grad): bit for bit,
on rows of every kind the record path routes differently -- rows with a
record, rows whose cavity is wider than a record (48 < tets <= 96, the fused
kernel), rows beyond the shared-memory capacities (the large kernel) --
and across record chunks of 1M rows."""
import numpy as np
import pytest
import torch

import natinterp3d_b200 as ni
from natinterp3d_b200 import autograd as nag

pytestmark = pytest.mark.gpu


def _mixed(rng):
    # uniform keys plus a small sphere of keys: queries inside the sphere
    # have cavities of tens to hundreds of tets
    keys = rng.uniform(0, 1, (3000, 3))
    d = rng.standard_normal((300, 3))
    keys = np.concatenate([keys, 0.5 + d / np.linalg.norm(d, axis=1, keepdims=True) * 0.06])
    d = rng.standard_normal((4000, 3))
    q = np.concatenate([
        0.5 + d / np.linalg.norm(d, axis=1, keepdims=True) * 0.06 * rng.uniform(0, 1.3, (4000, 1)),
        rng.uniform(0.05, 0.95, (4000, 3))])
    return keys, q


def _both(interp, q, v, g):
    dm = interp.device_mesh
    rowptr, cols, w64, tot, summ, rec = dm.weights_csr(q, interp.centroid, return_totals=True,
                                                       return_summary=True, keep_records=True)
    r2, c2, w2, t2 = dm.weights_csr(q, interp.centroid, return_totals=True)
    assert torch.equal(rowptr, r2) and torch.equal(cols, c2)
    assert torch.equal(w64.view(torch.int64), w2.view(torch.int64))
    assert torch.equal(tot.view(torch.int64), t2.view(torch.int64))
    g_rec = dm.query_grad(q, v, g, interp.centroid, rowptr, w64, tot, records=rec)
    g_new = dm.query_grad(q, v, g, interp.centroid, rowptr, w64, tot)
    return g_rec, g_new, summ


@pytest.mark.parametrize('qdt', [torch.float64, torch.float32])
def test_records_gradient_equals_recomputed(cuda_device, qdt):
    rng = np.random.default_rng(31)
    keys, qn = _mixed(rng)
    interp = ni.Interpolator(keys, device=cuda_device)
    q = torch.from_numpy(qn).to(cuda_device, qdt)
    vdt = torch.float32
    v = torch.from_numpy(rng.standard_normal((interp.n_keys, 5))).to(cuda_device, vdt)
    gdt = torch.float32 if qdt == torch.float32 else torch.float64
    g = torch.from_numpy(rng.standard_normal((q.shape[0], 5))).to(cuda_device, gdt)
    g_rec, g_new, summ = _both(interp, q, v, g)
    assert summ['rows_wide'] > 0 and summ['rows_large'] > 0
    assert torch.isfinite(g_new).all() and g_new.abs().sum() > 0
    assert torch.equal(g_rec, g_new)


def test_records_across_chunks(cuda_device):
    # more rows than one record chunk (1M): chunk c's records sit at its rows'
    # positions
    rng = np.random.default_rng(32)
    interp = ni.Interpolator(rng.uniform(0, 1, (20_000, 3)), device=cuda_device)
    M = (1 << 20) + 150_001
    q = torch.from_numpy(rng.uniform(0.03, 0.97, (M, 3))).to(cuda_device)
    v = torch.from_numpy(rng.standard_normal((interp.n_keys, 2))).to(cuda_device)
    g = torch.from_numpy(rng.standard_normal((M, 2))).to(cuda_device)
    g_rec, g_new, _ = _both(interp, q, v, g)
    assert torch.equal(g_rec, g_new)


def test_autograd_uses_records_and_matches(cuda_device):
    rng = np.random.default_rng(33)
    keys, qn = _mixed(rng)
    interp = ni.Interpolator(keys, device=cuda_device)
    v0 = torch.from_numpy(rng.standard_normal((interp.n_keys, 3))).to(cuda_device)
    go = torch.from_numpy(rng.standard_normal((qn.shape[0], 3))).to(cuda_device)
    grads = []
    for limit in (nag.RECORDS_MAX_BYTES, 0):  # records kept, then not
        old = nag.RECORDS_MAX_BYTES
        nag.RECORDS_MAX_BYTES = limit
        try:
            q = torch.from_numpy(qn).to(cuda_device).requires_grad_(True)
            v = v0.clone().requires_grad_(True)
            out = nag.interpolate(interp, q, v)
            (out * go).sum().backward()
            grads.append((out.detach(), q.grad, v.grad))
        finally:
            nag.RECORDS_MAX_BYTES = old
    for a, b in zip(*grads):
        assert torch.equal(a, b)


def test_records_refused_for_other_predicates(cuda_device):
    rng = np.random.default_rng(34)
    interp = ni.Interpolator(rng.uniform(0, 1, (500, 3)), device=cuda_device, predicates='exact')
    q = torch.from_numpy(rng.uniform(0.1, 0.9, (100, 3))).to(cuda_device)
    with pytest.raises(ValueError):
        interp.device_mesh.weights_csr(q, interp.centroid, keep_records=True)
