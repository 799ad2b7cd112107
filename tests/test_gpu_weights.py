"""get_weights rows far larger than the shared-memory kernel holds, in bulk.

400 keys within 1 % of a unit sphere, 14,000 queries within 0.1 of its
centre: every query's cavity holds most of the mesh and its row has hundreds
of natural neighbours (about 4.7M non-zeros in all).  The count pass runs
these rows in the large-capacity kernel and the fill pass recomputes them
straight into their CSR slices, so the total is bounded by nothing but the
CSR itself (natinterp3d grows its per-thread arenas the same way).  The rows
must equal the oracle's bit for bit, and partition unity.
"""
import numpy as np
import pytest

import natinterp3d_b200 as ni
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_bulk_large_rows_against_oracle(cuda_device):
    rng = np.random.default_rng(21)
    d = rng.standard_normal((400, 3))
    keys = d / np.linalg.norm(d, axis=1, keepdims=True) * (1 + 0.01 * rng.uniform(-1, 1, (400, 1)))
    d = rng.standard_normal((14_000, 3))
    q = d / np.linalg.norm(d, axis=1, keepdims=True) * 0.1 * rng.uniform(0, 1, (14_000, 1)) ** (1 / 3)
    interp = ni.Interpolator(keys, device=cuda_device)
    W = interp.get_weights(q)
    summ = interp.device_mesh.last_summary
    assert summ['rows_large'] == q.shape[0] and summ['rows_failed'] == 0
    assert W.nnz > (1 << 22)  # more than the former fixed staging arena held
    Wo = oracle.OracleMesh(*interp.mesh_arrays).weights(q - interp.centroid)
    assert np.array_equal(W.indptr, Wo.indptr)
    assert np.array_equal(W.indices, Wo.indices)
    assert np.array_equal(W.data.view(np.uint8), Wo.data.view(np.uint8))
    assert np.abs(np.asarray(W.sum(axis=1)).ravel() - 1).max() < 1e-10


def test_float32_weights_through_the_fill_pass(cuda_device):
    # rows of more than 24 entries are recomputed at fill time, also into
    # float32 weights
    rng = np.random.default_rng(22)
    keys = rng.uniform(0, 1, (3000, 3))
    q = rng.uniform(0.05, 0.95, (40_000, 3))
    interp = ni.Interpolator(keys, device=cuda_device)
    W64 = interp.get_weights(q)
    lens = np.diff(W64.indptr)
    assert (lens > 24).sum() > 0
    W32 = interp.get_weights(q.astype(np.float32))
    assert W32.dtype == np.float32
    Wo = oracle.OracleMesh(*interp.mesh_arrays).weights(
        q.astype(np.float32).astype(np.float64) - interp.centroid).astype(np.float32)
    assert np.array_equal(W32.indptr, Wo.indptr) and np.array_equal(W32.indices, Wo.indices)
    assert np.array_equal(W32.data.view(np.uint8), Wo.data.view(np.uint8))
