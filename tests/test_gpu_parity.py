"""GPU parity: the CUDA path (through the C ABI) against natinterp3d's golden
outputs and against the CPU oracle on the same meshes.  Integer outputs
(row pointers, columns) must be identical; float64 weights and
interpolations must be bit-identical (tolerance 0), because the kernels
evaluate every expression with natinterp3d's operand grouping and no FMA."""
import numpy as np
import pytest
import scipy.sparse
import torch

from conftest import golden_names, load_golden
from oracle import oracle

import natinterp3d_b200 as ni
from natinterp3d_b200._native import HostMesh

pytestmark = pytest.mark.gpu


def bitwise_csr(A, B):
    assert np.array_equal(A.indptr, B.indptr), 'row pointers differ'
    assert np.array_equal(A.indices, B.indices), 'column order differs'
    a = np.asarray(A.data)
    b = np.asarray(B.data)
    assert a.dtype == b.dtype
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), \
        'weights differ: max abs %g' % np.abs(a.astype(np.float64) - b).max()


def golden_interp(name):
    g = load_golden(name)
    I = ni.Interpolator.from_mesh(g['centroid'], g['vxyz'], g['tet_v'], g['tet_n'])
    return g, I


@pytest.mark.parametrize('name', golden_names())
def test_weights_match_natinterp3d_golden(name, cuda_device):
    g, I = golden_interp(name)
    W = I.get_weights(g['queries'])
    ref = scipy.sparse.csr_matrix((g['data'], g['indices'], g['indptr']), shape=W.shape)
    ref = ref.astype(g['queries'].dtype, copy=False)
    assert isinstance(W, scipy.sparse.csr_matrix)
    assert W.indices.dtype == np.int32 and W.indptr.dtype == np.int32
    bitwise_csr(W, ref)


@pytest.mark.parametrize('name', golden_names())
def test_interpolate_matches_natinterp3d_golden(name, cuda_device):
    g, I = golden_interp(name)
    ref = scipy.sparse.csr_matrix((g['data'], g['indices'], g['indptr']),
                                  shape=(g['queries'].shape[0], g['keys'].shape[0]))
    ref = ref.astype(g['queries'].dtype, copy=False)
    for values in (g['values'], g['values2'], g['values2'].astype(np.float32)):
        out = I.interpolate(g['queries'], values)
        if values.ndim == 1:
            expect = np.squeeze(ref @ values[:, None], axis=1)
        else:
            expect = ref @ values
        assert out.shape == expect.shape and out.dtype == expect.dtype
        assert np.array_equal(out, expect), np.abs(out - expect).max()


def build(keys):
    c = keys.mean(axis=0)
    hm = HostMesh(keys - c)
    arrays = hm.export()
    return c, arrays, hm


def test_uniform_10k_keys_100k_queries_against_oracle(cuda_device):
    # the small plain get_weights workload: seed 0, keys U[0,1]^3, queries U[0.05,0.95]^3
    rng = np.random.default_rng(0)
    keys = rng.uniform(0, 1, (10000, 3))
    q = rng.uniform(0.05, 0.95, (100000, 3))
    c, arrays, hm = build(keys)
    I = ni.Interpolator.from_mesh(c, *arrays)
    W = I.get_weights(q)
    ref = oracle.OracleMesh(*arrays).weights(q - c)
    bitwise_csr(W, ref)
    v = np.sin(3 * keys[:, 0]) + np.cos(2 * keys[:, 1]) * keys[:, 2]
    out = I.interpolate(q, v)
    assert np.array_equal(out, np.squeeze(ref @ v[:, None], axis=1))
    if oracle.ref_available():
        bitwise_csr(W, oracle.ref_query(hm.native_pointer(), q - c, keys.shape[0], nthreads=4))


def test_lattice_mixture_against_oracle(cuda_device):
    rng = np.random.default_rng(2)
    g = 16
    lat = np.stack(np.meshgrid(*[np.arange(g)] * 3, indexing='ij'), -1).reshape(-1, 3) / g
    means = rng.uniform(0, 1, (16, 3))
    mix = np.clip(means[rng.integers(0, 16, 4000)] + rng.normal(0, 0.01, (4000, 3)), 0, 1)
    keys = np.concatenate([lat, mix])
    q = np.concatenate([rng.uniform(1 / g, 1 - 2 / g, (10000, 3)),
                        np.clip(means[rng.integers(0, 16, 10000)] + rng.normal(0, 0.01, (10000, 3)), 0, 1)])
    c, arrays, _ = build(keys)
    I = ni.Interpolator.from_mesh(c, *arrays)
    W = I.get_weights(q)
    bitwise_csr(W, oracle.OracleMesh(*arrays).weights(q - c))
    # linear reproduction against the mesh (perturbed) coordinates, for
    # queries at least 0.01 inside the convex hull: closer to the hull a
    # super-simplex vertex can be a natural neighbour, whose share natinterp3d
    # drops before normalising (the flat, clipped faces of the mixture make
    # that band visible)
    from scipy.spatial import ConvexHull
    vx = arrays[0][:keys.shape[0]] + c
    a, b = np.array([0.3, -1.2, 2.0]), 0.7
    f = vx @ a + b
    out = I.interpolate(q, f)
    eq = ConvexHull(vx).equations
    depth = -(q @ eq[:, :3].T + eq[:, 3]).max(axis=1)
    deep = depth > 0.01
    assert deep.sum() > 15000
    assert np.abs(out[deep] - (q[deep] @ a + b)).max() < 1e-12


def test_large_cavities_use_large_kernel(cuda_device):
    # keys on a sphere: a query at the centre lies inside every circumsphere,
    # so its cavity is far larger than the shared-memory kernel's capacity
    rng = np.random.default_rng(5)
    d = rng.normal(size=(600, 3))
    keys = d / np.linalg.norm(d, axis=1, keepdims=True)
    q = np.concatenate([np.zeros((1, 3)), rng.uniform(-0.3, 0.3, (50, 3)), rng.uniform(-0.9, 0.9, (200, 3))])
    c, arrays, _ = build(keys)
    I = ni.Interpolator.from_mesh(c, *arrays)
    rowptr, cols, vals, summ = I.device_mesh.weights_csr(
        torch.from_numpy(q).to(cuda_device), c, return_summary=True)
    assert summ['rows_large'] >= 1 and summ['rows_failed'] == 0
    W = scipy.sparse.csr_matrix((vals.cpu().numpy(), cols.cpu().numpy(), rowptr.cpu().numpy()),
                                shape=(q.shape[0], keys.shape[0]))
    bitwise_csr(W, oracle.OracleMesh(*arrays).weights(q - c))
    v = rng.normal(size=(keys.shape[0], 3))
    out = I.interpolate(q, v)
    assert np.array_equal(out, W @ v)


def test_outside_super_simplex_rows_are_empty(cuda_device):
    rng = np.random.default_rng(6)
    keys = rng.normal(size=(200, 3))
    q = np.array([[1e3, 1e3, 1e3], [-1e4, 0, 0], [0.0, 0.0, 0.0]])
    c, arrays, _ = build(keys)
    I = ni.Interpolator.from_mesh(c, *arrays)
    rowptr, cols, vals, summ = I.device_mesh.weights_csr(torch.from_numpy(q).to(cuda_device), c,
                                                         return_summary=True)
    rp = rowptr.cpu().numpy()
    assert rp[1] == rp[0] and rp[2] == rp[1] and rp[3] > rp[2]
    assert summ['rows_outside'] == 2


def test_deterministic_and_device_api(cuda_device):
    rng = np.random.default_rng(7)
    keys = rng.uniform(0, 1, (3000, 3))
    q = rng.uniform(0, 1, (20000, 3))
    I = ni.Interpolator(keys)
    W1 = I.get_weights(q)
    W2 = I.get_weights(q)
    bitwise_csr(W1, W2)
    qd = torch.from_numpy(q).to(cuda_device)
    rowptr, cols, vals = I.get_weights_device(qd)
    assert np.array_equal(rowptr.cpu().numpy(), W1.indptr)
    assert np.array_equal(cols.cpu().numpy(), W1.indices)
    assert np.array_equal(vals.cpu().numpy(), W1.data)
    v = torch.from_numpy(rng.normal(size=(3000, 16)).astype(np.float32)).to(cuda_device)
    out = I.interpolate_device(qd, v)
    assert out.dtype == torch.float64 and out.shape == (20000, 16)
    assert np.array_equal(out.cpu().numpy(), W1 @ v.cpu().numpy())
    S = I.get_weights_device(qd, as_torch_csr=True)
    assert S.layout == torch.sparse_csr


def test_float32_queries_and_values(cuda_device):
    rng = np.random.default_rng(8)
    keys = rng.normal(size=(1000, 3)).astype(np.float32)
    q = (rng.normal(size=(3000, 3)) * 0.4).astype(np.float32)
    v = rng.normal(size=(1000, 2)).astype(np.float32)
    c, arrays, hm = build(np.asarray(keys, np.float64))
    I = ni.Interpolator.from_mesh(c, *arrays)
    W = I.get_weights(q)
    assert W.dtype == np.float32
    ref = oracle.OracleMesh(*arrays).weights(np.asarray(q, np.float64) - c).astype(np.float32)
    bitwise_csr(W, ref)
    out = I.interpolate(q, v)
    assert out.dtype == np.float32
    assert np.array_equal(out, ref @ v)


def test_pipelined_host_interpolate_matches_single_call(cuda_device):
    # more than two pipeline chunks: the chunked host path must return exactly
    # what one device-resident call returns
    from natinterp3d_b200 import natinterp3d as api
    rng = np.random.default_rng(9)
    keys = rng.uniform(0, 1, (20000, 3))
    I = ni.Interpolator(keys)
    M = 2 * api.PIPELINE_CHUNK + 12345
    q = rng.uniform(0.0, 1.0, (M, 3))
    v = rng.normal(size=(20000, 3)).astype(np.float32)
    out = I.interpolate(q, v)
    ref = I.interpolate_device(torch.from_numpy(q).to(cuda_device),
                               torch.from_numpy(v).to(cuda_device)).cpu().numpy()
    assert out.shape == (M, 3) and out.dtype == np.float64
    assert np.array_equal(out, ref)
    out1 = I.interpolate(q, v[:, 0])
    assert out1.shape == (M,) and np.array_equal(out1, ref[:, 0])
