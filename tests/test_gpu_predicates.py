"""GPU tests of the predicate modes against the CPU oracle's modes.

'fast' is natinterp3d's behaviour (the other GPU parity tests);
'audit' must return the same bits and count the uncertain and flipped
predicate evaluations exactly as the oracle does; 'exact' must match the
oracle's exact mode bit for bit, including queries lying exactly on faces,
edges and vertices, where the device's walk seed (a grid) and the oracle's
(the nearest tet centroid, or tet 0) reach different containing tets."""
import ctypes

import numpy as np
import pytest
import scipy.sparse
import torch

from conftest import dyadic_keys, golden_names, load_golden, on_face_queries
from oracle import oracle

import natinterp3d_b200 as ni
from natinterp3d_b200 import _native as N
from natinterp3d_b200 import autograd as nag
from natinterp3d_b200._native import HostMesh
from natinterp3d_b200.batch import BatchInterpolator

pytestmark = pytest.mark.gpu

COUNTERS = ('orient_uncertain', 'orient_flipped', 'insphere_uncertain', 'insphere_flipped')


def bitwise_csr(A, B):
    assert np.array_equal(A.indptr, B.indptr), 'row pointers differ'
    assert np.array_equal(A.indices, B.indices), 'column order differs'
    a, b = np.asarray(A.data), np.asarray(B.data)
    assert a.dtype == b.dtype
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), \
        'weights differ: max abs %g' % np.abs(a.astype(np.float64) - b).max()


def gpu_weights(I, q):
    dm = I.device_mesh
    qd = torch.from_numpy(np.ascontiguousarray(q, np.float64)).to(dm.device)
    rowptr, cols, vals, summ = dm.weights_csr(qd, I.centroid, return_summary=True)
    W = scipy.sparse.csr_matrix((vals.cpu().numpy(), cols.cpu().numpy(), rowptr.cpu().numpy()),
                                shape=(len(q), I.n_keys))
    return W, summ


def oracle_weights(arrays, qc, mode, first_tet=False):
    om = oracle.OracleMesh(*arrays)
    om.set_predicates(mode)
    om.set_seed(first_tet)
    W, st, _ = om.weights(qc, with_stats=True)
    return W, st, om.predicate_info()


def dyadic_case(seed=0, bits=10):
    keys = dyadic_keys(seed=seed, bits=bits)
    c = keys.mean(axis=0)
    arrays = HostMesh(keys - c).export()
    qc = on_face_queries(arrays[0], arrays[1], len(keys))
    q = qc + c
    assert np.array_equal(q - c, qc)  # the device sees exactly these points
    return keys, c, arrays, q, qc


@pytest.mark.parametrize('name', golden_names())
def test_audit_mode_matches_fast_and_counts_like_the_oracle(name, cuda_device):
    g = load_golden(name)
    arrays = (g['vxyz'], g['tet_v'], g['tet_n'])
    q = np.asarray(g['queries'], np.float64)
    I = ni.Interpolator.from_mesh(g['centroid'], *arrays)
    fast, _ = gpu_weights(I, q)
    I.set_predicates('audit')
    audit, summ = gpu_weights(I, q)
    bitwise_csr(audit, fast)
    _, st, pinfo = oracle_weights(arrays, q - g['centroid'], 'audit')
    # in-sphere tests: the same set of tets is tested whatever the walk's seed
    assert summ['insphere_uncertain'] == st['insphere_uncertain']
    assert summ['insphere_flipped'] == st['insphere_flipped']
    assert summ['orient_flipped'] <= summ['orient_uncertain']
    assert I.device_mesh.orientation_stats == {'uncertain': pinfo[0], 'flipped': pinfo[1]}
    stats = I.predicate_stats
    assert all(stats[k] == summ[k] for k in COUNTERS)


@pytest.mark.parametrize('name', golden_names())
def test_exact_mode_matches_the_oracle_on_goldens(name, cuda_device):
    g = load_golden(name)
    arrays = (g['vxyz'], g['tet_v'], g['tet_n'])
    q = np.asarray(g['queries'], np.float64)
    I = ni.Interpolator.from_mesh(g['centroid'], *arrays, predicates='exact')
    W, summ = gpu_weights(I, q)
    ref, st, _ = oracle_weights(arrays, q - g['centroid'], 'exact')
    bitwise_csr(W, ref)
    assert summ['insphere_uncertain'] == st['insphere_uncertain']
    assert summ['insphere_flipped'] == st['insphere_flipped']


def test_grid_golden_flips_natinterp3d_decisions(cuda_device):
    """On the 6^3 grid some of natinterp3d's in-sphere decisions are wrong; the
    audit counts them and the exact mode changes the weights."""
    g = load_golden('grid6')
    I = ni.Interpolator.from_mesh(g['centroid'], g['vxyz'], g['tet_v'], g['tet_n'],
                                  predicates='audit')
    q = np.asarray(g['queries'], np.float64)
    fast, summ = gpu_weights(I, q)
    assert summ['insphere_flipped'] > 0 and summ['rows_large'] > 0
    I.set_predicates('exact')
    exact, _ = gpu_weights(I, q)
    assert not (np.array_equal(fast.indptr, exact.indptr) and np.array_equal(fast.indices, exact.indices)
                and np.array_equal(fast.data, exact.data))


@pytest.mark.parametrize('first_tet', [False, True])
def test_exact_mode_on_faces_edges_and_vertices(first_tet, cuda_device):
    keys, c, arrays, q, qc = dyadic_case()
    I = ni.Interpolator.from_mesh(c, *arrays, predicates='exact')
    W, summ = gpu_weights(I, q)
    ref, st, _ = oracle_weights(arrays, qc, 'exact', first_tet=first_tet)
    bitwise_csr(W, ref)
    assert summ['orient_uncertain'] > 0 and summ['rows_large'] > 0
    assert summ['insphere_uncertain'] == st['insphere_uncertain']
    # fused interpolation in exact mode: scipy's order over the exact weights
    v = np.random.default_rng(2).standard_normal((len(keys), 3))
    assert np.array_equal(I.interpolate(q, v), oracle.spmm_like_scipy(ref, v))
    # float32 weights are sorted per row, as natinterp3d's astype leaves them
    Wf = I.get_weights(q.astype(np.float32))
    assert Wf.dtype == np.float32 and Wf.has_sorted_indices


def test_exact_mode_large_cavities(cuda_device):
    rng = np.random.default_rng(5)
    d = rng.normal(size=(600, 3))
    keys = d / np.linalg.norm(d, axis=1, keepdims=True)
    q = np.concatenate([np.zeros((1, 3)), rng.uniform(-0.3, 0.3, (50, 3))])
    c = keys.mean(axis=0)
    arrays = HostMesh(keys - c).export()
    for mode in ('audit', 'exact'):
        I = ni.Interpolator.from_mesh(c, *arrays, predicates=mode)
        W, summ = gpu_weights(I, q)
        ref, st, _ = oracle_weights(arrays, q - c, mode)
        assert summ['rows_large'] >= 1 and summ['rows_failed'] == 0
        bitwise_csr(W, ref)
        assert summ['insphere_uncertain'] == st['insphere_uncertain']


def test_batch_with_mixed_predicate_modes(cuda_device):
    cases = [dyadic_case(seed=s) for s in (0, 1)]
    rng = np.random.default_rng(3)
    rkeys = rng.uniform(0, 1, (3000, 3))
    keys_list = [cases[0][0], cases[1][0], rkeys]
    modes = ['exact', 'fast', 'audit']
    B = BatchInterpolator(keys_list, device=cuda_device, predicates=modes)
    qs = [cases[0][3], cases[1][3], rng.uniform(0.05, 0.95, (2000, 3))]
    vs = [rng.standard_normal((len(k), 2)) for k in keys_list]
    outs = B.interpolate(qs, vs)
    for p, (keys, q, v, mode) in enumerate(zip(keys_list, qs, vs, modes)):
        I = ni.Interpolator(keys, device=cuda_device, predicates=mode)
        assert np.array_equal(outs[p], I.interpolate(q, v))


def test_exact_mode_autograd_and_noalloc(cuda_device):
    keys, c, arrays, q, qc = dyadic_case(seed=4)
    I = ni.Interpolator.from_mesh(c, *arrays, predicates='exact')
    qd = torch.from_numpy(q).to(cuda_device).requires_grad_(True)
    vd = torch.from_numpy(np.random.default_rng(1).standard_normal((len(keys), 2))).to(cuda_device)
    out = nag.interpolate(I, qd, vd)
    assert torch.equal(out.detach(), I.interpolate_device(qd.detach(), vd))
    out.sum().backward()
    assert torch.isfinite(qd.grad).all()
    # the allocation-free entry point resolves the same predicates
    dm = I.device_mesh
    res = torch.empty((len(q), 2), dtype=torch.float64, device=cuda_device)
    cen = (ctypes.c_double * 3)(*[float(x) for x in c])
    summ = N.Summary()
    qv = qd.detach().contiguous()
    rc = N.cuda_lib().nif_interpolate_noalloc(
        dm._h, ctypes.c_void_p(qv.data_ptr()), N.NIF_F64, len(q), cen, ctypes.c_void_p(vd.data_ptr()),
        N.NIF_F64, 2, ctypes.c_void_p(res.data_ptr()), N.NIF_F64,
        ctypes.c_void_p(torch.cuda.current_stream(cuda_device).cuda_stream), ctypes.byref(summ))
    assert rc == N.NIF_OK and summ.rows_failed == 0 and summ.orient_uncertain > 0
    assert torch.equal(res, out.detach())


def test_random_queries_have_nothing_uncertain(cuda_device):
    rng = np.random.default_rng(8)
    keys = rng.uniform(0, 1, (20000, 3))
    q = rng.uniform(0.05, 0.95, (200000, 3))
    I = ni.Interpolator(keys, device=cuda_device)
    fast, _ = gpu_weights(I, q)
    for mode in ('audit', 'exact'):
        I.set_predicates(mode)
        W, summ = gpu_weights(I, q)
        bitwise_csr(W, fast)
        assert all(summ[k] == 0 for k in COUNTERS)
