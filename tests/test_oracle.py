"""CPU checker pins: the oracle restatement against natinterp3d's golden
outputs (committed fixtures) and, where natinterp3d's sources were built here,
against natinterp3d's own query code on freshly built meshes."""
import numpy as np
import pytest
import scipy.sparse

from conftest import golden_names, load_golden
from oracle import oracle


def csr_bitwise_equal(A, B):
    return (np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices)
            and np.array_equal(np.asarray(A.data, np.float64).view(np.int64),
                               np.asarray(B.data, np.float64).view(np.int64)))


@pytest.mark.parametrize('name', golden_names())
def test_oracle_matches_golden(name):
    g = load_golden(name)
    om = oracle.OracleMesh(g['vxyz'], g['tet_v'], g['tet_n'])
    qc = np.ascontiguousarray(g['queries'], np.float64) - g['centroid']
    W = om.weights(qc)
    ref = scipy.sparse.csr_matrix((g['data'], g['indices'], g['indptr']), shape=W.shape)
    assert csr_bitwise_equal(W, ref)


@pytest.mark.parametrize('name', golden_names())
def test_oracle_spmm_matches_scipy(name):
    g = load_golden(name)
    ref = scipy.sparse.csr_matrix((g['data'], g['indices'], g['indptr']),
                                  shape=(g['queries'].shape[0], g['keys'].shape[0]))
    y = oracle.spmm_like_scipy(ref, g['values'])
    assert np.array_equal(y.reshape(-1, 1), g['interp'])
    y2 = oracle.spmm_like_scipy(ref, g['values2'])
    assert np.array_equal(y2, g['interp2'])


def test_predicates_known_answers():
    a, b, c, d = [0., 0, 0], [1., 0, 0], [0., 1, 0], [0., 0, 1]
    assert oracle.orient(a, b, c, d) == pytest.approx(-1.0) or oracle.orient(a, b, c, d) == pytest.approx(1.0)
    assert oracle.orient(a, b, c, [0.3, 0.3, 0.0]) == 0.0
    # centre of the circumsphere is strictly inside; a far point is outside
    s = np.sign(oracle.orient(a, b, c, d))
    inside = oracle.insphere(a, b, c, d, [0.25, 0.25, 0.25]) * s
    outside = oracle.insphere(a, b, c, d, [5.0, 5.0, 5.0]) * s
    assert inside * outside < 0
    # a vertex lies on its own circumsphere: exactly zero
    assert oracle.insphere(a, b, c, d, a) == 0.0


def test_tet_geometry_shapes():
    g = load_golden('uniform_2k')
    om = oracle.OracleMesh(g['vxyz'], g['tet_v'], g['tet_n'])
    pos, tcc, fcc = om.tet_geometry()
    assert pos.shape == (g['tet_v'].shape[0],) and pos.all()
    # circumcentres are equidistant from the tet's vertices
    v = g['vxyz'][g['tet_v']]
    d = np.linalg.norm(v - tcc[:, None, :], axis=2)
    assert np.allclose(d, d[:, :1], rtol=1e-6)


needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason='natinterp3d reference library not built here')


@needs_ref
@pytest.mark.parametrize('seed,nk,nq', [(0, 3000, 6000), (1, 500, 2000)])
def test_oracle_matches_natinterp3d_uniform(seed, nk, nq):
    from natinterp3d_b200._native import HostMesh
    rng = np.random.default_rng(seed)
    keys = rng.uniform(0, 1, (nk, 3))
    q = rng.uniform(-0.1, 1.1, (nq, 3))
    c = keys.mean(axis=0)
    hm = HostMesh(keys - c)
    om = oracle.OracleMesh(*hm.export())
    W = om.weights(q - c)
    R = oracle.ref_query(hm.native_pointer(), q - c, nk, nthreads=2)
    assert csr_bitwise_equal(W, R)


@needs_ref
def test_oracle_matches_natinterp3d_lattice():
    from natinterp3d_b200._native import HostMesh
    rng = np.random.default_rng(4)
    g = 8
    lat = np.stack(np.meshgrid(*[np.arange(g)] * 3, indexing='ij'), -1).reshape(-1, 3) / g
    keys = np.concatenate([lat, rng.uniform(0, 1, (300, 3))])
    q = np.concatenate([rng.uniform(0.1, 0.8, (2000, 3)), lat[::3]])
    c = keys.mean(axis=0)
    hm = HostMesh(keys - c)
    assert hm.degeneracies()['cospherical'] > 0
    om = oracle.OracleMesh(*hm.export())
    W = om.weights(q - c)
    R = oracle.ref_query(hm.native_pointer(), q - c, keys.shape[0], nthreads=1)
    assert csr_bitwise_equal(W, R)


def test_oracle_counts_flops_inputs():
    g = load_golden('uniform_2k')
    om = oracle.OracleMesh(g['vxyz'], g['tet_v'], g['tet_n'])
    _, st, status = om.weights(g['queries'] - g['centroid'], with_stats=True)
    assert st['queries'] == g['queries'].shape[0] and st['errors'] == 0
    assert (status == 0).all()
    assert st['insphere'] > st['cavity'] > 0 and st['old_terms'] > 0 and st['new_terms'] > 0
