"""natinterp3d's own test properties, run against natinterp3d_b200.

natinterp3d's suite (tests/test_natinterp3d.py) checks the public API:
- partition of unity, non-negativity, linear precision and the local-coordinate identity;
- convergence under refinement;
- symmetric known answers and queries at data points;
- behaviour outside the hull;
- tiny key sets, large offsets and scales;
- output shapes and dtypes, reuse, the module-level functions, determinism and sparsity.

The same checks follow, with the same seeds and tolerances, through
``natinterp3d_b200``'s drop-in API (the GPU path).
"""
import numpy as np
import pytest
import scipy.sparse

import natinterp3d_b200 as natinterp3d

pytestmark = pytest.mark.gpu


def near_centre(keys, n, rng, margin=0.8):
    """Queries drawn around the key centroid, mostly inside the hull."""
    return keys.mean(axis=0) + rng.randn(n, 3) * keys.std(axis=0) * margin * 0.3


def row_sums(W):
    return np.asarray(W.sum(axis=1)).ravel()


# ---- properties of Sibson coordinates ----------------------------------------

def test_partition_of_unity_random():
    rng = np.random.RandomState(42)
    keys = rng.randn(200, 3)
    s = row_sums(natinterp3d.get_weights(near_centre(keys, 50, rng), keys))
    inside = s > 0.5
    assert inside.sum() > 30
    np.testing.assert_allclose(s[inside], 1.0, atol=1e-10)


def test_partition_of_unity_grid():
    xs = np.linspace(-1, 1, 6)
    keys = np.array(np.meshgrid(xs, xs, xs)).reshape(3, -1).T
    q = np.random.RandomState(7).uniform(-0.8, 0.8, (30, 3))
    s = row_sums(natinterp3d.get_weights(q, keys))
    inside = s > 0.5
    assert inside.sum() > 20
    np.testing.assert_allclose(s[inside], 1.0, atol=1e-10)


@pytest.mark.parametrize('parallel', [True, False])
def test_non_negative(parallel):
    rng = np.random.RandomState(99)
    keys = rng.randn(300, 3)
    W = natinterp3d.get_weights(near_centre(keys, 80, rng), keys, parallel=parallel)
    assert W.min() >= -1e-12


@pytest.fixture(scope='module')
def linear_case():
    rng = np.random.RandomState(12)
    keys = rng.randn(500, 3)
    q = near_centre(keys, 60, rng)
    W = natinterp3d.get_weights(q, keys)
    return keys, q, W, row_sums(W) > 0.5


def test_reproduces_constants(linear_case):
    keys, q, W, inside = linear_case
    r = np.asarray(W @ np.full((len(keys), 1), 7.0)).ravel()
    np.testing.assert_allclose(r[inside], 7.0, atol=1e-10)


def test_reproduces_affine_function(linear_case):
    keys, q, W, inside = linear_case
    a, b = np.array([2.0, -3.0, 5.0]), 1.0
    r = np.asarray(W @ (keys @ a + b)[:, None]).ravel()
    np.testing.assert_allclose(r[inside], (q @ a + b)[inside], atol=1e-8)


def test_reproduces_each_coordinate(linear_case):
    keys, q, W, inside = linear_case
    for d in range(3):
        r = np.asarray(W @ keys[:, d:d + 1]).ravel()
        np.testing.assert_allclose(r[inside], q[inside, d], atol=1e-8)


def test_weighted_key_positions_give_the_query():
    rng = np.random.RandomState(55)
    keys = rng.randn(300, 3)
    q = near_centre(keys, 40, rng)
    W = natinterp3d.get_weights(q, keys)
    inside = row_sums(W) > 0.5
    err = np.linalg.norm(np.asarray(W @ keys)[inside] - q[inside], axis=1)
    np.testing.assert_allclose(err, 0.0, atol=1e-8)


def test_error_falls_with_key_density():
    rng = np.random.RandomState(10)

    def f(x):
        return np.sin(x[:, 0]) + np.cos(x[:, 1]) + 0.5 * x[:, 2]

    q = rng.randn(100, 3) * 0.3
    errs = []
    for n in (200, 2000, 20000):
        keys = rng.randn(n, 3)
        errs.append(np.mean(np.abs(natinterp3d.interpolate(q, keys, f(keys)) - f(q))))
    assert errs[1] < errs[0] and errs[2] < errs[1]
    assert errs[2] < 2e-3


# ---- known geometric configurations ------------------------------------------

def test_cube_centre():
    keys = np.array([[-1, -1, -1], [-1, -1, 1], [-1, 1, -1], [-1, 1, 1],
                     [1, -1, -1], [1, -1, 1], [1, 1, -1], [1, 1, 1]], np.float64)
    w = np.asarray(natinterp3d.get_weights(np.zeros((1, 3)), keys).todense()).ravel()
    np.testing.assert_allclose(w, 1 / 8, atol=1e-4)


def test_regular_tetrahedron_centroid():
    keys = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], np.float64)
    w = np.asarray(natinterp3d.get_weights(keys.mean(axis=0, keepdims=True), keys).todense()).ravel()
    np.testing.assert_allclose(w, 0.25, atol=1e-10)


def test_octahedron_centre():
    keys = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float64)
    w = np.asarray(natinterp3d.get_weights(np.zeros((1, 3)), keys).todense()).ravel()
    np.testing.assert_allclose(w, 1 / 6, atol=1e-4)


def test_query_on_a_data_point():
    keys = np.random.RandomState(33).randn(50, 3)
    for idx in (0, 10, 25, 49):
        w = np.asarray(natinterp3d.get_weights(keys[idx:idx + 1], keys).todense()).ravel()
        assert w[idx] == pytest.approx(1.0, abs=1e-4)
        np.testing.assert_allclose(np.delete(w, idx), 0.0, atol=1e-4)


def test_interpolation_on_a_data_point():
    rng = np.random.RandomState(34)
    keys, values = rng.randn(50, 3), rng.randn(50)
    for idx in (0, 25, 49):
        r = natinterp3d.interpolate(keys[idx:idx + 1], keys, values)
        np.testing.assert_allclose(r[0], values[idx], atol=1e-3)


# ---- outside the hull, tiny and rescaled key sets ----------------------------

def test_far_queries_get_no_weights():
    keys = np.random.RandomState(20).randn(100, 3)
    s = row_sums(natinterp3d.get_weights(np.array([[100.0] * 3, [-100.0] * 3]), keys))
    np.testing.assert_allclose(s, 0.0, atol=1e-15)


def test_outside_query_is_finite():
    rng = np.random.RandomState(21)
    keys = rng.randn(100, 3)
    r = natinterp3d.interpolate(np.array([[100.0] * 3]), keys, rng.randn(100) + 10.0)
    assert np.all(np.isfinite(r))


@pytest.mark.parametrize('keys,q', [
    (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0.5, 0.5]], np.float64),
     np.array([[0.2, 0.2, 0.2]])),
    (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float64), np.array([[0.1, 0.1, 0.1]])),
])
def test_minimal_key_sets(keys, q):
    w = np.asarray(natinterp3d.get_weights(q, keys).todense()).ravel()
    assert w.sum() == pytest.approx(1.0, abs=1e-8)
    assert np.all(w >= -1e-12)


def test_single_query_shapes():
    rng = np.random.RandomState(77)
    keys = rng.randn(50, 3)
    q = np.zeros((1, 3))
    assert natinterp3d.get_weights(q, keys).shape == (1, 50)
    assert natinterp3d.interpolate(q, keys, rng.randn(50)).shape == (1,)


@pytest.mark.parametrize('seed,shift,scale', [(88, [1e6, -2e6, 3e6], 1.0), (89, 0.0, 1e4),
                                               (90, 0.0, 1e-4)])
def test_offsets_and_scales(seed, shift, scale):
    rng = np.random.RandomState(seed)
    keys = rng.randn(200, 3) * scale + np.asarray(shift)
    s = row_sums(natinterp3d.get_weights(near_centre(keys, 30, rng), keys))
    inside = s > 0.5
    assert inside.sum() > 15
    np.testing.assert_allclose(s[inside], 1.0, atol=1e-6)


# ---- API --------------------------------------------------------------------

@pytest.fixture(scope='module')
def api_data():
    rng = np.random.RandomState(1)
    return rng.randn(100, 3), rng.randn(50, 3) * 0.3


def test_value_shapes(api_data):
    keys, q = api_data
    assert natinterp3d.interpolate(q, keys, np.ones(100)).shape == (50,)
    assert natinterp3d.interpolate(q, keys, np.ones((100, 5))).shape == (50, 5)


def test_weight_matrix_type_and_shape(api_data):
    keys, q = api_data
    W = natinterp3d.get_weights(q, keys)
    assert isinstance(W, scipy.sparse.csr_matrix) and W.shape == (50, 100)


def test_parallel_flags_do_not_change_results():
    rng = np.random.RandomState(2)
    keys, q = rng.randn(200, 3), rng.randn(80, 3) * 0.3
    a = natinterp3d.get_weights(q, keys, parallel=True).toarray()
    b = natinterp3d.get_weights(q, keys, parallel=False).toarray()
    c = natinterp3d.get_weights(q, keys, parallel=True, num_threads=1).toarray()
    d = natinterp3d.get_weights(q, keys, parallel=True, num_threads=4).toarray()
    np.testing.assert_allclose(a, b, atol=1e-12)
    np.testing.assert_allclose(c, b, atol=1e-12)
    np.testing.assert_allclose(d, b, atol=1e-12)
    v = rng.randn(200)
    np.testing.assert_allclose(natinterp3d.interpolate(q, keys, v, parallel=True),
                               natinterp3d.interpolate(q, keys, v, parallel=False), atol=1e-12)


def test_interpolator_reuse():
    rng = np.random.RandomState(5)
    keys = rng.randn(100, 3)
    it = natinterp3d.Interpolator(keys)
    q1, q2 = rng.randn(20, 3) * 0.3, rng.randn(30, 3) * 0.3
    a = it.get_weights(q1)
    assert it.get_weights(q2).shape == (30, 100)
    np.testing.assert_allclose(a.toarray(), it.get_weights(q1).toarray(), atol=1e-15)
    v = rng.randn(100)
    np.testing.assert_allclose(it.interpolate(q1, v), it.interpolate(q1, v), atol=1e-15)


def test_float32_inputs():
    rng = np.random.RandomState(50)
    keys = rng.randn(100, 3).astype(np.float32)
    q = (rng.randn(20, 3) * 0.3).astype(np.float32)
    r = natinterp3d.interpolate(q, keys, rng.randn(100).astype(np.float32))
    assert r.dtype in (np.float32, np.float64) and r.shape == (20,)
    rng = np.random.RandomState(51)
    keys = rng.randn(100, 3).astype(np.float32)
    q = (rng.randn(20, 3) * 0.3).astype(np.float32)
    W = natinterp3d.get_weights(q, keys)
    assert W.shape == (20, 100)
    s = row_sums(W)
    np.testing.assert_allclose(s[s > 0.5], 1.0, atol=1e-6)


def test_module_functions_match_interpolator():
    rng = np.random.RandomState(60)
    keys, q, v = rng.randn(100, 3), rng.randn(20, 3) * 0.3, rng.randn(100)
    np.testing.assert_allclose(natinterp3d.interpolate(q, keys, v, parallel=False),
                               natinterp3d.Interpolator(keys, parallel=False).interpolate(q, v),
                               atol=1e-15)
    rng = np.random.RandomState(61)
    keys, q = rng.randn(100, 3), rng.randn(20, 3) * 0.3
    np.testing.assert_allclose(natinterp3d.get_weights(q, keys, parallel=False).toarray(),
                               natinterp3d.Interpolator(keys, parallel=False).get_weights(q).toarray(),
                               atol=1e-15)


@pytest.mark.parametrize('seed,parallel', [(70, True), (71, False)])
def test_deterministic(seed, parallel):
    rng = np.random.RandomState(seed)
    keys, q = rng.randn(200, 3), rng.randn(50, 3) * 0.3
    np.testing.assert_array_equal(natinterp3d.get_weights(q, keys, parallel=parallel).toarray(),
                                  natinterp3d.get_weights(q, keys, parallel=parallel).toarray())


def test_rows_are_sparse():
    rng = np.random.RandomState(80)
    keys, q = rng.randn(1000, 3), rng.randn(50, 3) * 0.3
    W = natinterp3d.get_weights(q, keys)
    assert np.diff(W.indptr).max() < 100


def test_original_regression():
    rng = np.random.RandomState(10)
    keys = rng.randn(10000, 3)

    def f(x):
        x = x * 0.1
        return np.sin(x[:, 0]) + np.cos(x[:, 1]) + np.tan(x[:, 2])

    q = rng.randn(100, 3)
    assert np.mean(np.abs(natinterp3d.interpolate(q, keys, f(keys)) - f(q))) < 1e-3


def test_bad_shapes_raise_value_error():
    keys = np.random.RandomState(0).randn(20, 3)
    with pytest.raises(ValueError):
        natinterp3d.Interpolator(keys[:, :2])
    it = natinterp3d.Interpolator(keys)
    with pytest.raises(ValueError):
        it.get_weights(np.zeros((4, 2)))
