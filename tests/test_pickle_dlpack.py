"""Interpolator pickling (the packed mesh travels, the device copy is rebuilt)
and the DLPack export of the device CSR."""
import pickle

import numpy as np
import pytest

import natinterp3d_b200 as ni


def _interp(seed=0, n=800):
    rng = np.random.default_rng(seed)
    return ni.Interpolator(rng.uniform(0, 1, (n, 3)), predicates='audit'), rng


def test_pickle_round_trip_keeps_the_mesh():
    it, _ = _interp()
    it2 = pickle.loads(pickle.dumps(it))
    assert np.array_equal(it2.centroid, it.centroid)
    for a, b in zip(it.mesh_arrays, it2.mesh_arrays):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    assert it2.n_keys == it.n_keys and it2.predicates == 'audit'
    assert it2.degeneracies == it.degeneracies


def test_unknown_pickle_format_is_rejected():
    it, _ = _interp()
    state = it.__getstate__()
    state['format'] = 99
    fresh = ni.Interpolator.__new__(ni.Interpolator)
    with pytest.raises(ValueError):
        fresh.__setstate__(state)


@pytest.mark.gpu
def test_pickle_round_trip_weights_bit_identical(cuda_device):
    it, rng = _interp(1, 3000)
    q = rng.uniform(0.05, 0.95, (20_000, 3))
    W = it.get_weights(q)  # builds the device mesh before pickling
    it.set_tuning({'blocks_per_sm': 6, 'bucket_shift': 0, 'tile': 4})
    it2 = pickle.loads(pickle.dumps(it))
    W2 = it2.get_weights(q)
    assert np.array_equal(W.indptr, W2.indptr) and np.array_equal(W.indices, W2.indices)
    assert np.array_equal(W.data.view(np.uint8), W2.data.view(np.uint8))
    assert it2.tuning == {'blocks_per_sm': 6, 'bucket_shift': 0, 'tile': 4}


@pytest.mark.gpu
def test_dlpack_export_is_the_device_csr(cuda_device):
    import torch
    it, rng = _interp(2, 2000)
    q = torch.from_numpy(rng.uniform(0.05, 0.95, (5000, 3))).to(cuda_device)
    caps = it.get_weights_dlpack(q)
    rowptr, cols, vals = (torch.from_dlpack(c) for c in caps)
    assert rowptr.device == q.device and rowptr.dtype == torch.int32 and cols.dtype == torch.int32
    W = it.get_weights(q.cpu().numpy())
    assert np.array_equal(rowptr.cpu().numpy(), W.indptr)
    assert np.array_equal(cols.cpu().numpy(), W.indices)
    assert np.array_equal(vals.cpu().numpy(), W.data)
