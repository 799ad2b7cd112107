"""GPU tests of the launch settings (nif_tuning) and the autotuner: every
setting gives bit-identical results (tolerance 0) on the plain, weights,
batched and allocation-free paths; invalid settings are rejected; the
autotuner keeps a candidate and caches it."""
import ctypes

import numpy as np
import pytest
import torch

import natinterp3d_b200 as ni
from natinterp3d_b200 import _native as N
from natinterp3d_b200 import tuning
from natinterp3d_b200.batch import BatchInterpolator
from natinterp3d_b200.device import _DT, _stream_ptr, _vp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def case(cuda_device):
    rng = np.random.default_rng(11)
    keys = rng.uniform(0, 1, (20000, 3))
    q = rng.uniform(0.02, 0.98, (150000, 3))
    v = rng.standard_normal((20000, 3)).astype(np.float32)
    I = ni.Interpolator(keys, device=cuda_device)
    qd = torch.from_numpy(q).to(cuda_device)
    vd = torch.from_numpy(v).to(cuda_device)
    return I, qd, vd


def test_default_tuning(case):
    I, _, _ = case
    assert I.tuning == {'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 8}


@pytest.mark.parametrize('cand', tuning.MESH_CANDIDATES + [
    {'blocks_per_sm': 6, 'tile': 1, 'bucket_shift': -2},
    {'blocks_per_sm': 8, 'tile': 1024, 'bucket_shift': 1}])
def test_every_setting_gives_identical_results(case, cand):
    I, qd, vd = case
    I.set_tuning({'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 8})
    ref_out = I.interpolate_device(qd, vd)
    ref_w = I.get_weights_device(qd)
    I.set_tuning(cand)
    assert I.tuning == cand
    out = I.interpolate_device(qd, vd)
    w = I.get_weights_device(qd)
    I.set_tuning({'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 8})
    assert torch.equal(out, ref_out)
    for a, b in zip(w, ref_w):
        assert torch.equal(a, b)


@pytest.mark.parametrize('bad', [
    {'blocks_per_sm': 7, 'tile': 0, 'bucket_shift': 0},
    {'blocks_per_sm': 8, 'tile': -1, 'bucket_shift': 0},
    {'blocks_per_sm': 8, 'tile': 1025, 'bucket_shift': 0},
    {'blocks_per_sm': 8, 'tile': 0, 'bucket_shift': 2},
    {'blocks_per_sm': 8, 'tile': 0, 'bucket_shift': -3}])
def test_invalid_settings_rejected(case, bad):
    I, _, _ = case
    before = I.tuning
    with pytest.raises(ValueError):
        I.set_tuning(bad)
    assert I.tuning == before


def test_workspace_size_does_not_depend_on_tuning(case):
    I, qd, _ = case
    dm = I.device_mesh
    sizes = set()
    for s in (-2, 0, 1):
        I.set_tuning({'blocks_per_sm': 8, 'tile': 0, 'bucket_shift': s})
        sizes.add(dm.workspace_bytes(qd.shape[0], N.NIF_MODE_WEIGHTS))
    I.set_tuning({'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 8})
    assert len(sizes) == 1


def test_noalloc_follows_tuning_with_capped_buckets(case):
    I, qd, vd = case
    dm = I.device_mesh
    lib = N.cuda_lib()
    M = 100000
    q = qd[:M].contiguous()
    ref = I.interpolate_device(q, vd)
    cen = (ctypes.c_double * 3)(*[float(c) for c in I.centroid])
    for cand in ({'blocks_per_sm': 6, 'tile': 32, 'bucket_shift': 1},
                 {'blocks_per_sm': 8, 'tile': 8, 'bucket_shift': -1}):
        I.set_tuning(cand)
        out = torch.empty_like(ref)
        summ = N.Summary()
        N.check(lib.nif_interpolate_noalloc(dm._h, _vp(q), _DT[q.dtype], M, cen, _vp(vd),
                                            _DT[vd.dtype], 3, _vp(out), _DT[out.dtype],
                                            _stream_ptr(dm.device), ctypes.byref(summ)),
                'nif_interpolate_noalloc')
        assert summ.rows_failed == 0
        assert torch.equal(out, ref)
    I.set_tuning({'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 8})


def test_autotuner_keeps_a_candidate_and_caches_it(case, tmp_path, monkeypatch):
    I, qd, vd = case
    monkeypatch.setenv('NATINTERP3D_B200_TUNING', str(tmp_path / 'tuning.json'))
    ref = I.interpolate_device(qd, vd)
    rep = I.tune(qd, vd, reps=1)
    assert not rep['cached'] and rep['tuning'] in tuning.MESH_CANDIDATES
    assert len(rep['times_ms']) == len(tuning.MESH_CANDIDATES)
    assert I.tuning == rep['tuning']
    assert torch.equal(I.interpolate_device(qd, vd), ref)
    I.set_tuning({'blocks_per_sm': 6, 'bucket_shift': 1, 'tile': 32})
    rep2 = I.tune(qd, vd)
    assert rep2['cached'] and rep2['tuning'] == rep['tuning'] and I.tuning == rep['tuning']
    rep3 = I.tune(qd, mode='weights', reps=1, candidates=tuning.MESH_CANDIDATES[:3])
    assert rep3['tuning'] in tuning.MESH_CANDIDATES[:3]
    I.set_tuning({'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 8})


def test_batch_settings_and_tuner(cuda_device, tmp_path, monkeypatch):
    monkeypatch.setenv('NATINTERP3D_B200_TUNING', str(tmp_path / 'tuning.json'))
    rng = np.random.default_rng(5)
    keys = [rng.uniform(0, 1, (n, 3)) + i for i, n in enumerate((300, 2500, 900, 4000))]
    qs = [k.min(0) + 0.1 + 0.8 * rng.uniform(0, 1, (m, 3)) * (k.max(0) - k.min(0))
          for k, m in zip(keys, (700, 3000, 50, 9000))]
    vals = [rng.standard_normal((k.shape[0], 2)).astype(np.float32) for k in keys]
    b = BatchInterpolator(keys, device=cuda_device)
    assert b.get_tuning() == {'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 64}
    qoff = b.query_offsets([len(q) for q in qs])
    qcat = torch.from_numpy(np.concatenate(qs)).to(cuda_device)
    vcat = torch.from_numpy(np.concatenate(vals)).to(cuda_device)
    ref = b.interpolate_per_problem(qcat, qoff, vcat)
    for cand in tuning.BATCH_CANDIDATES + [{'blocks_per_sm': 6, 'tile': 1, 'bucket_shift': 0}]:
        b.set_tuning(cand)
        assert torch.equal(b.interpolate_device(qcat, qoff, vcat), ref)
    with pytest.raises(ValueError):
        b.set_tuning({'blocks_per_sm': 8, 'tile': 0, 'bucket_shift': 0})
    rep = b.tune(qcat, qoff, vcat, reps=1)
    assert rep['tuning'] in tuning.BATCH_CANDIDATES and b.get_tuning() == rep['tuning']
    assert torch.equal(b.capture(qcat, qoff, vcat).replay(), ref)
