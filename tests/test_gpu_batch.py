"""GPU tests of the batched path: many uneven problems in one pipeline."""
import numpy as np
import pytest
import torch

import natinterp3d_b200 as ni
from natinterp3d_b200.batch import BatchInterpolator

pytestmark = pytest.mark.gpu


def uneven_problems(P, seed, kmin=200, kmax=6000, qmin=50, qmax=4000):
    rng = np.random.default_rng(seed)
    keys, queries = [], []
    for _ in range(P):
        nk = int(np.exp(rng.uniform(np.log(kmin), np.log(kmax))))
        nq = int(np.exp(rng.uniform(np.log(qmin), np.log(qmax))))
        lo = rng.uniform(-3, 3, 3)
        side = rng.uniform(0.5, 2.0, 3)
        keys.append(lo + side * rng.uniform(0, 1, (nk, 3)))
        queries.append(lo + side * (0.025 + 0.95 * rng.uniform(0, 1, (nq, 3))))
    return keys, queries


@pytest.fixture(scope='module')
def batch_case(cuda_device):
    keys, queries = uneven_problems(14, 0)
    b = BatchInterpolator(keys, device=cuda_device)
    rng = np.random.default_rng(1)
    values = [rng.standard_normal((k.shape[0], 4)).astype(np.float32) for k in keys]
    qoff = b.query_offsets([len(q) for q in queries])
    qcat = torch.from_numpy(np.concatenate(queries)).to(cuda_device)
    vcat = torch.from_numpy(np.concatenate(values)).to(cuda_device)
    return b, keys, queries, values, qoff, qcat, vcat


def test_batch_equals_per_problem_calls(batch_case):
    b, keys, queries, values, qoff, qcat, vcat = batch_case
    out = b.interpolate_device(qcat, qoff, vcat)
    ref = b.interpolate_per_problem(qcat, qoff, vcat)
    assert out.dtype == torch.float64 and out.shape == (qcat.shape[0], 4)
    assert torch.equal(out, ref)


def test_batch_equals_independent_interpolators(batch_case):
    b, keys, queries, values, qoff, qcat, vcat = batch_case
    outs = b.interpolate(queries, values)
    for p in (0, 5, 13):
        it = ni.Interpolator.from_mesh(b.interpolators[p].centroid, *b.interpolators[p].mesh_arrays)
        assert np.array_equal(outs[p], it.interpolate(queries[p], values[p]))


def test_graph_replay_matches_eager(batch_case):
    b, keys, queries, values, qoff, qcat, vcat = batch_case
    eager = b.interpolate_device(qcat, qoff, vcat)
    g = b.capture(qcat, qoff, vcat)
    for _ in range(2):
        g.out.zero_()
        out = g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out, eager)
    assert g.summary().rows_failed == 0


def test_batch_float64_scalar_values(cuda_device):
    keys, queries = uneven_problems(5, 2)
    b = BatchInterpolator(keys, device=cuda_device)
    rng = np.random.default_rng(3)
    values = [rng.standard_normal(k.shape[0]) for k in keys]
    outs = b.interpolate(queries, values)
    for p in range(5):
        assert outs[p].shape == (len(queries[p]),)
        assert np.array_equal(outs[p], b.interpolators[p].interpolate(queries[p], values[p]))


@pytest.mark.parametrize('chunk', [1000, 4000])
def test_pipelined_host_batch_matches_single_call(batch_case, monkeypatch, chunk):
    """Host batches above two pipeline chunks go through problem groups on a
    copy stream; the results equal the single-call path bit for bit."""
    import natinterp3d_b200.natinterp3d as api
    b, keys, queries, values, qoff, qcat, vcat = batch_case
    ref = b.interpolate(queries, values)
    monkeypatch.setattr(api, 'PIPELINE_CHUNK', chunk)
    assert qoff[-1] > 2 * chunk
    outs = b.interpolate(queries, values)
    for p in range(b.P):
        assert outs[p].dtype == ref[p].dtype and np.array_equal(outs[p], ref[p])
    scal = [v[:, 0].astype(np.float64) for v in values]
    outs = b.interpolate(queries, scal)
    monkeypatch.setattr(api, 'PIPELINE_CHUNK', 1 << 21)
    ref = b.interpolate(queries, scal)
    for p in range(b.P):
        assert outs[p].shape == (len(queries[p]),) and np.array_equal(outs[p], ref[p])
