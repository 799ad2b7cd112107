"""Parity on two north-star workloads at their full sizes, against
natinterp3d's own code and the oracle:

* interpolate at scale: 1,000,000 keys uniform in [0,1]^3, 10,000,000
  queries uniform in [0.02,0.98]^3, values D=3 float32 N(0,1), seed 1 (the
  benchmark's default workload).  The first 2,000,000 rows of ``get_weights``
  are compared bit for bit with natinterp3d's own query code
  (getInsertionFreeWeightsParallel) run on the same mesh object, and the
  interpolation of all 10M rows -- through the chunked host pipeline -- with
  those rows' ``W @ values``; over all 10M rows the weights sum to one and an
  affine field is reproduced.
* uneven batch: the benchmark's 512 problems (keys log-uniform in [500, 100k],
  queries log-uniform in [1k, 200k], values D=4 float32, seed 4), all solved
  in one batched launch; every 16th problem's rows are compared bit for bit
  with the oracle's ``W @ values`` on that problem's mesh.
"""
import argparse
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

import bench
import natinterp3d_b200 as ni
from natinterp3d_b200.batch import BatchInterpolator
from oracle import oracle

pytestmark = pytest.mark.gpu


def _bitwise_csr(A, B):
    assert np.array_equal(A.indptr, B.indptr), 'row pointers differ'
    assert np.array_equal(A.indices, B.indices), 'column order differs'
    assert np.array_equal(np.asarray(A.data).view(np.uint8), np.asarray(B.data).view(np.uint8))


def _threads():
    return len(os.sched_getaffinity(0))


@pytest.mark.skipif(not oracle.ref_available(), reason="natinterp3d's query library not built")
def test_interpolate_at_scale_against_natinterp3d(cuda_device):
    args = argparse.Namespace(keys=1_000_000, queries=10_000_000, dim=3, seed=1)
    keys, queries, values = bench.make_data(args)
    interp = ni.Interpolator(keys, device=cuda_device, keep_host_mesh=True)
    c = interp.centroid
    n_cmp = 2_000_000
    W = interp.get_weights(queries[:n_cmp])
    Wr = oracle.ref_query(interp.host_mesh.native_pointer(), queries[:n_cmp] - c, keys.shape[0],
                          _threads())
    _bitwise_csr(W, Wr)
    # all 10M rows through the host pipeline (chunked uploads and downloads)
    out = interp.interpolate(queries, values)
    assert out.dtype == np.float64 and out.shape == (queries.shape[0], 3)
    assert np.array_equal(out[:n_cmp], Wr @ values)
    del W, Wr
    # size-independent properties over every row
    qd = torch.from_numpy(queries).to(cuda_device)
    ones = torch.ones(keys.shape[0], dtype=torch.float64, device=cuda_device)
    s, summ = interp.device_mesh.interpolate(qd, ones, c, return_summary=True)
    assert summ['rows_failed'] == 0 and summ['rows_outside'] == 0
    assert torch.abs(s - 1).max().item() < 1e-12
    a, b = np.array([0.3, -1.2, 2.0]), 0.7
    vx = interp.mesh_arrays[0][:keys.shape[0]] + c
    f = torch.from_numpy(vx @ a + b).to(cuda_device)
    lin = interp.interpolate_device(qd, f).cpu().numpy()
    deep = np.all((queries > 0.05) & (queries < 0.95), axis=1)
    assert np.abs(lin - (queries @ a + b))[deep].max() < 1e-12


def test_uneven_batch_against_oracle(cuda_device):
    keys, queries, values = bench.batched_workload(512, 4)
    b = BatchInterpolator(keys, device=cuda_device)
    qoff = b.query_offsets([len(q) for q in queries])
    qcat = torch.from_numpy(np.concatenate(queries)).to(cuda_device)
    vcat = torch.from_numpy(np.concatenate(values)).to(cuda_device)
    # one batched launch for all 512 problems; raises if any row failed
    out = b.interpolate_device(qcat, qoff, vcat).cpu().numpy()
    sample = list(range(0, 512, 16))

    def check(p):
        it = b.interpolators[p]
        W = oracle.OracleMesh(*it.mesh_arrays).weights(queries[p] - it.centroid)
        return p, np.array_equal(out[qoff[p]:qoff[p + 1]], W @ values[p])

    with ThreadPoolExecutor(min(len(sample), _threads())) as ex:
        results = list(ex.map(check, sample))
    bad = [p for p, ok in results if not ok]
    assert not bad, 'problems differing from the oracle: %r' % bad
