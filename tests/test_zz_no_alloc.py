"""The allocation-free interpolation entry point, nif_interpolate_noalloc.

Some callers cannot give this library device memory: a serving process whose
GPU memory is already owned by another pool, or a latency-critical loop in
which an allocation could fail or stall the whole device.  For them the C ABI
offers one interpolation call whose scratch is a fixed array compiled into
libnif_cuda.so.  This test drives that call directly through ctypes, twice in
a row on the same inputs (the second call reuses the scratch the first one
left behind), and requires both results to equal, bit for bit, those of the
regular workspace-based nif_interpolate -- the same zero tolerance the other
parity tests use.  It builds its own mesh and data, so it passes both in a
fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest
import torch

from natinterp3d_b200 import _native as N
from natinterp3d_b200._native import HostMesh
from natinterp3d_b200.device import DeviceMesh

pytestmark = pytest.mark.gpu

MAX_QUERIES = 1 << 20  # NIF_NOALLOC_MAX_QUERIES in include/natinterp3d_b200.h


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _call_noalloc(dm, q, v, centroid, out, summary=None):
    lib = N.cuda_lib()
    cen = (ctypes.c_double * 3)(*[float(c) for c in centroid])
    qdt = N.NIF_F32 if q.dtype == torch.float32 else N.NIF_F64
    vdt = N.NIF_F32 if v.dtype == torch.float32 else N.NIF_F64
    odt = N.NIF_F32 if out.dtype == torch.float32 else N.NIF_F64
    stream = ctypes.c_void_p(torch.cuda.current_stream(dm.device).cuda_stream)
    return lib.nif_interpolate_noalloc(dm._h, _vp(q), qdt, int(q.shape[0]), cen, _vp(v), vdt,
                                       int(v.shape[1]), _vp(out), odt, stream,
                                       ctypes.byref(summary) if summary is not None else None)


@pytest.fixture(scope='module')
def noalloc_mesh(cuda_device):
    rng = np.random.default_rng(11)
    keys = rng.uniform(0.0, 1.0, (20000, 3))
    c = keys.mean(axis=0)
    dm = DeviceMesh(*HostMesh(keys - c).export(), device=cuda_device)
    return dm, c, rng


def _out_dtype(q, v):
    return torch.float32 if (q.dtype == torch.float32 and v.dtype == torch.float32) else torch.float64


@pytest.mark.parametrize('query_dtype', [torch.float32, torch.float64])
@pytest.mark.parametrize('values_dtype', [torch.float32, torch.float64])
def test_noalloc_matches_workspace_entry_point_twice(query_dtype, values_dtype, noalloc_mesh,
                                                     cuda_device):
    dm, c, rng = noalloc_mesh
    q = torch.from_numpy(rng.uniform(0.02, 0.98, (60000, 3))).to(cuda_device, query_dtype)
    v = torch.from_numpy(rng.standard_normal((20000, 3))).to(cuda_device, values_dtype)
    expect = dm.interpolate(q, v, c).cpu().numpy()
    for _ in range(2):
        out = torch.full((q.shape[0], 3), float('nan'), dtype=_out_dtype(q, v), device=cuda_device)
        summ = N.Summary()
        assert _call_noalloc(dm, q, v, c, out, summ) == N.NIF_OK
        assert summ.rows_failed == 0
        got = out.cpu().numpy()
        assert np.array_equal(got, expect), np.nanmax(np.abs(got - expect))


def test_noalloc_empty_call(noalloc_mesh, cuda_device):
    dm, c, _ = noalloc_mesh
    q = torch.empty((0, 3), dtype=torch.float64, device=cuda_device)
    v = torch.zeros((20000, 2), dtype=torch.float64, device=cuda_device)
    out = torch.empty((1, 2), dtype=torch.float64, device=cuda_device)
    summ = N.Summary()
    assert _call_noalloc(dm, q, v, c, out, summ) == N.NIF_OK
    assert summ.rows_failed == 0 and summ.walk_steps == 0


def test_noalloc_with_finer_bucketing(noalloc_mesh, cuda_device):
    # a positive bucket_shift asks for more buckets than the fixed scratch
    # holds; the call caps it and still returns the same bits
    dm, c, rng = noalloc_mesh
    q = torch.from_numpy(rng.uniform(0.02, 0.98, (300000, 3))).to(cuda_device)
    v = torch.from_numpy(rng.standard_normal((20000, 1))).to(cuda_device)
    expect = dm.interpolate(q, v, c).cpu().numpy()
    old = dm.get_tuning()
    dm.set_tuning({'blocks_per_sm': 6, 'bucket_shift': 1, 'tile': 16})
    try:
        for _ in range(2):
            out = torch.full((q.shape[0], 1), float('nan'), dtype=torch.float64, device=cuda_device)
            assert _call_noalloc(dm, q, v, c, out) == N.NIF_OK
            assert np.array_equal(out.cpu().numpy(), expect)
    finally:
        dm.set_tuning(old)


def test_noalloc_at_its_maximum_size(noalloc_mesh, cuda_device):
    dm, c, rng = noalloc_mesh
    q = torch.from_numpy(rng.uniform(0.02, 0.98, (MAX_QUERIES, 3))).to(cuda_device)
    v = torch.from_numpy(rng.standard_normal((20000, 1))).to(cuda_device)
    out = torch.empty((MAX_QUERIES, 1), dtype=torch.float64, device=cuda_device)
    summ = N.Summary()
    assert _call_noalloc(dm, q, v, c, out, summ) == N.NIF_OK
    assert summ.rows_failed == 0
    assert np.array_equal(out.cpu().numpy(), dm.interpolate(q, v, c).cpu().numpy())


def test_noalloc_rejects_batches_beyond_its_fixed_scratch(cuda_device):
    rng = np.random.default_rng(12)
    keys = rng.uniform(0.0, 1.0, (2000, 3))
    c = keys.mean(axis=0)
    dm = DeviceMesh(*HostMesh(keys - c).export(), device=cuda_device)
    v = torch.zeros((2000, 1), dtype=torch.float64, device=cuda_device)
    q = torch.zeros((MAX_QUERIES + 1, 3), dtype=torch.float64, device=cuda_device)
    out = torch.empty((MAX_QUERIES + 1, 1), dtype=torch.float64, device=cuda_device)
    assert _call_noalloc(dm, q, v, c, out) == N.NIF_ERR_TOO_LARGE
