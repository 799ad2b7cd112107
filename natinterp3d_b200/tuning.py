"""Autotuner of the query kernels' launch settings (``nif_tuning``).

The settings change speed only: every candidate gives bit-identical output,
and :func:`tune` checks that on its sample before keeping a winner.  For one
mesh (``Interpolator``) the candidates are

  blocks_per_sm  6 or 8      resident 4-warp blocks per SM of the
                             one-warp-per-query row kernel (80 or 64
                             registers a thread)
  tile           0, 8, 32    static grid stride, or tiles of 8 / 32
                             consecutive bucket-ordered queries a warp pulls
                             from a device counter
  bucket_shift   -1, 0, 1    Morton bucket resolution of the query order,
                             in bits per axis relative to the size default

and for a batch (``BatchInterpolator``) blocks_per_sm 6 or 8 times tiles of
16, 32, 64 or 128 queries.  Each candidate runs once untimed, then ``reps``
times between CUDA events on the current stream; the smallest time wins.

Lanes per query stay at one warp.  Groups of 16 or 8 lanes (two or four
queries per warp) diverge between their queries' control flow and ran
0.62x and 0.32x as fast as one warp per query on the 1M-key / 10M-query
interpolation workload, so they are not candidates.  The shared-memory
capacities of the fast kernel (tested-tet hash 256, cavity 96, boundary
faces 128, neighbours 64) are fixed: at 8 blocks per SM registers, not
shared memory, limit residency, and rows beyond them go to the large-row
kernel whatever their size.

Results are cached per (GPU name, mode, key count, query count, dtypes,
value columns, predicate mode) in a JSON file (``NATINTERP3D_B200_TUNING``,
default ``~/.cache/natinterp3d_b200/tuning.json``); counts are rounded to
powers of two.
"""
import itertools
import json
import math
import os

import numpy as np
import torch

__all__ = ['MESH_CANDIDATES', 'BATCH_CANDIDATES', 'tune', 'tune_batch', 'cache_path']

MESH_CANDIDATES = [{'blocks_per_sm': b, 'tile': t, 'bucket_shift': s}
                   for b, t, s in itertools.product((8, 6), (8, 0, 32), (0, -1, 1))]
BATCH_CANDIDATES = [{'blocks_per_sm': b, 'tile': t, 'bucket_shift': 0}
                    for b, t in itertools.product((8, 6), (64, 16, 32, 128))]


def cache_path():
    return os.environ.get('NATINTERP3D_B200_TUNING',
                          os.path.join(os.path.expanduser('~'), '.cache', 'natinterp3d_b200',
                                       'tuning.json'))


def _load_cache():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(key, entry):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = _load_cache()
        data[key] = entry
        tmp = path + '.tmp%d' % os.getpid()
        with open(tmp, 'w') as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache only costs a re-tune


def _p2(n):
    return 0 if n <= 0 else int(round(math.log2(n)))


def _time(fn, reps):
    fn()  # untimed: first launch of an instantiation queries its occupancy
    torch.cuda.synchronize()
    best = float('inf')
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _same(a, b):
    if isinstance(a, tuple):
        return all(torch.equal(x, y) for x, y in zip(a, b))
    return torch.equal(a, b)


def _search(candidates, apply, run, reps):
    """Times every candidate; returns (best, report).  Raises if any candidate's
    output differs from the first one's."""
    ref = None
    report = []
    for cand in candidates:
        apply(cand)
        out = run()
        torch.cuda.synchronize()
        if ref is None:
            ref = out
        elif not _same(ref, out):
            raise RuntimeError('launch setting %r changed the results' % (cand,))
        report.append((cand, _time(run, reps)))
    best = min(report, key=lambda r: r[1])[0]
    apply(best)
    return best, report


def tune(interp, query_points, values=None, mode='interpolate', max_queries=2_000_000, reps=3,
         candidates=None, use_cache=True):
    """Pick the fastest launch settings of ``interp``'s query kernels for
    queries like ``query_points`` and set them on the interpolator.

    mode 'interpolate' times ``interpolate_device(q, values)`` (values: the
    caller's value array, or random float32 columns when None); mode
    'weights' times ``get_weights_device(q)``.  At most ``max_queries``
    evenly strided queries of the input are used.  Returns
    ``{'tuning': best, 'times_ms': [(candidate, ms), ...], 'cached': bool}``.
    """
    if mode not in ('interpolate', 'weights'):
        raise ValueError("mode must be 'interpolate' or 'weights'")
    dm = interp.device_mesh
    q = query_points if isinstance(query_points, torch.Tensor) else \
        torch.from_numpy(np.ascontiguousarray(query_points))
    if q.dtype not in (torch.float32, torch.float64):
        q = q.to(torch.float64)
    q = q.reshape(-1, 3)
    M_full = int(q.shape[0])
    if M_full == 0:
        return {'tuning': dm.get_tuning(), 'times_ms': [], 'cached': False}
    step = max(1, -(-M_full // max_queries))
    q = q[::step].contiguous().to(dm.device)
    if mode == 'interpolate':
        if values is None:
            v = torch.randn(interp.n_keys, 1, dtype=torch.float32, device=dm.device)
        else:
            v = values if isinstance(values, torch.Tensor) else torch.from_numpy(np.asarray(values))
            v = v.reshape(interp.n_keys, -1).contiguous().to(dm.device)
        run = lambda: interp.interpolate_device(q, v, check=False)  # noqa: E731
        vdesc = '%s/D%d' % (str(v.dtype).replace('torch.', ''), v.shape[1])
    else:
        run = lambda: interp.get_weights_device(q)  # noqa: E731
        vdesc = '-'
    key = '|'.join([torch.cuda.get_device_name(dm.device), mode, 'k2^%d' % _p2(interp.n_keys),
                    'q2^%d' % _p2(M_full), str(q.dtype).replace('torch.', ''), vdesc,
                    interp.predicates])
    if use_cache and candidates is None:
        hit = _load_cache().get(key)
        if hit is not None:
            interp.set_tuning(hit['tuning'])
            return {'tuning': hit['tuning'], 'times_ms': hit.get('times_ms', []), 'cached': True}
    with torch.cuda.device(dm.device):
        best, report = _search(candidates or MESH_CANDIDATES, interp.set_tuning, run, reps)
    entry = {'tuning': best, 'times_ms': [(c, round(t, 3)) for c, t in report],
             'sample_queries': int(q.shape[0])}
    if use_cache and candidates is None:
        _store_cache(key, entry)
    return {'tuning': best, 'times_ms': entry['times_ms'], 'cached': False}


def tune_batch(batch, queries, query_offsets, values, reps=3, candidates=None, use_cache=True):
    """Pick the fastest launch settings of ``batch``'s persistent row kernel for
    these inputs (all problems, as passed to ``interpolate_device``) and set
    them on the batch.  Returns the same report as :func:`tune`."""
    qoff = np.asarray(query_offsets.cpu().numpy() if isinstance(query_offsets, torch.Tensor)
                      else query_offsets, np.int64)
    v = values.reshape(values.shape[0], -1)
    key = '|'.join([torch.cuda.get_device_name(batch.device), 'batch', 'P%d' % batch.P,
                    'k2^%d' % _p2(int(batch.n_keys.sum())), 'q2^%d' % _p2(int(qoff[-1])),
                    str(queries.dtype).replace('torch.', ''),
                    '%s/D%d' % (str(values.dtype).replace('torch.', ''), v.shape[1])])
    if use_cache and candidates is None:
        hit = _load_cache().get(key)
        if hit is not None:
            batch.set_tuning(hit['tuning'])
            return {'tuning': hit['tuning'], 'times_ms': hit.get('times_ms', []), 'cached': True}
    run = lambda: batch.interpolate_device(queries, query_offsets, values, check=False)  # noqa: E731
    with torch.cuda.device(batch.device):
        best, report = _search(candidates or BATCH_CANDIDATES, batch.set_tuning, run, reps)
    entry = {'tuning': best, 'times_ms': [(c, round(t, 3)) for c, t in report]}
    if use_cache and candidates is None:
        _store_cache(key, entry)
    return {'tuning': best, 'times_ms': entry['times_ms'], 'cached': False}
