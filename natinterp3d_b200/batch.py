"""Many independent Sibson problems at once.

``BatchInterpolator(list_of_key_arrays)`` builds one Delaunay mesh per
problem (natinterp3d's constructor, run on a pool of host threads -- the
constructor is C and releases the GIL), keeps every mesh resident on the GPU
and groups them into one batch.  ``interpolate_device`` then evaluates all
problems in one pipeline with no host synchronisation (bucketing by problem
and Morton cell, one persistent row kernel fed by a device work counter);
``capture`` records that pipeline once as a CUDA graph for fixed shapes and
``BatchGraph.replay`` re-runs it.  Each problem's result is exactly what
``Interpolator(keys_p).interpolate(queries_p, values_p)`` returns.
"""
import ctypes
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _native as N
from .device import _DT, DeviceMesh, _stream_ptr, _vp
from . import natinterp3d as _api
from .natinterp3d import Interpolator

__all__ = ['BatchInterpolator', 'BatchGraph']


class BatchInterpolator:
    """``predicates``: one mode for all problems ('fast', 'audit', 'exact'; see
    :class:`Interpolator`) or a list with one mode per problem."""

    def __init__(self, keys_list, device=None, threads=None, predicates='fast'):
        if not keys_list:
            raise ValueError('need at least one key set')
        threads = threads or min(len(keys_list), len(os.sched_getaffinity(0)))
        keys_list = [np.ascontiguousarray(k, np.float64) for k in keys_list]
        modes = [predicates] * len(keys_list) if isinstance(predicates, str) else list(predicates)
        if len(modes) != len(keys_list):
            raise ValueError('need one predicate mode per problem')
        with ThreadPoolExecutor(max(1, threads)) as ex:
            self.interpolators = list(ex.map(
                lambda km: Interpolator(km[0], device=device, predicates=km[1]),
                zip(keys_list, modes)))
        self.P = len(self.interpolators)
        # the batch records each mesh's predicate mode now (nif_batch_create)
        self.meshes = [it.device_mesh for it in self.interpolators]
        self.device = self.meshes[0].device
        self.n_keys = np.array([m.n_keys for m in self.meshes], np.int64)
        self._lib = N.cuda_lib()
        nb = ctypes.c_size_t()
        N.check(self._lib.nif_batch_bytes(self.P, ctypes.byref(nb)), 'nif_batch_bytes')
        with torch.cuda.device(self.device):
            self._buf = torch.empty(int(nb.value), dtype=torch.uint8, device=self.device)
            handles = (ctypes.c_void_p * self.P)(*[m._h.value for m in self.meshes])
            self._h = ctypes.c_void_p()
            N.check(self._lib.nif_batch_create(self.P, handles, _vp(self._buf), nb.value,
                                               _stream_ptr(self.device), ctypes.byref(self._h)),
                    'nif_batch_create')
            koff = np.zeros(self.P + 1, np.int64)
            koff[1:] = np.cumsum(self.n_keys)
            self.key_offsets = torch.from_numpy(koff).to(self.device)
            cens = np.stack([it.centroid for it in self.interpolators])
            self.centroids = torch.from_numpy(np.ascontiguousarray(cens)).to(self.device)

    # ------------------------------------------------------------------ tuning
    def set_tuning(self, tuning):
        """Launch settings of later batch calls (``blocks_per_sm`` 6 or 8,
        ``tile`` 1..1024 queries per work item; ``bucket_shift`` is ignored).
        A graph captured earlier keeps the settings it was captured with."""
        t = N.Tuning.from_dict(tuning)
        rc = self._lib.nif_batch_set_tuning(self._h, ctypes.byref(t))
        if rc == N.NIF_ERR_ARG:
            raise ValueError('invalid batch tuning %r' % (tuning,))
        N.check(rc, 'nif_batch_set_tuning')

    def get_tuning(self):
        t = N.Tuning()
        N.check(self._lib.nif_batch_get_tuning(self._h, ctypes.byref(t)), 'nif_batch_get_tuning')
        return t.as_dict()

    def tune(self, queries, query_offsets, values, **kw):
        """Time the candidate launch settings on these inputs and keep the
        fastest (:func:`natinterp3d_b200.tuning.tune_batch`)."""
        from .tuning import tune_batch
        return tune_batch(self, queries, query_offsets, values, **kw)

    # ------------------------------------------------------------------ helpers
    def query_offsets(self, counts):
        off = np.zeros(self.P + 1, np.int64)
        off[1:] = np.cumsum(np.asarray(counts, np.int64))
        return off

    def workspace(self, total_queries):
        nb = ctypes.c_size_t()
        N.check(self._lib.nif_batch_workspace_bytes(self._h, int(total_queries), ctypes.byref(nb)),
                'nif_batch_workspace_bytes')
        return torch.empty(int(nb.value), dtype=torch.uint8, device=self.device)

    def _launch(self, q, qoff, v, out, ws):
        D = int(out.shape[1])
        N.check(self._lib.nif_batch_interpolate(
            self._h, _vp(q), _DT[q.dtype], _vp(qoff), _vp(self.centroids), _vp(v), _DT[v.dtype],
            _vp(self.key_offsets), D, _vp(out), _DT[out.dtype], int(q.shape[0]), _vp(ws), ws.numel(),
            _stream_ptr(self.device)), 'nif_batch_interpolate')

    def summary(self, total_queries, ws, stream=None):
        """Row counters of the last batch call on ``ws``, read through
        ``stream`` (default: the current stream), the only stream it waits for."""
        s = N.Summary()
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else _stream_ptr(self.device)
        N.check(self._lib.nif_batch_summary(self._h, int(total_queries), _vp(ws), ws.numel(), sp,
                                            ctypes.byref(s)), 'nif_batch_summary')
        return s

    def _prepare(self, q, qoff, v):
        q = q.contiguous()
        if q.dim() != 2 or q.shape[1] != 3:
            raise ValueError('queries must have shape (total_queries, 3)')
        v2 = v.reshape(int(self.n_keys.sum()), -1).contiguous()
        if isinstance(qoff, torch.Tensor):
            qoff_d = qoff.to(self.device, torch.int64)
        else:
            qoff_d = torch.as_tensor(np.asarray(qoff, np.int64), device=self.device)
        out_dtype = torch.float32 if (q.dtype == torch.float32 and v2.dtype == torch.float32) \
            else torch.float64
        out = torch.empty((q.shape[0], v2.shape[1]), dtype=out_dtype, device=self.device)
        return q, qoff_d, v2, out

    # ------------------------------------------------------------------ API
    def interpolate_device(self, queries, query_offsets, values, check=True):
        """All problems at once.  queries [sum M_p, 3] and values [sum N_p, D]
        concatenated by problem; query_offsets int64 [P+1]."""
        q, qoff, v, out = self._prepare(queries, query_offsets, values)
        with torch.cuda.device(self.device):
            ws = self.workspace(q.shape[0])
            self._launch(q, qoff, v, out, ws)
            if check:
                DeviceMesh._raise_rows(self.summary(q.shape[0], ws))
        return out

    def interpolate(self, queries_list, values_list):
        """Host API: lists of per-problem arrays in, list of per-problem outputs back."""
        if len(queries_list) != self.P or len(values_list) != self.P:
            raise ValueError('need one query array and one value array per problem')
        vals = [np.asarray(v) for v in values_list]
        squeeze = vals[0].ndim == 1
        qs = [np.asarray(q, np.float64).reshape(-1, 3) for q in queries_list]
        qoff = self.query_offsets([len(q) for q in qs])
        if qoff[-1] > 2 * _api.PIPELINE_CHUNK:
            out = self._interpolate_pipelined(qs, qoff, vals)
        else:
            qcat = np.concatenate(qs)
            vcat = np.concatenate([v.reshape(v.shape[0], -1) for v in vals])
            out = self.interpolate_device(torch.from_numpy(qcat).to(self.device), qoff,
                                          torch.from_numpy(np.ascontiguousarray(vcat)).to(self.device))
            out = out.cpu().numpy()
        parts = [out[qoff[p]:qoff[p + 1]] for p in range(self.P)]
        return [p[:, 0] for p in parts] if squeeze else parts

    def _interpolate_pipelined(self, qs, qoff, vals):
        """Large host batches in groups of consecutive problems (about
        PIPELINE_CHUNK queries each): while one group's batch call runs, the
        next group's queries and values go to the device and the previous
        group's results come back, on a separate copy stream through pinned
        staging buffers.  Each call sees the other problems as empty (zero
        queries), so its results are those of the whole batch.  Row counters
        are read once at the end."""
        dev = self.device
        M = int(qoff[-1])
        D = int(vals[0].reshape(vals[0].shape[0], -1).shape[1])
        vdt = torch.float32 if all(v.dtype == np.float32 for v in vals) else torch.float64
        odt = torch.float64  # queries are float64 on this path
        out = np.empty((M, D), np.float64)
        ko = self.key_offsets.cpu().numpy()
        groups, p0 = [], 0
        while p0 < self.P:
            p1 = p0 + 1
            while p1 < self.P and qoff[p1 + 1] - qoff[p0] <= _api.PIPELINE_CHUNK:
                p1 += 1
            groups.append((p0, p1))
            p0 = p1
        cap = max(int(qoff[b] - qoff[a]) for a, b in groups)
        kcap = max(int(ko[b] - ko[a]) for a, b in groups)
        compute = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(device=dev)
        qstage = [torch.empty((cap, 3), dtype=torch.float64, pin_memory=True) for _ in range(2)]
        vstage = [torch.empty((kcap, D), dtype=vdt, pin_memory=True) for _ in range(2)]
        ostage = [torch.empty((cap, D), dtype=odt, pin_memory=True) for _ in range(2)]
        with torch.cuda.device(dev):
            vd = torch.empty((int(ko[-1]), D), dtype=vdt, device=dev)
            # two workspaces in turn: a group's counters are read (on the copy
            # stream) before the group two later reuses its workspace
            wss = [self.workspace(cap) for _ in range(2)]
            pending, counters = None, []

            def drain(item):
                slot, (a, b), res, done = item
                copy.wait_event(done)
                with torch.cuda.stream(copy):
                    ostage[slot][:b - a].copy_(res, non_blocking=True)
                    res.record_stream(copy)
                copy.synchronize()
                out[a:b] = ostage[slot][:b - a].numpy()
                counters.append(self.summary(b - a, wss[slot], stream=copy))

            for k, (g0, g1) in enumerate(groups):
                a, b = int(qoff[g0]), int(qoff[g1])
                ka, kb = int(ko[g0]), int(ko[g1])
                slot = k % 2
                qn, vn = qstage[slot].numpy(), vstage[slot].numpy()
                np.concatenate(qs[g0:g1], out=qn[:b - a])
                np.concatenate([v.reshape(v.shape[0], -1) for v in vals[g0:g1]], out=vn[:kb - ka],
                               casting='same_kind')
                goff = torch.from_numpy(np.clip(qoff - a, 0, b - a))
                with torch.cuda.stream(copy):
                    qd = qstage[slot][:b - a].to(dev, non_blocking=True)
                    vd[ka:kb].copy_(vstage[slot][:kb - ka], non_blocking=True)
                    gd = goff.to(dev, non_blocking=True)
                    loaded = torch.cuda.Event()
                    loaded.record(copy)
                compute.wait_event(loaded)
                qd.record_stream(compute)
                gd.record_stream(compute)
                res = torch.empty((b - a, D), dtype=odt, device=dev)
                self._launch(qd, gd, vd, res, wss[slot])
                done = torch.cuda.Event()
                done.record(compute)
                if pending is not None:
                    drain(pending)
                    # the staging slot of the drained group is free again
                pending = (slot, (a, b), res, done)
            drain(pending)
            for summ in counters:
                DeviceMesh._raise_rows(summ)
        return out

    def interpolate_per_problem(self, queries, query_offsets, values):
        """The same result with one plain call per problem (for comparison)."""
        q, qoff, v, out = self._prepare(queries, query_offsets, values)
        qo = np.asarray(qoff.cpu().numpy() if isinstance(qoff, torch.Tensor) else qoff, np.int64)
        ko = self.key_offsets.cpu().numpy()
        for p, it in enumerate(self.interpolators):
            if qo[p + 1] == qo[p]:
                continue
            out[qo[p]:qo[p + 1]] = it.device_mesh.interpolate(
                q[qo[p]:qo[p + 1]], v[ko[p]:ko[p + 1]], it.centroid, check=False)
        return out

    def capture(self, queries, query_offsets, values):
        """Record the batched pipeline for these (fixed) inputs as a CUDA graph."""
        return BatchGraph(self, queries, query_offsets, values)

    def close(self):
        if getattr(self, '_h', None) is not None and self._h.value:
            self._lib.nif_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchGraph:
    """A captured batched interpolation; ``replay()`` re-runs it and returns ``out``."""

    def __init__(self, batch, queries, query_offsets, values):
        self.batch = batch
        self.q, self.qoff, self.v, self.out = batch._prepare(queries, query_offsets, values)
        with torch.cuda.device(batch.device):
            self.ws = batch.workspace(self.q.shape[0])
            # one eager run first: initialises the kernels' launch configuration
            batch._launch(self.q, self.qoff, self.v, self.out, self.ws)
            torch.cuda.synchronize(batch.device)
            self.graph = torch.cuda.CUDAGraph()
            stream = torch.cuda.Stream(device=batch.device)
            with torch.cuda.graph(self.graph, stream=stream):
                batch._launch(self.q, self.qoff, self.v, self.out, self.ws)

    def replay(self):
        self.graph.replay()
        return self.out

    def summary(self):
        return self.batch.summary(self.q.shape[0], self.ws)
