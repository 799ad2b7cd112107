"""natinterp3d's public API (natinterp3d.py:9-137 of natinterp3d), on one GPU.

Same names, arguments, return types and errors:

* ``Interpolator(data_points, parallel=True, num_threads=None)`` builds the
  Delaunay tetrahedralization with natinterp3d's own constructor, then keeps
  the mesh resident on the GPU;
* ``Interpolator.get_weights(query_points)`` -> ``scipy.sparse.csr_matrix``
  (M, N) with int32 indices, dtype = query dtype, columns of each row in
  natinterp3d's order;
* ``Interpolator.interpolate(query_points, values)`` -> ndarray (M,) or (M, D);
* module-level ``get_weights`` / ``interpolate``.

``parallel`` and ``num_threads`` are accepted for compatibility and have no
effect.  ``device`` selects the CUDA device (default: the current one).
There is no CPU fallback: without a CUDA device the query methods raise.

``predicates`` (an extension) selects the geometric predicates: 'fast' is
natinterp3d's behaviour and the default; 'audit' gives identical results and
counts the predicate evaluations that the static error bound cannot certify
(``predicate_stats``); 'exact' decides them exactly.

``constructor`` (an extension) selects who builds the tetrahedralization:
'host' (the default) is natinterp3d's own constructor; 'gpu' builds the same
Delaunay tetrahedralization of keys + super-simplex on the GPU with exact
predicates (``construction`` reports its counters and checks).  For keys in
general position the two give the same set of tets, stored in another order,
so weights agree to rounding and the column order of a row may differ.  Key
sets that are degenerate for exact arithmetic (which natinterp3d perturbs
randomly) fall back to the host constructor with a warning.

Device-resident variants (``get_weights_device``, ``interpolate_device``)
take and return torch tensors on the mesh's GPU.
"""
import os
from typing import Optional

import warnings

import numpy as np
import scipy.sparse
import torch

from . import _native as N
from ._native import HostMesh
from .device import DeviceMesh, GPUConstructionError, gpu_delaunay

_FLOATS = (np.dtype(np.float32), np.dtype(np.float64))
PIPELINE_CHUNK = 1 << 21  # queries per chunk of the pipelined host interpolation


HOST_STAGE = 1 << 24  # bytes per pinned staging buffer of device-to-host copies


def _to_host(t):
    """A device tensor as a numpy array in pageable host memory: copied
    through two reused pinned staging buffers on a side stream, the copy of
    one piece overlapping the host-side copy (multithreaded) of the previous;
    large results come back several times faster than a direct pageable copy,
    whose first touch of fresh host pages is single-threaded."""
    t = t.contiguous()
    n = t.numel()
    out = torch.empty(t.shape, dtype=t.dtype)
    if n * t.element_size() <= HOST_STAGE:
        out.copy_(t)
        return out.numpy()
    flat, dst = t.view(-1), out.view(-1)
    step = HOST_STAGE // t.element_size()
    dev = t.device
    copy = torch.cuda.Stream(device=dev)
    copy.wait_stream(torch.cuda.current_stream(dev))
    stage = [torch.empty(step, dtype=t.dtype, pin_memory=True) for _ in range(2)]
    done = [None, None]
    pieces = [(a, min(n, a + step)) for a in range(0, n, step)]

    def issue(k):
        a, b = pieces[k]
        with torch.cuda.stream(copy):
            stage[k % 2][:b - a].copy_(flat[a:b], non_blocking=True)
            done[k % 2] = torch.cuda.Event()
            done[k % 2].record(copy)

    issue(0)
    for k, (a, b) in enumerate(pieces):
        if k + 1 < len(pieces):
            issue(k + 1)
        done[k % 2].synchronize()
        dst[a:b].copy_(stage[k % 2][:b - a])
    flat.record_stream(copy)
    return out.numpy()


def pipeline_bounds(M, chunk):
    """Row ranges of a pipelined call: full chunks, with a first and a last
    chunk of chunk/8 rows, whose upload and whose download plus host copy are
    the only transfers that cannot overlap a kernel."""
    small = max(1, chunk // 8)
    first = min(M, small)
    bounds, a = [(0, first)], first
    while M - a > chunk + small:
        bounds.append((a, a + chunk))
        a += chunk
    if M - a > small:
        bounds.append((a, M - small))
        a = M - small
    if M > a:
        bounds.append((a, M))
    return bounds


def interpolate(
    queries: np.ndarray,
    keys: np.ndarray,
    values: np.ndarray,
    parallel: bool = True,
    num_threads: Optional[int] = None,
    device=None,
) -> np.ndarray:
    """Natural-neighbour (Sibson) interpolation of ``values`` known at ``keys``,
    evaluated at ``queries``.  Shapes: queries (M, 3), keys (N, 3), values (N,)
    or (N, D); returns (M,) or (M, D)."""
    interpolator = Interpolator(keys, parallel=parallel, num_threads=num_threads, device=device)
    return interpolator.interpolate(queries, values)


def get_weights(
    queries: np.ndarray,
    keys: np.ndarray,
    parallel: bool = True,
    num_threads: Optional[int] = None,
    device=None,
) -> scipy.sparse.csr_matrix:
    """Sibson coordinates of ``queries`` with respect to ``keys`` as an (M, N)
    CSR matrix."""
    interpolator = Interpolator(keys, parallel=parallel, num_threads=num_threads, device=device)
    return interpolator.get_weights(queries)


class Interpolator:
    """Natural-neighbour interpolator for 3-D data points.

    Build once per key set and reuse: the Delaunay construction (natinterp3d's
    own, on the host) is the expensive part; queries run on the GPU.

    Args:
        data_points: (N, 3) data sites.
        parallel, num_threads: accepted for compatibility with natinterp3d; unused.
        device: CUDA device for the resident mesh (default: current device).
        keep_host_mesh: keep natinterp3d's host mesh object alive (only needed
            to run natinterp3d's CPU query on the same mesh for comparison).
        predicates: 'fast' (natinterp3d's non-robust signs), 'audit' or 'exact'.
        constructor: 'host' (natinterp3d's constructor) or 'gpu' (the same
            Delaunay tetrahedralization built on the GPU; degenerate key sets
            fall back to 'host').
    """

    def __init__(
        self,
        data_points: np.ndarray,
        parallel: bool = True,
        num_threads: Optional[int] = None,
        device=None,
        keep_host_mesh: bool = False,
        predicates: str = 'fast',
        constructor: str = 'host',
    ):
        data_points = np.ascontiguousarray(data_points, np.float64)
        if data_points.ndim != 2 or data_points.shape[1] != 3:
            raise ValueError('Data points must have shape (num_data_points, 3)')
        if constructor not in ('host', 'gpu'):
            raise ValueError("constructor must be 'host' or 'gpu'")
        # natinterp3d.py:88-90: centre on the key centroid before triangulating
        self._centroid = data_points.mean(axis=0)
        centered = data_points - self._centroid
        self.n_keys = int(data_points.shape[0])
        self.parallel = parallel
        self.num_threads = num_threads
        self._device_arg = device
        self._dmesh = None
        self._mesh_arrays = None
        self._mesh_dev = None
        self.host_mesh = None
        self.construction = {'constructor': 'host'}
        if constructor == 'gpu':
            try:
                self._mesh_dev, info = gpu_delaunay(centered, device)
                self.construction = dict(info, constructor='gpu')
                self.degeneracies = {'coplanar': 0, 'cospherical': 0}
            except GPUConstructionError as e:
                warnings.warn('%s; using natinterp3d\'s host constructor' % e, RuntimeWarning)
                self.construction = dict(e.info, constructor='host', gpu_declined=str(e))
        if self._mesh_dev is None:
            host = HostMesh(centered)
            self.degeneracies = host.degeneracies()
            self._mesh_arrays = host.export()
            self.host_mesh = host if keep_host_mesh else None
            if not keep_host_mesh:
                host.close()
        self._predicates = 'fast'
        self.set_predicates(predicates)

    @property
    def mesh_arrays(self):
        """(vxyz, tet_v, tet_n): the packed mesh as numpy arrays (copied from
        the device on first use for a GPU-built mesh)."""
        if self._mesh_arrays is None and getattr(self, '_mesh_dev', None) is not None:
            self._mesh_arrays = tuple(t.cpu().numpy() for t in self._mesh_dev)
        return self._mesh_arrays

    @mesh_arrays.setter
    def mesh_arrays(self, arrays):
        self._mesh_arrays = arrays
        self._mesh_dev = None

    @classmethod
    def from_mesh(cls, centroid, vxyz, tet_v, tet_n, device=None, predicates='fast'):
        """An interpolator over an already exported mesh (see :meth:`save_mesh`)."""
        self = cls.__new__(cls)
        self._centroid = np.asarray(centroid, np.float64).reshape(3)
        self.mesh_arrays = (np.ascontiguousarray(vxyz, np.float64),
                            np.ascontiguousarray(tet_v, np.int32),
                            np.ascontiguousarray(tet_n, np.int32))
        self.n_keys = self.mesh_arrays[0].shape[0] - 4
        self.parallel, self.num_threads = True, None
        self.degeneracies = None
        self.host_mesh = None
        self.construction = {'constructor': 'saved mesh'}
        self._device_arg = device
        self._dmesh = None
        self._predicates = 'fast'
        self.set_predicates(predicates)
        return self

    def save_mesh(self, path):
        """Write the centroid and the packed mesh to an .npz file."""
        vxyz, tet_v, tet_n = self.mesh_arrays
        np.savez(path, centroid=self._centroid, vxyz=vxyz, tet_v=tet_v, tet_n=tet_n)

    @classmethod
    def load_mesh(cls, path, device=None):
        z = np.load(path)
        return cls.from_mesh(z['centroid'], z['vxyz'], z['tet_v'], z['tet_n'], device=device)

    # ------------------------------------------------------------------ pickling
    def __getstate__(self):
        """The key centroid and the packed mesh (natinterp3d's own mesh,
        perturbations included), the predicate mode and launch settings; the
        device-resident copy is rebuilt on first use after unpickling.  The
        CUDA device is kept as its index (the current device where it does
        not exist)."""
        vxyz, tet_v, tet_n = self.mesh_arrays
        dev = self._device_arg
        if isinstance(dev, torch.device):
            dev = dev.index
        elif isinstance(dev, str):
            dev = torch.device(dev).index
        return {'format': 1, 'centroid': self._centroid, 'vxyz': vxyz, 'tet_v': tet_v,
                'tet_n': tet_n, 'parallel': self.parallel, 'num_threads': self.num_threads,
                'degeneracies': self.degeneracies, 'predicates': self._predicates,
                'tuning': getattr(self, '_tuning', None), 'device': dev,
                'construction': getattr(self, 'construction', None)}

    def __setstate__(self, state):
        if state.get('format') != 1:
            raise ValueError('unknown Interpolator pickle format %r' % (state.get('format'),))
        dev = state['device']
        if dev is not None and not (torch.cuda.is_available() and dev < torch.cuda.device_count()):
            dev = None
        self._centroid = np.asarray(state['centroid'], np.float64).reshape(3)
        self.mesh_arrays = (np.ascontiguousarray(state['vxyz'], np.float64),
                            np.ascontiguousarray(state['tet_v'], np.int32),
                            np.ascontiguousarray(state['tet_n'], np.int32))
        self.n_keys = self.mesh_arrays[0].shape[0] - 4
        self.parallel, self.num_threads = state['parallel'], state['num_threads']
        self.degeneracies = state['degeneracies']
        self.host_mesh = None
        self._device_arg = dev
        self._dmesh = None
        self._predicates = state['predicates']
        self._tuning = state['tuning']
        self.construction = state.get('construction') or {'constructor': 'host'}

    @property
    def centroid(self):
        return self._centroid

    @property
    def device_mesh(self) -> DeviceMesh:
        if self._dmesh is None:
            src = getattr(self, '_mesh_dev', None)
            self._dmesh = DeviceMesh(*(src if src is not None else self.mesh_arrays),
                                     device=self._device_arg)
            self._dmesh.set_predicates(self._predicates)
            if getattr(self, '_tuning', None) is not None:
                self._dmesh.set_tuning(self._tuning)
        return self._dmesh

    # ------------------------------------------------------------------ tuning
    def set_tuning(self, tuning):
        """Launch settings of the query kernels for the following calls
        (``blocks_per_sm`` 6 or 8, ``bucket_shift`` -2..1, ``tile`` 0..1024);
        they change speed only, never results."""
        self.device_mesh.set_tuning(tuning)
        self._tuning = dict(tuning)

    @property
    def tuning(self):
        return self.device_mesh.get_tuning()

    def tune(self, query_points, values=None, mode='interpolate', **kw):
        """Time the candidate launch settings on (a sample of) these queries
        and keep the fastest; see :func:`natinterp3d_b200.tuning.tune`."""
        from .tuning import tune
        return tune(self, query_points, values, mode=mode, **kw)

    def set_predicates(self, mode):
        """'fast', 'audit' or 'exact' for the following calls."""
        if mode not in ('fast', 'audit', 'exact'):
            raise ValueError("predicates must be one of 'fast', 'audit', 'exact'")
        self._predicates = mode
        if self._dmesh is not None:
            self._dmesh.set_predicates(mode)

    @property
    def predicates(self):
        return self._predicates

    @property
    def predicate_stats(self):
        """Counters of the last query call ('audit' and 'exact' modes): walk
        orientation and cavity in-sphere tests natinterp3d makes whose fast
        value the error bound cannot certify (*_uncertain) and those whose
        decision the exact sign changes (*_flipped); plus the mesh's tets with
        an uncertain / flipped orientation flag."""
        dm = self.device_mesh
        s = dm.last_summary or {}
        keys = ('orient_uncertain', 'orient_flipped', 'insphere_uncertain', 'insphere_flipped')
        out = {k: int(s.get(k, 0)) for k in keys}
        out['tets_orientation_uncertain'] = dm.orientation_stats['uncertain']
        out['tets_orientation_flipped'] = dm.orientation_stats['flipped']
        return out

    @property
    def device(self):
        return self.device_mesh.device

    # ------------------------------------------------------------------ host API
    def get_weights(self, query_points: np.ndarray) -> scipy.sparse.csr_matrix:
        """Natural interpolation weights (Sibson coordinates) of the query points."""
        query_points = np.asarray(query_points)
        out_dtype = query_points.dtype
        q = self._host_queries(query_points)
        dm = self.device_mesh
        qd = torch.from_numpy(q).to(dm.device)
        rowptr, cols, vals = dm.weights_csr(qd, self._centroid, vals_dtype=torch.float64)
        M = q.shape[0]
        W = scipy.sparse.csr_matrix(
            (_to_host(vals), _to_host(cols), _to_host(rowptr)), shape=(M, self.n_keys))
        # natinterp3d.py:117; a dtype-changing astype also canonicalises the
        # CSR (sorted columns), exactly as it does for natinterp3d's result
        return W.astype(out_dtype, copy=False)

    def interpolate(self, query_points: np.ndarray, values: np.ndarray) -> np.ndarray:
        """Interpolated values at the query points: (M,) for values (N,), (M, D)
        for values (N, D)."""
        query_points = np.asarray(query_points)
        values = np.asarray(values)
        qdt = query_points.dtype
        if qdt not in _FLOATS or values.dtype not in _FLOATS or values.ndim not in (1, 2):
            # dtypes the fused kernel does not cover: the weights still come
            # from the GPU and scipy forms the product, as natinterp3d does
            weights = self.get_weights(query_points)
            if len(values.shape) == 1:
                return np.squeeze(weights @ values[:, np.newaxis], axis=1)
            return weights @ values
        if values.shape[0] != self.n_keys:
            raise ValueError('dimension mismatch')
        q = self._host_queries(query_points)
        dm = self.device_mesh
        vd = torch.from_numpy(np.ascontiguousarray(values)).to(dm.device)
        if q.shape[0] > 2 * PIPELINE_CHUNK:
            return self._interpolate_pipelined(q, vd)
        qd = torch.from_numpy(q).to(dm.device)
        out = dm.interpolate(qd, vd, self._centroid)
        return out.cpu().numpy()

    def _interpolate_pipelined(self, q, vd):
        """Large host batches in chunks: while the kernels of one chunk run, the
        next chunk's queries go to the device and the previous chunk's results
        come back, on a separate copy stream through pinned staging buffers."""
        dm = self.device_mesh
        dev = dm.device
        M = q.shape[0]
        D = 1 if vd.dim() == 1 else int(vd.shape[1])
        odt = torch.float32 if (q.dtype == np.float32 and vd.dtype == torch.float32) else torch.float64
        out = np.empty((M, D), dtype=np.float32 if odt == torch.float32 else np.float64)
        bounds = pipeline_bounds(M, PIPELINE_CHUNK)
        compute = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(device=dev)
        staging = [torch.empty((PIPELINE_CHUNK, D), dtype=odt, pin_memory=True) for _ in range(2)]
        # two workspaces in turn: a chunk's counters are read (on the copy
        # stream) before the chunk two later reuses its workspace
        wss = [dm._workspace(PIPELINE_CHUNK, N.NIF_MODE_INTERP) for _ in range(2)]
        counters = []
        pending = None  # (slot, rows, device result, event, row-counter handle)

        def drain(item):
            slot, (a, b), res, done, handle = item
            copy.wait_event(done)
            with torch.cuda.stream(copy):
                staging[slot][:b - a].copy_(res.reshape(b - a, D), non_blocking=True)
                res.record_stream(copy)
            copy.synchronize()
            out[a:b] = staging[slot][:b - a].numpy()
            # the chunk's row counters, read on the copy stream (the compute
            # stream runs on); its workspace is free once this returns
            counters.append(dm.pending_summary(handle, copy))

        with torch.cuda.device(dev):
            for k, (a, b) in enumerate(bounds):
                with torch.cuda.stream(copy):
                    qd = torch.from_numpy(q[a:b]).to(dev)
                    loaded = torch.cuda.Event()
                    loaded.record(copy)
                compute.wait_event(loaded)
                qd.record_stream(compute)
                res, handle = dm.interpolate(qd, vd, self._centroid, return_summary=True,
                                             check=False, sync=False, ws=wss[k % 2])
                done = torch.cuda.Event()
                done.record(compute)
                if pending is not None:
                    drain(pending)
                pending = (k % 2, (a, b), res, done, handle)
            drain(pending)
            pending = None
        dm.raise_pending(counters)
        return out[:, 0] if vd.dim() == 1 else out

    # -------------------------------------------------------- device-resident API
    def get_weights_device(self, queries: torch.Tensor, dtype=None, as_torch_csr=False):
        """Weights of device queries; returns (rowptr, cols, vals) device tensors
        or a ``torch.sparse_csr_tensor`` when ``as_torch_csr``."""
        dm = self.device_mesh
        vdt = dtype or (torch.float32 if queries.dtype == torch.float32 else torch.float64)
        rowptr, cols, vals = dm.weights_csr(queries, self._centroid, vals_dtype=vdt)
        if as_torch_csr:
            return torch.sparse_csr_tensor(rowptr, cols, vals, size=(queries.shape[0], self.n_keys))
        return rowptr, cols, vals

    def get_weights_dlpack(self, queries: torch.Tensor, dtype=None):
        """The device CSR of :meth:`get_weights_device` as three DLPack
        capsules (indptr int32 [M+1], indices int32 [nnz], data [nnz]) for
        other CUDA array libraries, with no copy: e.g. with CuPy,
        ``cupyx.scipy.sparse.csr_matrix((cp.from_dlpack(data),
        cp.from_dlpack(indices), cp.from_dlpack(indptr)), shape=(M, N))``.
        Columns within a row are in natinterp3d's order."""
        from torch.utils.dlpack import to_dlpack
        rowptr, cols, vals = self.get_weights_device(queries, dtype=dtype)
        return to_dlpack(rowptr), to_dlpack(cols), to_dlpack(vals)

    def interpolate_device(self, queries: torch.Tensor, values: torch.Tensor, check=True):
        return self.device_mesh.interpolate(queries, values, self._centroid, check=check)

    # ------------------------------------------------------------------ helpers
    @staticmethod
    def _host_queries(query_points):
        if query_points.ndim != 2 or query_points.shape[1] != 3:
            raise ValueError('Query points must have shape (num_query_points, 3)')
        if query_points.dtype in _FLOATS:
            # the device converts float32 to float64 exactly, then subtracts
            # the centroid in float64 (natinterp3d.py:115)
            return np.ascontiguousarray(query_points)
        return np.ascontiguousarray(query_points, np.float64)


def default_num_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
