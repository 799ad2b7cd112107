"""Device-resident mesh and the query calls of libnif_cuda.so.

PyTorch provides device memory and the stream; the computation is the
library's own sm_100a kernels.  All tensors passed to the library are
contiguous CUDA tensors on the mesh's device.
"""
import ctypes

import numpy as np
import torch

from . import _native as N

_DT = {torch.float64: N.NIF_F64, torch.float32: N.NIF_F32}
_NP_DT = {np.dtype(np.float64): N.NIF_F64, np.dtype(np.float32): N.NIF_F32}


def _stream_ptr(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _vp(t):
    """Device address of a tensor; a zero-element view of an allocated buffer
    passes its storage's address (PyTorch reports 0 for empty tensors)."""
    if t is None:
        return ctypes.c_void_p(0)
    if t.numel() > 0:
        return ctypes.c_void_p(t.data_ptr())
    st = t.untyped_storage()
    return ctypes.c_void_p(st.data_ptr() if st.size() > 0 else 0)


def _check_device_tensor(t, device, name):
    if not isinstance(t, torch.Tensor) or t.device != device:
        raise ValueError('%s must be a tensor on %s' % (name, device))


class RowRecords:
    """Every row's cavity record from one weights call (nif_weights_count_records)
    and that call's workspace, for the gradient of the same queries."""

    def __init__(self, q, M, centroid, ws, rec):
        self.q, self.M, self.centroid, self.ws, self.rec = q, M, centroid, ws, rec

    @property
    def nbytes(self):
        return self.ws.numel() + self.rec.numel()


class GPUConstructionError(RuntimeError):
    """The GPU constructor cannot decide this key set (``code``: the status)."""

    def __init__(self, code, info):
        self.code, self.info = code, info
        super().__init__('GPU Delaunay construction: %s (status %d)'
                         % (N._ERR_NAMES.get(code, 'error'), code))


def gpu_delaunay(centered, device=None):
    """The Delaunay tetrahedralization of ``centered`` keys (N, 3) plus
    natinterp3d's super-simplex, built on the GPU (``nif_delaunay_build``).

    Returns ((vxyz, tet_v, tet_n) as device tensors in natinterp3d's packed
    layout, info dict with the construction's counters and exact checks).
    Raises GPUConstructionError where the key set is degenerate for exact
    arithmetic or exceeds the builder's capacities; natinterp3d's host
    constructor handles those sets (with its random perturbations)."""
    if not torch.cuda.is_available():
        raise RuntimeError('natinterp3d_b200 needs a CUDA device')
    dev = torch.device('cuda', torch.cuda.current_device() if device is None
                       else torch.device(device).index or 0)
    lib = N.cuda_lib()
    keys = np.ascontiguousarray(centered, np.float64)
    n = int(keys.shape[0])
    cap, nb = ctypes.c_int(), ctypes.c_size_t()
    N.check(lib.nif_delaunay_max_tets(n, ctypes.byref(cap)), 'nif_delaunay_max_tets')
    N.check(lib.nif_delaunay_workspace_bytes(n, ctypes.byref(nb)), 'nif_delaunay_workspace_bytes')
    info = N.DelaunayInfo()
    with torch.cuda.device(dev):
        d_keys = torch.from_numpy(keys).to(dev)
        ws = torch.empty(int(nb.value), dtype=torch.uint8, device=dev)
        vxyz = torch.empty((n + 4, 3), dtype=torch.float64, device=dev)
        tv = torch.empty((cap.value, 4), dtype=torch.int32, device=dev)
        tn = torch.empty((cap.value, 4), dtype=torch.int32, device=dev)
        rc = lib.nif_delaunay_build(_vp(d_keys), n, _vp(ws), ws.numel(), _vp(vxyz), _vp(tv), _vp(tn),
                                    cap.value, _stream_ptr(dev), ctypes.byref(info))
        del ws
    if rc != N.NIF_OK:
        raise GPUConstructionError(rc, info.as_dict())
    T = int(info.n_tets)
    return (vxyz, tv[:T].clone(), tn[:T].clone()), info.as_dict()


class DeviceMesh:
    """natinterp3d's mesh uploaded to one GPU (resident arrays + seed grid).
    The packed arrays are numpy arrays, or CUDA tensors already on the device
    (a GPU-built mesh)."""

    def __init__(self, vxyz, tet_v, tet_n, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError('natinterp3d_b200 needs a CUDA device (there is no CPU query path)')
        on_device = isinstance(vxyz, torch.Tensor) and vxyz.is_cuda
        if on_device and device is None:
            device = vxyz.device
        self.device = torch.device('cuda', torch.cuda.current_device() if device is None
                                   else torch.device(device).index or 0)
        self._lib = N.cuda_lib()
        if not on_device:
            vxyz = np.ascontiguousarray(vxyz, np.float64)
            tet_v = np.ascontiguousarray(tet_v, np.int32)
            tet_n = np.ascontiguousarray(tet_n, np.int32)
        self.n_vertices, self.n_tets = int(vxyz.shape[0]), int(tet_v.shape[0])
        self.n_keys = self.n_vertices - 4
        nbytes = ctypes.c_size_t()
        N.check(self._lib.nif_dmesh_bytes(self.n_vertices, self.n_tets, ctypes.byref(nbytes)),
                'nif_dmesh_bytes')
        with torch.cuda.device(self.device):
            self._buf = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
            if on_device:
                d_v = vxyz.to(self.device, torch.float64).contiguous()
                d_tv = tet_v.to(self.device, torch.int32).contiguous()
                d_tn = tet_n.to(self.device, torch.int32).contiguous()
            else:
                d_v = torch.from_numpy(vxyz).to(self.device)
                d_tv = torch.from_numpy(tet_v).to(self.device)
                d_tn = torch.from_numpy(tet_n).to(self.device)
            self._vertices = d_v   # keys' coordinates (the transpose product's key order)
            self._h = ctypes.c_void_p()
            N.check(self._lib.nif_dmesh_create(_vp(d_v), _vp(d_tv), _vp(d_tn), self.n_vertices,
                                               self.n_tets, _vp(self._buf), nbytes.value,
                                               _stream_ptr(self.device), ctypes.byref(self._h)),
                    'nif_dmesh_create')
        info = (ctypes.c_int64 * 8)()
        N.check(self._lib.nif_dmesh_info(self._h, info), 'nif_dmesh_info')
        # octree over the tet centroids (point-location seeds): nodes, node levels
        self.octree_stats = {'nodes': int(info[2]), 'levels': int(info[3])}
        # tets whose orient3dfast sign the error bound cannot certify, and
        # those whose "> 0" flag the exact sign changes
        self.orientation_stats = {'uncertain': int(info[5]), 'flipped': int(info[6])}
        self.predicates = 'fast'
        self.last_summary = None

    def set_predicates(self, mode):
        """'fast' (natinterp3d's signs, the default), 'audit' (the same
        results, uncertain and flipped predicate evaluations counted in the
        call summaries) or 'exact' (exact signs)."""
        if mode not in N.PREDICATE_MODES:
            raise ValueError("predicates must be one of 'fast', 'audit', 'exact'")
        N.check(self._lib.nif_dmesh_set_predicates(self._h, N.PREDICATE_MODES[mode]),
                'nif_dmesh_set_predicates')
        self.predicates = mode

    def set_tuning(self, tuning):
        """Launch settings of later query calls (``nif_tuning``: a dict with
        ``blocks_per_sm`` 6 or 8, ``bucket_shift`` -2..1, ``tile`` 0..1024).
        Results do not depend on them."""
        t = N.Tuning.from_dict(tuning)
        rc = self._lib.nif_dmesh_set_tuning(self._h, ctypes.byref(t))
        if rc == N.NIF_ERR_ARG:
            raise ValueError('invalid tuning %r' % (tuning,))
        N.check(rc, 'nif_dmesh_set_tuning')

    def get_tuning(self):
        t = N.Tuning()
        N.check(self._lib.nif_dmesh_get_tuning(self._h, ctypes.byref(t)), 'nif_dmesh_get_tuning')
        return t.as_dict()

    @property
    def nbytes(self):
        return self._buf.numel()

    def workspace_bytes(self, M, mode):
        nb = ctypes.c_size_t()
        N.check(self._lib.nif_query_workspace_bytes(self._h, int(M), mode, ctypes.byref(nb)),
                'nif_query_workspace_bytes')
        return int(nb.value)

    def _workspace(self, M, mode):
        return torch.empty(self.workspace_bytes(M, mode), dtype=torch.uint8, device=self.device)

    @staticmethod
    def _raise_rows(summary):
        if summary.rows_failed:
            code = summary.first_status
            if code == N.NIF_ERR_WALK:
                raise RuntimeError('%d queries did not converge in the point-location walk '
                                   '(step limit reached)' % summary.rows_failed)
            raise RuntimeError('%d queries exceed the per-query capacity of the large-row kernel '
                               '(cavity larger than 4096 tets)' % summary.rows_failed)

    def records_bytes(self, M):
        nb = ctypes.c_size_t()
        N.check(self._lib.nif_records_bytes(int(M), ctypes.byref(nb)), 'nif_records_bytes')
        return int(nb.value)

    def weights_csr(self, q, centroid, vals_dtype=torch.float64, return_summary=False,
                    return_totals=False, keep_records=False):
        """Sibson weights of device queries q [M, 3] (float32/float64, caller frame).

        Returns (rowptr int32 [M+1], cols int32 [nnz], vals [nnz]) on the device,
        plus the per-row normalisers (float64 [M]) when ``return_totals``.
        With ``keep_records`` (meshes with the default fast predicates) every
        row's cavity record is kept and a ``RowRecords`` is appended, which
        ``query_grad(..., records=)`` takes to skip point location and the
        cavity search.
        """
        _check_device_tensor(q, self.device, 'queries')
        q = q.contiguous()
        if q.dim() != 2 or q.shape[1] != 3:
            raise ValueError('Query points must have shape (num_query_points, 3)')
        if q.dtype not in _DT:
            q = q.to(torch.float64)
        M = int(q.shape[0])
        cen = (ctypes.c_double * 3)(*[float(c) for c in centroid])
        if keep_records and self.predicates != 'fast':
            raise ValueError("cavity records are kept for meshes with predicates='fast' only")
        with torch.cuda.device(self.device):
            ws = self._workspace(M, N.NIF_MODE_WEIGHTS)
            rowptr = torch.empty(M + 1, dtype=torch.int32, device=self.device)
            summ = N.Summary()
            if keep_records:
                rec = torch.empty(self.records_bytes(M), dtype=torch.uint8, device=self.device)
                rc = self._lib.nif_weights_count_records(
                    self._h, _vp(q), _DT[q.dtype], M, cen, _vp(ws), ws.numel(), _vp(rowptr),
                    _vp(rec), rec.numel(), _stream_ptr(self.device), ctypes.byref(summ))
            else:
                rc = self._lib.nif_weights_count(self._h, _vp(q), _DT[q.dtype], M, cen, _vp(ws),
                                                 ws.numel(), _vp(rowptr), _stream_ptr(self.device),
                                                 ctypes.byref(summ))
            if rc == N.NIF_ERR_OVERFLOW:
                raise OverflowError('Total number of nonzero weights exceeds int32 limit')
            N.check(rc, 'nif_weights_count')
            self.last_summary = summ.as_dict()
            self._raise_rows(summ)
            nnz = int(summ.nnz)
            # at least one element each, so the library always gets real pointers
            cols = torch.empty(max(nnz, 1), dtype=torch.int32, device=self.device)[:nnz]
            vals = torch.empty(max(nnz, 1), dtype=vals_dtype, device=self.device)[:nnz]
            totals = torch.empty(max(M, 1), dtype=torch.float64, device=self.device)[:M] \
                if return_totals else None
            N.check(self._lib.nif_weights_fill(self._h, _vp(q), _DT[q.dtype], M, cen, _vp(ws),
                                               ws.numel(), _vp(rowptr),
                                               _vp(vals), _DT[vals_dtype], _vp(cols), _vp(totals),
                                               _stream_ptr(self.device)), 'nif_weights_fill')
        out = (rowptr, cols, vals)
        if return_totals:
            out = out + (totals,)
        if return_summary:
            out = out + (summ.as_dict(),)
        if keep_records:
            out = out + (RowRecords(q, M, tuple(float(c) for c in centroid), ws, rec),)
        return out

    def interpolate(self, q, values, centroid, return_summary=False, check=True, sync=True, ws=None):
        """out[M, D] = W(q) @ values without materialising W (device tensors).

        With ``sync=False`` and ``return_summary`` the row counters are left on
        the device (returned as a pending handle for :meth:`raise_pending`).
        ``ws``: a workspace of at least ``workspace_bytes(M, NIF_MODE_INTERP)``
        bytes to use instead of a new one."""
        _check_device_tensor(q, self.device, 'queries')
        _check_device_tensor(values, self.device, 'values')
        q = q.contiguous()
        if q.dim() != 2 or q.shape[1] != 3:
            raise ValueError('Query points must have shape (num_query_points, 3)')
        if values.dim() not in (1, 2) or values.shape[0] != self.n_keys:
            raise ValueError('values must have shape (%d,) or (%d, D)' % (self.n_keys, self.n_keys))
        squeeze = values.dim() == 1
        v = values.reshape(self.n_keys, -1).contiguous()
        if q.dtype not in _DT or v.dtype not in _DT:
            raise TypeError('queries and values must be float32 or float64')
        out_dtype = torch.float32 if (q.dtype == torch.float32 and v.dtype == torch.float32) \
            else torch.float64
        M, D = int(q.shape[0]), int(v.shape[1])
        cen = (ctypes.c_double * 3)(*[float(c) for c in centroid])
        with torch.cuda.device(self.device):
            if ws is None:
                ws = self._workspace(M, N.NIF_MODE_INTERP)
            out = torch.empty((M, D), dtype=out_dtype, device=self.device)
            summ = N.Summary()
            want = check or (return_summary and sync)
            N.check(self._lib.nif_interpolate(self._h, _vp(q), _DT[q.dtype], M, cen, _vp(v),
                                              _DT[v.dtype], D, _vp(out), _DT[out_dtype], _vp(ws),
                                              ws.numel(), _stream_ptr(self.device),
                                              ctypes.byref(summ) if want else None),
                    'nif_interpolate')
            if want:
                self.last_summary = summ.as_dict()
            if check:
                self._raise_rows(summ)
        out = out[:, 0] if squeeze else out
        if return_summary:
            if not sync and not check:
                return out, (M, ws)   # counters stay on the device
            return out, summ.as_dict()
        return out

    def pending_summary(self, pending, stream=None):
        """Row counters of one interpolate(..., sync=False) call, read through
        ``stream`` (a torch.cuda.Stream ordered after the call; default: the
        current stream), which is the only stream this waits for.  Afterwards
        the call's workspace may be released."""
        M, ws = pending
        summ = N.Summary()
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else _stream_ptr(self.device)
        N.check(self._lib.nif_query_summary(self._h, int(M), N.NIF_MODE_INTERP, _vp(ws),
                                            ws.numel(), sp, ctypes.byref(summ)), 'nif_query_summary')
        return summ.as_dict()

    def raise_pending(self, pending):
        """Row counters of interpolate(..., sync=False) calls (pending handles,
        read here after the calls ran, or dicts from :meth:`pending_summary`):
        keep their sum as ``last_summary`` and raise if any row failed."""
        total = None
        for item in pending:
            d = item if isinstance(item, dict) else self.pending_summary(item)
            total = d if total is None else {k: (v + d[k] if k != 'first_status' else v or d[k])
                                             for k, v in total.items()}
        if total is not None:
            self.last_summary = total
            self._raise_rows(N.Summary.from_dict(total))

    # -------------------------------------------------------------- sparse / grad
    def spmm(self, rowptr, cols, vals, x):
        """W @ x for a device CSR W (rows = len(rowptr) - 1, columns = n_keys)."""
        x2 = x.reshape(x.shape[0], -1).contiguous()
        M, D = int(rowptr.numel()) - 1, int(x2.shape[1])
        out_dtype = torch.float32 if (vals.dtype == torch.float32 and x2.dtype == torch.float32) \
            else torch.float64
        y = torch.empty((M, D), dtype=out_dtype, device=self.device)
        with torch.cuda.device(self.device):
            N.check(self._lib.nif_spmm(M, int(x2.shape[0]), _vp(rowptr), _vp(cols), _vp(vals),
                                       _DT[vals.dtype], _vp(x2), _DT[x2.dtype], D, _vp(y),
                                       _DT[out_dtype], _stream_ptr(self.device)), 'nif_spmm')
        return y

    @property
    def key_rank(self):
        """Position of each key in a Morton order of the keys (int32 [n_keys] on
        the device; computed on first use): the order in which the transpose
        product visits the keys, so that neighbouring keys share their
        gradient rows in L2."""
        if getattr(self, '_key_rank', None) is None:
            v = self._vertices[:self.n_keys]
            lo = v.min(0).values
            span = (v.max(0).values - lo).clamp_min(1e-300)
            cell = ((v - lo) / span * 1023.0).to(torch.int64).clamp_(0, 1023)
            code = torch.zeros(self.n_keys, dtype=torch.int64, device=self.device)
            for b in range(10):
                for a in range(3):
                    code |= ((cell[:, a] >> b) & 1) << (3 * b + a)
            order = torch.argsort(code, stable=True)
            rank = torch.empty_like(order)
            rank[order] = torch.arange(self.n_keys, device=self.device)
            self._key_rank = rank.to(torch.int32)
        return self._key_rank

    def spmm_t(self, rowptr, cols, vals, x, n_cols):
        """W^T @ x (deterministic, CSC by stable sort) for a device CSR W.  When
        W's columns are this mesh's keys the columns are visited in a spatial
        order of the keys (same results, fewer HBM re-reads)."""
        x2 = x.reshape(x.shape[0], -1).contiguous()
        M, D, nnz = int(rowptr.numel()) - 1, int(x2.shape[1]), int(cols.numel())
        out_dtype = torch.float32 if (vals.dtype == torch.float32 and x2.dtype == torch.float32) \
            else torch.float64
        y = torch.empty((n_cols, D), dtype=out_dtype, device=self.device)
        nb = ctypes.c_size_t()
        N.check(self._lib.nif_spmm_t_workspace_bytes(M, n_cols, nnz, ctypes.byref(nb)),
                'nif_spmm_t_workspace_bytes')
        with torch.cuda.device(self.device):
            ws = torch.empty(max(int(nb.value), 256), dtype=torch.uint8, device=self.device)
            if n_cols == self.n_keys and getattr(self, '_vertices', None) is not None:
                N.check(self._lib.nif_spmm_t_ordered(
                    M, n_cols, nnz, _vp(rowptr), _vp(cols), _vp(vals), _DT[vals.dtype], _vp(x2),
                    _DT[x2.dtype], D, _vp(y), _DT[out_dtype], _vp(self.key_rank), _vp(ws),
                    ws.numel(), _stream_ptr(self.device)), 'nif_spmm_t_ordered')
            else:
                N.check(self._lib.nif_spmm_t(M, n_cols, nnz, _vp(rowptr), _vp(cols), _vp(vals),
                                             _DT[vals.dtype], _vp(x2), _DT[x2.dtype], D, _vp(y),
                                             _DT[out_dtype], _vp(ws), ws.numel(),
                                             _stream_ptr(self.device)), 'nif_spmm_t')
        return y

    def query_grad(self, q, values, gout, centroid, rowptr, weights, totals, records=None):
        """d loss / d queries for gout = d loss / d interpolate(q, values), given the
        forward pass's CSR (rowptr, float64 weights) and row normalisers.  With
        ``records`` (the forward's ``RowRecords``, same queries) the rows start
        from the kept cavity records instead of locating and flooding again."""
        q = q.contiguous()
        v = values.reshape(self.n_keys, -1).contiguous()
        M, D = int(q.shape[0]), int(v.shape[1])
        gdt = torch.float32 if (q.dtype == torch.float32 and v.dtype == torch.float32) \
            else torch.float64
        g = gout.reshape(M, D).to(gdt).contiguous()
        gq = torch.empty((M, 3), dtype=q.dtype, device=self.device)
        cen = (ctypes.c_double * 3)(*[float(c) for c in centroid])
        with torch.cuda.device(self.device):
            summ = N.Summary()
            w64 = weights if weights.dtype == torch.float64 else weights.to(torch.float64)
            if records is not None:
                if records.M != M or records.q.data_ptr() != q.data_ptr() or \
                        records.centroid != tuple(float(c) for c in centroid):
                    raise ValueError('records belong to another weights call')
                N.check(self._lib.nif_query_grad_records(
                    self._h, _vp(q), _DT[q.dtype], M, cen, _vp(rowptr), _vp(w64), _vp(totals),
                    _vp(v), _DT[v.dtype], D, _vp(g), _DT[gdt], _vp(gq), _vp(records.ws),
                    records.ws.numel(), _vp(records.rec), records.rec.numel(),
                    _stream_ptr(self.device), ctypes.byref(summ)), 'nif_query_grad_records')
            else:
                ws = self._workspace(M, N.NIF_MODE_INTERP)
                N.check(self._lib.nif_query_grad(self._h, _vp(q), _DT[q.dtype], M, cen, _vp(rowptr),
                                                 _vp(w64), _vp(totals), _vp(v), _DT[v.dtype], D,
                                                 _vp(g), _DT[gdt], _vp(gq), _vp(ws), ws.numel(),
                                                 _stream_ptr(self.device), ctypes.byref(summ)),
                        'nif_query_grad')
            self._raise_rows(summ)
        return gq

    def close(self):
        if getattr(self, '_h', None) is not None and self._h.value:
            self._lib.nif_dmesh_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
