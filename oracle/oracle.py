"""Python wrappers of the CPU checker -- TEST INFRASTRUCTURE ONLY.

* :class:`OracleMesh` / :func:`oracle_weights` -- the C restatement in
  ``nif_oracle.c`` over the packed mesh arrays.
* :class:`RefLib` -- natinterp3d's own query code (``_ref``), run either on a
  mesh it builds itself or on the natinterp3d mesh object behind a product
  ``HostMesh`` (same sources and flags, so the same struct layout).

Nothing in the product imports this module.
"""
import ctypes
import os

import numpy as np
import scipy.sparse

from . import build_oracle

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_void_p = ctypes.c_void_p

STATS_FIELDS = ('queries', 'walk_steps', 'insphere', 'cavity', 'boundary', 'neighbours',
                'old_terms', 'new_terms', 'face_cc', 'coincident', 'outside', 'empty', 'errors',
                'orient_uncertain', 'orient_flipped', 'insphere_uncertain', 'insphere_flipped')

PREDICATE_MODES = {'fast': 0, 'audit': 1, 'exact': 2}

_olib = None
_rlib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        path = build_oracle.ORACLE_SO
        if not os.path.exists(path):
            build_oracle.build_oracle()
        lib = ctypes.CDLL(path)
        lib.orc_mesh_new.argtypes = [c_double_p, ctypes.c_int, c_int_p, c_int_p, ctypes.c_int]
        lib.orc_mesh_new.restype = c_void_p
        lib.orc_mesh_free.argtypes = [c_void_p]
        lib.orc_mesh_free.restype = None
        lib.orc_weights.argtypes = [c_void_p, c_double_p, ctypes.c_int,
                                    ctypes.POINTER(c_double_p), ctypes.POINTER(c_int_p), c_int_p,
                                    ctypes.POINTER(ctypes.c_byte), ctypes.POINTER(ctypes.c_long)]
        lib.orc_weights.restype = ctypes.c_int
        lib.orc_free.argtypes = [c_void_p]
        lib.orc_free.restype = None
        lib.orc_spmm.argtypes = [ctypes.c_int, ctypes.c_int, c_int_p, c_int_p, c_double_p,
                                 c_double_p, c_double_p]
        lib.orc_spmm.restype = None
        lib.orc_tet_geometry.argtypes = [c_void_p, ctypes.POINTER(ctypes.c_ubyte), c_double_p,
                                         c_double_p]
        lib.orc_tet_geometry.restype = None
        lib.orc_orient.argtypes = [c_double_p] * 4
        lib.orc_orient.restype = ctypes.c_double
        lib.orc_insphere.argtypes = [c_double_p] * 5
        lib.orc_insphere.restype = ctypes.c_double
        lib.orc_mesh_set_predicates.argtypes = [c_void_p, ctypes.c_int]
        lib.orc_mesh_set_predicates.restype = ctypes.c_int
        lib.orc_mesh_predicate_info.argtypes = [c_void_p, ctypes.POINTER(ctypes.c_long)]
        lib.orc_mesh_predicate_info.restype = None
        lib.orc_mesh_set_seed.argtypes = [c_void_p, ctypes.c_int]
        lib.orc_mesh_set_seed.restype = ctypes.c_int
        for name, n in (('orc_orient_exact_sign', 4), ('orc_insphere_exact_sign', 5),
                        ('orc_orient_uncertain', 4), ('orc_insphere_uncertain', 5)):
            fn = getattr(lib, name)
            fn.argtypes = [c_double_p] * n
            fn.restype = ctypes.c_int
        _olib = lib
    return _olib


def _dp(a):
    return a.ctypes.data_as(c_double_p)


def _ip(a):
    return a.ctypes.data_as(c_int_p)


def _take_csr(lib_free, vals_p, cols_p, rowptr, M, N):
    nnz = int(rowptr[M])
    vals = np.ctypeslib.as_array(vals_p, shape=(max(nnz, 1),))[:nnz].copy() if nnz else \
        np.empty(0, np.float64)
    cols = np.ctypeslib.as_array(cols_p, shape=(max(nnz, 1),))[:nnz].copy() if nnz else \
        np.empty(0, np.int32)
    lib_free(ctypes.cast(vals_p, c_void_p))
    lib_free(ctypes.cast(cols_p, c_void_p))
    return scipy.sparse.csr_matrix((vals, cols.astype(np.int32), rowptr), shape=(M, N))


class OracleMesh:
    """The C restatement bound to one packed mesh (arrays are kept alive here)."""

    def __init__(self, vxyz, tet_v, tet_n):
        self.vxyz = np.ascontiguousarray(vxyz, np.float64)
        self.tet_v = np.ascontiguousarray(tet_v, np.int32)
        self.tet_n = np.ascontiguousarray(tet_n, np.int32)
        self.n_keys = self.vxyz.shape[0] - 4
        self._lib = _oracle_lib()
        self._h = self._lib.orc_mesh_new(_dp(self.vxyz), self.vxyz.shape[0], _ip(self.tet_v),
                                         _ip(self.tet_n), self.tet_v.shape[0])
        if not self._h:
            raise RuntimeError('orc_mesh_new failed')

    def set_predicates(self, mode):
        """'fast' (natinterp3d's signs), 'audit' (same signs, uncertain
        evaluations counted) or 'exact'."""
        if self._lib.orc_mesh_set_predicates(self._h, PREDICATE_MODES[mode]) != 0:
            raise ValueError(mode)

    def set_seed(self, first_tet):
        """Walk seed: the nearest tet centroid (natinterp3d's k-d tree seed, the
        default) or, with ``first_tet``, tet 0 (natinterp3d without its k-d tree)."""
        self._lib.orc_mesh_set_seed(self._h, int(bool(first_tet)))

    def predicate_info(self):
        """(tets with an uncertain orientation sign, tets whose flag the exact sign flips)"""
        out = (ctypes.c_long * 2)()
        self._lib.orc_mesh_predicate_info(self._h, out)
        return int(out[0]), int(out[1])

    def weights(self, queries_centered, with_stats=False):
        """CSR of Sibson weights (natinterp3d row/column order) for centred queries."""
        q = np.ascontiguousarray(queries_centered, np.float64).reshape(-1, 3)
        M = q.shape[0]
        rowptr = np.empty(M + 1, np.int32)
        vals_p, cols_p = c_double_p(), c_int_p()
        status = np.zeros(max(M, 1), np.int8)
        stats = np.zeros(len(STATS_FIELDS), np.int64)
        rc = self._lib.orc_weights(self._h, _dp(q), M, ctypes.byref(vals_p), ctypes.byref(cols_p),
                                   _ip(rowptr), status.ctypes.data_as(ctypes.POINTER(ctypes.c_byte)),
                                   stats.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
        if rc != 0:
            raise RuntimeError('orc_weights failed with status %d' % rc)
        W = _take_csr(self._lib.orc_free, vals_p, cols_p, rowptr, M, self.n_keys)
        if with_stats:
            return W, dict(zip(STATS_FIELDS, stats.tolist())), status[:M]
        return W

    def tet_geometry(self):
        T = self.tet_v.shape[0]
        pos = np.empty(T, np.uint8)
        tcc = np.empty((T, 3), np.float64)
        fcc = np.empty((T, 4, 3), np.float64)
        self._lib.orc_tet_geometry(self._h, pos.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                                   _dp(tcc), _dp(fcc))
        return pos, tcc, fcc

    def close(self):
        if getattr(self, '_h', None):
            self._lib.orc_mesh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spmm_like_scipy(W, x):
    """W @ x accumulated row by row in stored order, as scipy's csr_matvecs does."""
    lib = _oracle_lib()
    x = np.ascontiguousarray(x, np.float64)
    x2 = x.reshape(x.shape[0], -1)
    M, D = W.shape[0], x2.shape[1]
    y = np.empty((M, D), np.float64)
    lib.orc_spmm(M, D, _ip(np.ascontiguousarray(W.indptr, np.int32)),
                 _ip(np.ascontiguousarray(W.indices, np.int32)),
                 _dp(np.ascontiguousarray(W.data, np.float64)), _dp(x2), _dp(y))
    return y.reshape((M,) + x.shape[1:])


def orient(a, b, c, d):
    lib = _oracle_lib()
    arr = [np.ascontiguousarray(p, np.float64) for p in (a, b, c, d)]
    return lib.orc_orient(*[_dp(p) for p in arr])


def insphere(a, b, c, d, e):
    lib = _oracle_lib()
    arr = [np.ascontiguousarray(p, np.float64) for p in (a, b, c, d, e)]
    return lib.orc_insphere(*[_dp(p) for p in arr])


def _pts(*ps):
    arr = [np.ascontiguousarray(p, np.float64) for p in ps]
    return arr, [_dp(p) for p in arr]


def orient_exact_sign(a, b, c, d):
    keep, ptrs = _pts(a, b, c, d)
    return _oracle_lib().orc_orient_exact_sign(*ptrs)


def insphere_exact_sign(a, b, c, d, e):
    keep, ptrs = _pts(a, b, c, d, e)
    return _oracle_lib().orc_insphere_exact_sign(*ptrs)


def orient_uncertain(a, b, c, d):
    keep, ptrs = _pts(a, b, c, d)
    return bool(_oracle_lib().orc_orient_uncertain(*ptrs))


def insphere_uncertain(a, b, c, d, e):
    keep, ptrs = _pts(a, b, c, d, e)
    return bool(_oracle_lib().orc_insphere_uncertain(*ptrs))


# --------------------------------------------------------------------------
# natinterp3d's own code (oracle/_ref)
# --------------------------------------------------------------------------

def ref_available():
    return os.path.exists(build_oracle.REF_SO)


def _ref_lib():
    global _rlib
    if _rlib is None:
        path = build_oracle.REF_SO
        if not os.path.exists(path):
            build_oracle.build_ref()
        if not os.path.exists(path):
            raise RuntimeError('natinterp3d reference library not available')
        lib = ctypes.CDLL(path)
        lib.ref_build.argtypes = [c_double_p, ctypes.c_int, ctypes.POINTER(c_void_p),
                                  ctypes.POINTER(c_void_p)]
        lib.ref_build.restype = ctypes.c_int
        lib.ref_free.argtypes = [c_void_p, c_void_p]
        lib.ref_free.restype = None
        lib.ref_num_tets.argtypes = [c_void_p]
        lib.ref_num_tets.restype = ctypes.c_int
        lib.ref_query.argtypes = [c_void_p, c_double_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(c_double_p), ctypes.POINTER(c_int_p), c_int_p]
        lib.ref_query.restype = ctypes.c_int
        lib.ref_free_buffer.argtypes = [c_void_p]
        lib.ref_free_buffer.restype = None
        if hasattr(lib, 'ref_orient3d_robust'):
            lib.ref_orient3d_robust.argtypes = [c_double_p] * 4
            lib.ref_orient3d_robust.restype = ctypes.c_double
            lib.ref_insphere_robust.argtypes = [c_double_p] * 5
            lib.ref_insphere_robust.restype = ctypes.c_double
        _rlib = lib
    return _rlib


def ref_query(native_mesh_ptr, queries_centered, n_keys, nthreads=0):
    """natinterp3d's getInsertionFreeWeights[Parallel] on a natinterp3d mesh object."""
    lib = _ref_lib()
    q = np.ascontiguousarray(queries_centered, np.float64).reshape(-1, 3)
    M = q.shape[0]
    rowptr = np.empty(M + 1, np.int32)
    vals_p, cols_p = c_double_p(), c_int_p()
    rc = lib.ref_query(native_mesh_ptr, _dp(q), M, int(nthreads), int(n_keys),
                       ctypes.byref(vals_p), ctypes.byref(cols_p), _ip(rowptr))
    if rc != 0:
        raise OverflowError('Total number of nonzero weights exceeds int32 limit')
    return _take_csr(lib.ref_free_buffer, vals_p, cols_p, rowptr, M, n_keys)


def ref_orient3d_robust(a, b, c, d):
    """Shewchuk's adaptive exact orient3d as shipped (and never called) by natinterp3d."""
    keep, ptrs = _pts(a, b, c, d)
    return _ref_lib().ref_orient3d_robust(*ptrs)


def ref_insphere_robust(a, b, c, d, e):
    keep, ptrs = _pts(a, b, c, d, e)
    return _ref_lib().ref_insphere_robust(*ptrs)


class RefInterpolator:
    """natinterp3d's Interpolator, restated over the reference library: the
    key centroid is subtracted in numpy exactly as natinterp3d.py:88-90, 115."""

    def __init__(self, keys, num_threads=None):
        keys = np.ascontiguousarray(keys, np.float64)
        self.n_keys = keys.shape[0]
        self.centroid = keys.mean(axis=0)
        centered = keys - self.centroid
        if num_threads is None:
            try:
                num_threads = len(os.sched_getaffinity(0))
            except AttributeError:
                num_threads = os.cpu_count() or 1
        self.num_threads = num_threads
        self._lib = _ref_lib()
        self._m, self._ps = c_void_p(), c_void_p()
        self._lib.ref_build(_dp(centered), self.n_keys, ctypes.byref(self._m), ctypes.byref(self._ps))

    def get_weights(self, queries):
        out_dtype = queries.dtype
        q = np.ascontiguousarray(queries, np.float64) - self.centroid
        W = ref_query(self._m, q, self.n_keys, self.num_threads)
        return W.astype(out_dtype, copy=False)

    def interpolate(self, queries, values):
        W = self.get_weights(queries)
        if values.ndim == 1:
            return np.squeeze(W @ values[:, np.newaxis], axis=1)
        return W @ values

    def close(self):
        if getattr(self, '_m', None) is not None and self._m.value:
            self._lib.ref_free(self._m, self._ps)
            self._m = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
