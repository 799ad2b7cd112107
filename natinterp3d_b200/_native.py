"""ctypes bindings for the two native libraries (C ABI in include/natinterp3d_b200.h).

The libraries are loaded from ``natinterp3d_b200/lib``.  A missing CUDA
library is an error, never a silent fallback: there is no CPU query path in
this package.
"""
import ctypes
import os

import numpy as np

from . import _build

c_int = ctypes.c_int
c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_void_p = ctypes.c_void_p
c_double_p = ctypes.POINTER(ctypes.c_double)
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_size_t = ctypes.c_size_t

# status codes shared by both libraries (include/natinterp3d_b200.h)
NIF_OK = 0
NIF_ERR_ARG = -1
NIF_ERR_DEGENERATE = -2
NIF_ERR_NOMEM = -3
NIF_ERR_INTERNAL = -4
NIF_ERR_OVERFLOW = -5
NIF_ERR_WALK = -6
NIF_ERR_CUDA = -7
NIF_ERR_CAPACITY = -8
NIF_ERR_WORKSPACE = -9
NIF_ERR_TOO_LARGE = -10

_ERR_NAMES = {
    NIF_ERR_ARG: 'invalid argument',
    NIF_ERR_DEGENERATE: 'degenerate key set',
    NIF_ERR_NOMEM: 'out of memory',
    NIF_ERR_INTERNAL: 'internal error',
    NIF_ERR_OVERFLOW: 'nnz overflow',
    NIF_ERR_WALK: 'point-location walk step limit reached',
    NIF_ERR_CUDA: 'CUDA error',
    NIF_ERR_CAPACITY: 'per-query capacity exceeded',
    NIF_ERR_WORKSPACE: 'workspace too small',
    NIF_ERR_TOO_LARGE: 'more queries than the fixed scratch holds',
}


class NativeError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        super().__init__('%s failed: %s (status %d)' % (what, _ERR_NAMES.get(code, 'error'), code))


def check(code, what):
    if code != NIF_OK:
        raise NativeError(code, what)


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


# --------------------------------------------------------------------------
# host mesh constructor
# --------------------------------------------------------------------------
_mesh_lib = None


def mesh_lib():
    global _mesh_lib
    if _mesh_lib is None:
        path = _build.MESH_SO
        if not os.path.exists(path):
            path = _build.build_mesh_lib()
        lib = ctypes.CDLL(path)
        lib.nif_mesh_build.argtypes = [c_double_p, c_int, ctypes.POINTER(c_void_p)]
        lib.nif_mesh_build.restype = c_int
        lib.nif_mesh_free.argtypes = [c_void_p]
        lib.nif_mesh_free.restype = None
        lib.nif_mesh_sizes.argtypes = [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]
        lib.nif_mesh_sizes.restype = c_int
        lib.nif_mesh_export.argtypes = [c_void_p, c_double_p, c_int32_p, c_int32_p]
        lib.nif_mesh_export.restype = c_int
        lib.nif_mesh_degeneracies.argtypes = [c_void_p, ctypes.POINTER(c_int),
                                              ctypes.POINTER(c_int)]
        lib.nif_mesh_degeneracies.restype = c_int
        lib.nif_mesh_native.argtypes = [c_void_p]
        lib.nif_mesh_native.restype = c_void_p
        _mesh_lib = lib
    return _mesh_lib


class HostMesh:
    """natinterp3d's Delaunay mesh of a (centred) key set, built on the host.

    Owns the natinterp3d mesh object; ``export()`` returns the packed arrays
    (vxyz [N+4, 3] float64, tet_v [T, 4] int32, tet_n [T, 4] int32).
    """

    def __init__(self, keys_centered):
        keys = np.ascontiguousarray(keys_centered, dtype=np.float64)
        if keys.ndim != 2 or keys.shape[1] != 3:
            raise ValueError('Data points must have shape (num_data_points, 3)')
        self._lib = mesh_lib()
        self._h = c_void_p()
        self.n = int(keys.shape[0])
        rc = self._lib.nif_mesh_build(_ptr(keys, ctypes.c_double), self.n, ctypes.byref(self._h))
        if rc == NIF_ERR_DEGENERATE or rc == NIF_ERR_ARG:
            raise ValueError('natinterp3d cannot triangulate this key set: it needs at least one '
                             'point and a non-zero, finite extent along every axis')
        check(rc, 'nif_mesh_build')
        nv, nt = c_int(), c_int()
        check(self._lib.nif_mesh_sizes(self._h, ctypes.byref(nv), ctypes.byref(nt)),
              'nif_mesh_sizes')
        self.n_vertices, self.n_tets = nv.value, nt.value

    def export(self):
        vxyz = np.empty((self.n_vertices, 3), np.float64)
        tet_v = np.empty((self.n_tets, 4), np.int32)
        tet_n = np.empty((self.n_tets, 4), np.int32)
        check(self._lib.nif_mesh_export(self._h, _ptr(vxyz, ctypes.c_double),
                                         _ptr(tet_v, ctypes.c_int32), _ptr(tet_n, ctypes.c_int32)),
              'nif_mesh_export')
        return vxyz, tet_v, tet_n

    def degeneracies(self):
        a, b = c_int(), c_int()
        check(self._lib.nif_mesh_degeneracies(self._h, ctypes.byref(a), ctypes.byref(b)),
              'nif_mesh_degeneracies')
        return {'coplanar': a.value, 'cospherical': b.value}

    def native_pointer(self):
        return self._lib.nif_mesh_native(self._h)

    def close(self):
        if getattr(self, '_h', None) is not None and self._h.value:
            self._lib.nif_mesh_free(self._h)
            self._h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# device library
# --------------------------------------------------------------------------
NIF_F64 = 0
NIF_F32 = 1
NIF_MODE_WEIGHTS = 0
NIF_MODE_INTERP = 1
# predicate modes (nif_dmesh_set_predicates)
PREDICATE_MODES = {'fast': 0, 'audit': 1, 'exact': 2}


class Summary(ctypes.Structure):
    _fields_ = [('nnz', ctypes.c_int64), ('rows_large', ctypes.c_int64),
                ('rows_failed', ctypes.c_int64), ('rows_outside', ctypes.c_int64),
                ('walk_steps', ctypes.c_int64), ('first_status', ctypes.c_int32),
                ('rows_wide', ctypes.c_int32), ('orient_uncertain', ctypes.c_int64),
                ('orient_flipped', ctypes.c_int64), ('insphere_uncertain', ctypes.c_int64),
                ('insphere_flipped', ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

    @classmethod
    def from_dict(cls, d):
        s = cls()
        for k, _ in cls._fields_:
            if k in d:
                setattr(s, k, int(d[k]))
        return s


class DelaunayInfo(ctypes.Structure):
    """nif_delaunay_info: outcome and exact checks of a GPU construction."""
    _fields_ = [('n_tets', ctypes.c_int64), ('rounds', ctypes.c_int32),
                ('max_cavity', ctypes.c_int32), ('exact_evaluations', ctypes.c_int64),
                ('tet_slots', ctypes.c_int32), ('error', ctypes.c_int32),
                ('bad_orientation', ctypes.c_int64), ('bad_adjacency', ctypes.c_int64),
                ('non_delaunay_faces', ctypes.c_int64), ('cospherical_faces', ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(ctypes.Structure):
    """nif_tuning: launch settings of the query kernels (speed only, never results)."""
    _fields_ = [('blocks_per_sm', ctypes.c_int32), ('bucket_shift', ctypes.c_int32),
                ('tile', ctypes.c_int32), ('reserved', ctypes.c_int32)]

    def as_dict(self):
        return {'blocks_per_sm': self.blocks_per_sm, 'bucket_shift': self.bucket_shift,
                'tile': self.tile}

    @classmethod
    def from_dict(cls, d):
        return cls(int(d['blocks_per_sm']), int(d.get('bucket_shift', 0)), int(d.get('tile', 0)), 0)


# every symbol include/natinterp3d_b200.h declares for libnif_cuda.so, with its ctypes signature
CUDA_SIGNATURES = {
    'nif_dmesh_bytes': (c_int, [c_int, c_int, ctypes.POINTER(c_size_t)]),
    'nif_dmesh_create': (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_size_t,
                                 c_void_p, ctypes.POINTER(c_void_p)]),
    'nif_dmesh_destroy': (None, [c_void_p]),
    'nif_dmesh_info': (c_int, [c_void_p, ctypes.POINTER(c_int64)]),
    'nif_dmesh_set_predicates': (c_int, [c_void_p, c_int]),
    'nif_dmesh_set_tuning': (c_int, [c_void_p, ctypes.POINTER(Tuning)]),
    'nif_dmesh_get_tuning': (c_int, [c_void_p, ctypes.POINTER(Tuning)]),
    'nif_query_workspace_bytes': (c_int, [c_void_p, c_int64, c_int, ctypes.POINTER(c_size_t)]),
    'nif_weights_count': (c_int, [c_void_p, c_void_p, c_int, c_int64, c_double_p, c_void_p,
                                  c_size_t, c_void_p, c_void_p, ctypes.POINTER(Summary)]),
    'nif_weights_fill': (c_int, [c_void_p, c_void_p, c_int, c_int64, c_double_p, c_void_p, c_size_t,
                                 c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    'nif_interpolate': (c_int, [c_void_p, c_void_p, c_int, c_int64, c_double_p, c_void_p, c_int,
                                c_int, c_void_p, c_int, c_void_p, c_size_t, c_void_p,
                                ctypes.POINTER(Summary)]),
    'nif_profile_enable': (c_int, [c_int]),
    'nif_profile_read': (c_int, [c_double_p]),
    'nif_profile_kernels': (c_int, [c_double_p, c_double_p]),
    'nif_measure_fp64_peak': (c_int, [c_double_p, c_double_p]),
    'nif_query_summary': (c_int, [c_void_p, c_int64, c_int, c_void_p, c_size_t, c_void_p,
                                  ctypes.POINTER(Summary)]),
    'nif_spmm': (c_int, [c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                         c_int, c_void_p, c_int, c_void_p]),
    'nif_spmm_t_workspace_bytes': (c_int, [c_int64, c_int64, c_int64, ctypes.POINTER(c_size_t)]),
    'nif_spmm_t': (c_int, [c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                           c_int, c_int, c_void_p, c_int, c_void_p, c_size_t, c_void_p]),
    'nif_spmm_t_ordered': (c_int, [c_int64, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_int,
                                   c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                   c_size_t, c_void_p]),
    'nif_query_grad': (c_int, [c_void_p, c_void_p, c_int, c_int64, c_double_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                               c_void_p, c_size_t, c_void_p, ctypes.POINTER(Summary)]),
    'nif_records_bytes': (c_int, [c_int64, ctypes.POINTER(c_size_t)]),
    'nif_delaunay_max_tets': (c_int, [c_int, ctypes.POINTER(c_int)]),
    'nif_delaunay_workspace_bytes': (c_int, [c_int, ctypes.POINTER(c_size_t)]),
    'nif_delaunay_build': (c_int, [c_void_p, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p,
                                   c_int, c_void_p, ctypes.POINTER(DelaunayInfo)]),
    'nif_weights_count_records': (c_int, [c_void_p, c_void_p, c_int, c_int64, c_double_p, c_void_p,
                                          c_size_t, c_void_p, c_void_p, c_size_t, c_void_p,
                                          ctypes.POINTER(Summary)]),
    'nif_query_grad_records': (c_int, [c_void_p, c_void_p, c_int, c_int64, c_double_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_int,
                                       c_void_p, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p,
                                       ctypes.POINTER(Summary)]),
    'nif_batch_bytes': (c_int, [c_int, ctypes.POINTER(c_size_t)]),
    'nif_batch_create': (c_int, [c_int, ctypes.POINTER(c_void_p), c_void_p, c_size_t, c_void_p,
                                 ctypes.POINTER(c_void_p)]),
    'nif_batch_destroy': (None, [c_void_p]),
    'nif_batch_workspace_bytes': (c_int, [c_void_p, c_int64, ctypes.POINTER(c_size_t)]),
    'nif_batch_set_tuning': (c_int, [c_void_p, ctypes.POINTER(Tuning)]),
    'nif_batch_get_tuning': (c_int, [c_void_p, ctypes.POINTER(Tuning)]),
    'nif_batch_interpolate': (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int,
                                      c_void_p, c_int, c_void_p, c_int, c_int64, c_void_p, c_size_t,
                                      c_void_p]),
    'nif_batch_summary': (c_int, [c_void_p, c_int64, c_void_p, c_size_t, c_void_p,
                                  ctypes.POINTER(Summary)]),
    'nif_interpolate_noalloc': (c_int, [c_void_p, c_void_p, c_int, c_int64, c_double_p, c_void_p,
                                        c_int, c_int, c_void_p, c_int, c_void_p,
                                        ctypes.POINTER(Summary)]),
}

MESH_SIGNATURES = ('nif_mesh_build', 'nif_mesh_free', 'nif_mesh_sizes', 'nif_mesh_export',
                   'nif_mesh_degeneracies', 'nif_mesh_native')

_cuda_lib = None


def cuda_lib():
    """libnif_cuda.so; raises if it is missing (there is no CPU query path)."""
    global _cuda_lib
    if _cuda_lib is None:
        path = _build.CUDA_SO
        if not os.path.exists(path):
            raise RuntimeError('natinterp3d_b200 CUDA library not built (%s); run '
                               'python -m natinterp3d_b200._build' % path)
        lib = ctypes.CDLL(path)
        for name, (res, args) in CUDA_SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _cuda_lib = lib
    return _cuda_lib
