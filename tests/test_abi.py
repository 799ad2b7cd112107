"""The C ABI: both shared libraries load without a GPU and export every
symbol include/natinterp3d_b200.h declares; host-side argument checks."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, 'include', 'natinterp3d_b200.h')


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\b(nif_[a-z0-9_]+)\s*\(', src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert 'nif_weights_count' in names and 'nif_mesh_build' in names and len(names) >= 14


def test_libraries_export_every_declared_symbol():
    from natinterp3d_b200 import _native
    mesh = _native.mesh_lib()
    cuda = _native.cuda_lib()
    missing = [n for n in declared_functions()
               if not hasattr(mesh if n.startswith('nif_mesh_') else cuda, n)]
    assert not missing, missing
    assert set(_native.CUDA_SIGNATURES) | set(_native.MESH_SIGNATURES) == set(declared_functions())


def test_cuda_size_queries_without_gpu():
    from natinterp3d_b200 import _native
    lib = _native.cuda_lib()
    nb = ctypes.c_size_t()
    assert lib.nif_dmesh_bytes(1004, 6480, ctypes.byref(nb)) == 0
    # vertices + tets + circumcentres + seed grid
    assert nb.value > 6480 * (16 + 16 + 4 + 32 + 128) + 1004 * 32
    assert lib.nif_dmesh_bytes(3, 10, ctypes.byref(nb)) == _native.NIF_ERR_ARG
    assert lib.nif_dmesh_create(None, None, None, 10, 10, None, 0, None,
                                ctypes.byref(ctypes.c_void_p())) == _native.NIF_ERR_ARG
    assert lib.nif_query_workspace_bytes(None, 10, 0, ctypes.byref(nb)) == _native.NIF_ERR_ARG


def test_records_size_matches_the_header():
    # the header documents 788 bytes a row of kept cavity records: a 16-byte
    # head, 48 entries of 16 bytes and a 4-byte slot of the wide-row queue
    from natinterp3d_b200 import _native
    lib = _native.cuda_lib()
    nb = ctypes.c_size_t()
    M = 1_000_000
    assert lib.nif_records_bytes(M, ctypes.byref(nb)) == 0
    assert 788 * M <= nb.value <= 788 * M + 4096
    assert lib.nif_records_bytes(0, ctypes.byref(nb)) == 0 and nb.value <= 4096
    assert lib.nif_records_bytes(-1, ctypes.byref(nb)) == _native.NIF_ERR_ARG


def test_mesh_export_is_consistent():
    from natinterp3d_b200._native import HostMesh
    rng = np.random.default_rng(0)
    keys = rng.uniform(0, 1, (500, 3))
    hm = HostMesh(keys - keys.mean(0))
    vxyz, tv, tn = hm.export()
    assert vxyz.shape == (504, 3) and tv.shape == tn.shape and tv.shape[1] == 4
    assert tv.min() >= 0 and tv.max() < 504
    assert np.array_equal(vxyz[:500], keys - keys.mean(0))  # no perturbation on random data
    # neighbour relation is symmetric and faces match (face f opposite p[3-f])
    face = [(0, 1, 2), (3, 1, 0), (0, 2, 3), (3, 2, 1)]
    for t in range(tv.shape[0]):
        for f in range(4):
            nb = tn[t, f]
            if nb < 0:
                continue
            assert t in tn[nb]
            assert set(tv[t, list(face[f])]) <= set(tv[nb])


def test_degenerate_keys_rejected():
    from natinterp3d_b200._native import HostMesh
    with pytest.raises(ValueError):
        HostMesh(np.zeros((5, 3)))
    flat = np.random.default_rng(0).uniform(0, 1, (20, 3))
    flat[:, 2] = 0.5
    with pytest.raises(ValueError):
        HostMesh(flat)
    with pytest.raises(ValueError):
        HostMesh(np.zeros((5, 2)))


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    """nif_summary and nif_tuning as the C compiler lays them out from the
    header, against the ctypes structures the package passes to the library."""
    import shutil
    import subprocess
    from natinterp3d_b200 import _native
    cc = shutil.which('gcc') or shutil.which('cc')
    if cc is None:
        pytest.skip('no C compiler')
    src = tmp_path / 'layout.c'
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "natinterp3d_b200.h"\n'
        'int main(void) {\n'
        '  printf("%zu %zu %zu %zu\\n", sizeof(nif_summary), offsetof(nif_summary, first_status),\n'
        '         offsetof(nif_summary, orient_uncertain), offsetof(nif_summary, insphere_flipped));\n'
        '  printf("%zu %zu %zu\\n", sizeof(nif_tuning), offsetof(nif_tuning, bucket_shift),\n'
        '         offsetof(nif_tuning, tile));\n'
        '  return 0;\n}\n')
    exe = tmp_path / 'layout'
    subprocess.run([cc, '-I', os.path.join(ROOT, 'include'), str(src), '-o', str(exe)], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split('\n')
    S, T = _native.Summary, _native.Tuning
    assert [int(x) for x in lines[0].split()] == [
        ctypes.sizeof(S), S.first_status.offset, S.orient_uncertain.offset, S.insphere_flipped.offset]
    assert [int(x) for x in lines[1].split()] == [
        ctypes.sizeof(T), T.bucket_shift.offset, T.tile.offset]
