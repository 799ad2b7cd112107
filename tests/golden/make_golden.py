"""Generates the golden fixtures in this directory from natinterp3d itself.

For every case the key set is triangulated by natinterp3d's own constructor
(through the product's constructor library, which compiles natinterp3d's
sources), the mesh is exported, and natinterp3d's own query code
(``oracle/_ref``, natinterp3d's sources compiled in place) computes the CSR
weights on exactly that mesh object.  The fixture stores the inputs, the
exported mesh and natinterp3d's CSR arrays, so a GPU run can upload the same
mesh and compare bit for bit without natinterp3d being present.

Run from the repository root where the natinterp3d sources are available:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from natinterp3d_b200._native import HostMesh  # noqa: E402
from oracle import oracle  # noqa: E402


def lattice_mixture(rng, g, n_mix, n_comp):
    lat = np.stack(np.meshgrid(*[np.arange(g)] * 3, indexing='ij'), -1).reshape(-1, 3) / g
    means = rng.uniform(0, 1, (n_comp, 3))
    mix = np.clip(means[rng.integers(0, n_comp, n_mix)] + rng.normal(0, 0.01, (n_mix, 3)), 0, 1)
    return np.concatenate([lat, mix]), means


def cases():
    rng = np.random.default_rng(0)
    keys = rng.uniform(0, 1, (2000, 3))
    q = rng.uniform(0.05, 0.95, (4000, 3))
    yield 'uniform_2k', keys, q

    rng = np.random.default_rng(3)
    keys, means = lattice_mixture(rng, 10, 600, 8)
    half = 1500
    q = np.concatenate([rng.uniform(1 / 10, 1 - 2 / 10, (half, 3)),
                        np.clip(means[rng.integers(0, 8, half)] + rng.normal(0, 0.01, (half, 3)), 0, 1)])
    yield 'lattice_mixture', keys, q

    cube = np.array([[-1, -1, -1], [-1, -1, 1], [-1, 1, -1], [-1, 1, 1],
                     [1, -1, -1], [1, -1, 1], [1, 1, -1], [1, 1, 1]], np.float64)
    yield 'cube_centre', cube, np.zeros((1, 3))
    octa = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float64)
    yield 'octahedron_centre', octa, np.zeros((1, 3))
    tet = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], np.float64)
    yield 'regular_tet_centroid', tet, tet.mean(axis=0, keepdims=True)
    five = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0.5, 0.5]], np.float64)
    yield 'five_points', five, np.array([[0.2, 0.2, 0.2], [0.1, 0.3, 0.2]])

    r = np.random.RandomState(33)
    keys = r.randn(60, 3)
    yield 'queries_at_keys', keys, np.concatenate([keys, keys[::3] + 1e-9])

    r = np.random.RandomState(20)
    keys = r.randn(100, 3)
    yield 'outside', keys, np.array([[100.0, 100.0, 100.0], [-100.0, -100.0, -100.0],
                                     [4.0, 4.0, 4.0], [3.0, 0.0, 0.0], [0.0, 0.0, 0.0]])

    xs = np.linspace(-1, 1, 6)
    grid = np.array(np.meshgrid(xs, xs, xs)).reshape(3, -1).T
    r = np.random.RandomState(7)
    yield 'grid6', grid, np.concatenate([r.uniform(-0.8, 0.8, (300, 3)), grid[::5]])

    r = np.random.RandomState(88)
    off = np.array([1e6, -2e6, 3e6])
    keys = r.randn(300, 3) + off
    yield 'large_offset', keys, keys.mean(0) + r.randn(200, 3) * keys.std(0) * 0.24
    r = np.random.RandomState(89)
    keys = r.randn(300, 3) * 1e4
    yield 'large_scale', keys, keys.mean(0) + r.randn(200, 3) * keys.std(0) * 0.24
    r = np.random.RandomState(90)
    keys = r.randn(300, 3) * 1e-4
    yield 'small_scale', keys, keys.mean(0) + r.randn(200, 3) * keys.std(0) * 0.24

    r = np.random.RandomState(51)
    keys = r.randn(400, 3).astype(np.float32)
    yield 'float32', keys, (r.randn(500, 3) * 0.3).astype(np.float32)


def main():
    out_dir = HERE
    for name, keys, queries in cases():
        keys64 = np.ascontiguousarray(keys, np.float64)
        centroid = keys64.mean(axis=0)
        hm = HostMesh(keys64 - centroid)
        vxyz, tet_v, tet_n = hm.export()
        qc = np.ascontiguousarray(queries, np.float64) - centroid
        W = oracle.ref_query(hm.native_pointer(), qc, keys.shape[0], nthreads=1)
        values = np.sin(3 * keys64[:, 0]) + np.cos(2 * keys64[:, 1]) * keys64[:, 2]
        vals2 = np.stack([keys64[:, 0], 2 * keys64[:, 1] - keys64[:, 2] + 1.0], axis=1)
        np.savez_compressed(
            os.path.join(out_dir, name + '.npz'),
            keys=keys, queries=queries, centroid=centroid, vxyz=vxyz, tet_v=tet_v, tet_n=tet_n,
            indptr=W.indptr, indices=W.indices, data=W.data,
            values=values, interp=W @ values[:, None], values2=vals2, interp2=W @ vals2,
            degeneracies=np.array([hm.degeneracies()['coplanar'], hm.degeneracies()['cospherical']]))
        hm.close()
        print('%-22s keys %5d queries %5d tets %6d nnz %7d' % (name, keys.shape[0], queries.shape[0],
                                                             tet_v.shape[0], W.nnz))


if __name__ == '__main__':
    main()
