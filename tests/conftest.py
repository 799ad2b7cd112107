import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200); parity tests through the C ABI')


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(GOLDEN_DIR, '*.npz')))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN_DIR, name + '.npz'))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope='session')
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail('GPU test selected but no CUDA device is visible')
    return torch.device('cuda', 0)


def dyadic_keys(seed=0, n=1024, bits=10):
    """n distinct keys on a 2^-bits grid (n a power of two, so the key centroid
    and the centred coordinates are exact doubles)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 1 << bits, (4 * n, 3))
    _, idx = np.unique(k, axis=0, return_index=True)
    k = k[np.sort(idx)[:n]]
    assert len(k) == n
    return k.astype(np.float64) / (1 << bits)


def on_face_queries(vxyz, tet_v, n_keys, count=300, seed=1):
    """Centred queries lying exactly on mesh edges, faces and vertices: dyadic
    convex combinations of vertices of interior tets (exact when the vertices
    are short dyadic numbers), plus a few generic interior points."""
    rng = np.random.default_rng(seed)
    inner = np.where((tet_v < n_keys).all(axis=1))[0]
    ts = rng.choice(inner, count, replace=False)
    P = vxyz[tet_v[ts]]
    edge = 0.5 * P[:, 0] + 0.5 * P[:, 1]
    face = 0.5 * P[:, 0] + 0.25 * P[:, 1] + 0.25 * P[:, 2]
    vert = P[:count // 3, 3]
    generic = P.mean(axis=1)
    return np.concatenate([edge, face, vert, generic])
