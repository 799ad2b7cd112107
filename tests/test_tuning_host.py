"""Host side of the launch settings: the candidate lists stay inside the
ranges nif_dmesh_set_tuning / nif_batch_set_tuning accept, the ctypes mirror
of nif_tuning has the C layout, and the tuning cache round-trips.  Also the
chunking of pipelined host calls."""
import ctypes

from natinterp3d_b200 import _native as N
from natinterp3d_b200 import tuning


def test_candidates_in_range():
    for c in tuning.MESH_CANDIDATES:
        assert c['blocks_per_sm'] in (6, 8) and -2 <= c['bucket_shift'] <= 1
        assert 0 <= c['tile'] <= 1024
    for c in tuning.BATCH_CANDIDATES:
        assert c['blocks_per_sm'] in (6, 8) and 1 <= c['tile'] <= 1024
    assert len({tuple(sorted(c.items())) for c in tuning.MESH_CANDIDATES}) == 18


def test_tuning_struct_layout():
    assert ctypes.sizeof(N.Tuning) == 16
    t = N.Tuning.from_dict({'blocks_per_sm': 6, 'tile': 32, 'bucket_shift': -1})
    assert t.as_dict() == {'blocks_per_sm': 6, 'tile': 32, 'bucket_shift': -1} and t.reserved == 0


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setenv('NATINTERP3D_B200_TUNING', str(tmp_path / 'sub' / 'tuning.json'))
    assert tuning._load_cache() == {}
    tuning._store_cache('k1', {'tuning': tuning.MESH_CANDIDATES[4]})
    tuning._store_cache('k2', {'tuning': tuning.BATCH_CANDIDATES[1]})
    data = tuning._load_cache()
    assert data['k1']['tuning'] == tuning.MESH_CANDIDATES[4]
    assert data['k2']['tuning'] == tuning.BATCH_CANDIDATES[1]
    assert tuning._p2(1) == 0 and tuning._p2(1_000_000) == 20


def test_pipeline_bounds_cover_rows_in_order():
    from natinterp3d_b200.natinterp3d import pipeline_bounds
    chunk = 1 << 21
    for M in (1, 7, chunk // 8, chunk, 2 * chunk + 12345, 10_000_000, 3 * chunk):
        b = pipeline_bounds(M, chunk)
        assert b[0][0] == 0 and b[-1][1] == M
        assert all(b[i][1] == b[i + 1][0] for i in range(len(b) - 1))
        assert all(0 < y - x <= chunk for x, y in b)
    b = pipeline_bounds(10_000_000, chunk)
    assert b[0] == (0, chunk // 8) and b[-1][1] - b[-1][0] == chunk // 8
