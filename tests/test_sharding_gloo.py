"""Multi-process (world size 2, gloo, CPU) tests of the sharding host logic.

The rows are computed by the CPU oracle here (no GPU in these tests); on a
GPU box the same functions take the CUDA interpolator as the row function."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse
import torch.multiprocessing as mp

from natinterp3d_b200.sharding import shard_bounds


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, keys, queries, values, out_dir):
    import torch
    import torch.distributed as dist
    from natinterp3d_b200.sharding import broadcast_mesh, sharded_interpolate, sharded_weights
    from oracle import oracle
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        it = broadcast_mesh(keys if rank == 0 else None)
        om = oracle.OracleMesh(*it.mesh_arrays)
        c = it.centroid

        def rows(q):
            W = om.weights(np.asarray(q) - c)
            return W.indptr, W.indices, W.data

        def interp(q):
            rp, cc, vv = rows(q)
            W = scipy.sparse.csr_matrix((vv, cc, rp), shape=(len(q), len(keys)))
            return torch.from_numpy(oracle.spmm_like_scipy(W, values))

        lo, rowptr, cols, vals, total = sharded_weights(queries, rows)
        _, full = sharded_interpolate(queries, interp, gather=True)
        np.savez(os.path.join(out_dir, 'r%d.npz' % rank), lo=lo, rowptr=rowptr, cols=cols, vals=vals,
                 total=total, full=full.numpy(), vx=it.mesh_arrays[0], tv=it.mesh_arrays[1],
                 cen=c)
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_everything():
    for M in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            b = [shard_bounds(M, r, world) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == M
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in b]
            assert max(sizes) - min(sizes) <= 1


def test_two_rank_gloo_sharded_rows_equal_single_process(tmp_path):
    from oracle import oracle
    from natinterp3d_b200._native import HostMesh
    rng = np.random.default_rng(0)
    keys = rng.uniform(0, 1, (1500, 3))
    queries = rng.uniform(0.05, 0.95, (2001, 3))
    values = rng.standard_normal((1500, 2))
    port = _free_port()
    ctx = mp.get_context('spawn')
    procs = [ctx.Process(target=_worker, args=(r, 2, port, keys, queries, values, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / ('r%d.npz' % r)) for r in range(2))
    # identical mesh on both ranks (broadcast from rank 0)
    assert np.array_equal(r0['vx'], r1['vx']) and np.array_equal(r0['tv'], r1['tv'])
    # stitched CSR equals the single-process oracle on the same mesh
    c = keys.mean(axis=0)
    ref = oracle.OracleMesh(*HostMesh(keys - c).export()).weights(queries - c)
    rowptr = np.concatenate([r0['rowptr'][:-1], r1['rowptr']])
    assert int(r0['total']) == int(r1['total']) == ref.nnz
    assert np.array_equal(rowptr, ref.indptr)
    assert np.array_equal(np.concatenate([r0['cols'], r1['cols']]), ref.indices)
    assert np.array_equal(np.concatenate([r0['vals'], r1['vals']]), ref.data)
    assert np.array_equal(r0['full'], oracle.spmm_like_scipy(ref, values))
    assert np.array_equal(r0['full'], r1['full'])
