"""Multi-process (world size 2, gloo, CPU) tests of the sharding host logic.

The rows are computed by the CPU oracle here (no GPU in these tests); on a
GPU box the same functions take the CUDA interpolator as the row function."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse
import torch.multiprocessing as mp

from natinterp3d_b200.sharding import shard_bounds, shard_problems


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


def _grad_worker(rank, world, port, W_dense, g, v0, out_dir):
    import torch
    import torch.distributed as dist
    from natinterp3d_b200.sharding import allreduce_grad, shard_bounds
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        lo, hi = shard_bounds(W_dense.shape[0], rank, world)
        v = torch.from_numpy(v0.copy()).requires_grad_(True)
        Wl = torch.from_numpy(W_dense[lo:hi])
        out = Wl @ allreduce_grad(v)          # this rank's rows of W @ v
        (out * torch.from_numpy(g[lo:hi])).sum().backward()
        np.save(os.path.join(out_dir, 'g%d.npy' % rank), v.grad.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_values_gradient_is_summed_over_shards(tmp_path):
    """Each rank differentiates its own query rows; allreduce_grad leaves every
    rank with d loss / d values of the whole batch, W^T g."""
    from oracle import oracle
    from natinterp3d_b200._native import HostMesh
    rng = np.random.default_rng(3)
    keys = rng.uniform(0, 1, (400, 3))
    q = rng.uniform(0.1, 0.9, (301, 3))
    c = keys.mean(axis=0)
    W = oracle.OracleMesh(*HostMesh(keys - c).export()).weights(q - c).toarray()
    g = rng.standard_normal((301, 2))
    v0 = rng.standard_normal((400, 2))
    port = _free_port()
    ctx = mp.get_context('spawn')
    procs = [ctx.Process(target=_grad_worker, args=(r, 2, port, W, g, v0, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    g0, g1 = (np.load(tmp_path / ('g%d.npy' % r)) for r in range(2))
    assert np.array_equal(g0, g1)
    np.testing.assert_allclose(g0, W.T @ g, rtol=1e-12, atol=1e-12)


def test_shard_problems_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(np.log(1e3), np.log(2e5), 512)).astype(int)
    for world in (1, 2, 3, 8):
        parts = shard_problems(costs, world)
        assert sorted(p for part in parts for p in part) == list(range(512))
        loads = [costs[part].sum() for part in parts]
        assert max(loads) - min(loads) <= costs.max()
        assert all(part == sorted(part) for part in parts)
    assert shard_problems([5, 1], 4) == [[0], [1], [], []]


class _OracleBatch:
    """A batch_factory for CPU tests: the oracle in place of the GPU batch."""

    def __init__(self, keys_list):
        from oracle import oracle
        from natinterp3d_b200._native import HostMesh
        self.items = []
        for k in keys_list:
            c = k.mean(axis=0)
            self.items.append((c, oracle.OracleMesh(*HostMesh(k - c).export())))

    def interpolate(self, queries_list, values_list):
        from oracle import oracle
        return [oracle.spmm_like_scipy(om.weights(q - c), v)
                for (c, om), q, v in zip(self.items, queries_list, values_list)]


def _batch_worker(rank, world, port, keys_list, q_list, v_list, out_dir):
    import pickle
    import torch.distributed as dist
    from natinterp3d_b200.sharding import sharded_batch_interpolate
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        full = sharded_batch_interpolate(keys_list, q_list, v_list, batch_factory=_OracleBatch)
        with open(os.path.join(out_dir, 'b%d.pkl' % rank), 'wb') as f:
            pickle.dump(full, f)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_problem_sharded_batch(tmp_path):
    import pickle
    from natinterp3d_b200._native import HostMesh
    from oracle import oracle
    rng = np.random.default_rng(9)
    keys_list = [rng.uniform(0, 1, (n, 3)) for n in (300, 120, 500, 80, 260)]
    q_list = [rng.uniform(0.1, 0.9, (m, 3)) for m in (400, 50, 900, 30, 220)]
    v_list = [rng.standard_normal((len(k), 2)) for k in keys_list]
    port = _free_port()
    ctx = mp.get_context('spawn')
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, keys_list, q_list, v_list,
                                                     str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    r0, r1 = (pickle.load(open(tmp_path / ('b%d.pkl' % r), 'rb')) for r in range(2))
    assert sorted(r0) == list(range(5)) and sorted(r1) == list(range(5))
    for p in range(5):
        c = keys_list[p].mean(axis=0)
        W = oracle.OracleMesh(*HostMesh(keys_list[p] - c).export()).weights(q_list[p] - c)
        expect = oracle.spmm_like_scipy(W, v_list[p])
        assert np.array_equal(r0[p], expect) and np.array_equal(r1[p], expect)
