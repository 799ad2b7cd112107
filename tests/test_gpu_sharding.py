"""The sharding helpers over NCCL with the CUDA interpolator, world size 1
(the GPU tests run on one GPU; the two-rank host logic is tested with gloo on
CPU in test_sharding_gloo.py)."""
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

import natinterp3d_b200 as ni
from natinterp3d_b200 import autograd as nag
from natinterp3d_b200.sharding import (allreduce_grad, broadcast_mesh, sharded_batch_interpolate,
                                       sharded_interpolate, sharded_weights)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def nccl_group(cuda_device):
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    torch.cuda.set_device(cuda_device)
    dist.init_process_group('nccl', init_method='tcp://127.0.0.1:%d' % port, rank=0, world_size=1,
                            device_id=cuda_device)
    yield
    dist.destroy_process_group()


def test_nccl_sharded_paths_match_single_process(nccl_group, cuda_device):
    rng = np.random.default_rng(12)
    keys = rng.uniform(0, 1, (3000, 3))
    q = rng.uniform(0.05, 0.95, (5000, 3))
    v = rng.standard_normal((3000, 2))
    it = broadcast_mesh(keys, device=cuda_device)
    ref = ni.Interpolator(keys, device=cuda_device)
    W = ref.get_weights(q)

    def rows(qs):
        rp, cols, vals = it.get_weights_device(torch.from_numpy(qs).to(cuda_device))
        return rp, cols.cpu().numpy(), vals.cpu().numpy()

    lo, rowptr, cols, vals, total = sharded_weights(q, rows)
    assert lo == 0 and total == W.nnz
    assert np.array_equal(rowptr, W.indptr) and np.array_equal(cols, W.indices)
    assert np.array_equal(vals, W.data)
    _, full = sharded_interpolate(q, lambda qs: it.interpolate_device(
        torch.from_numpy(qs).to(cuda_device), torch.from_numpy(v).to(cuda_device)), gather=True)
    assert np.array_equal(full.cpu().numpy(), ref.interpolate(q, v))


def test_nccl_allreduce_grad_and_problem_sharding(nccl_group, cuda_device):
    rng = np.random.default_rng(13)
    keys = rng.uniform(0, 1, (2000, 3))
    it = ni.Interpolator(keys, device=cuda_device)
    q = torch.from_numpy(rng.uniform(0.1, 0.9, (4000, 3))).to(cuda_device)
    v0 = torch.from_numpy(rng.standard_normal((2000, 3))).to(cuda_device)
    g = torch.from_numpy(rng.standard_normal((4000, 3))).to(cuda_device)
    grads = []
    for wrap in (False, True):
        v = v0.clone().requires_grad_(True)
        out = nag.interpolate(it, q, allreduce_grad(v) if wrap else v)
        (out * g).sum().backward()
        grads.append(v.grad)
    assert torch.equal(grads[0], grads[1])   # one rank: the sum over ranks is its own gradient

    keys_list = [rng.uniform(0, 1, (n, 3)) for n in (500, 1500, 800)]
    q_list = [rng.uniform(0.1, 0.9, (m, 3)) for m in (300, 2000, 700)]
    v_list = [rng.standard_normal((len(k), 2)) for k in keys_list]
    res = sharded_batch_interpolate(keys_list, q_list, v_list, device=cuda_device)
    for p in range(3):
        expect = ni.Interpolator(keys_list[p], device=cuda_device).interpolate(q_list[p], v_list[p])
        assert np.array_equal(res[p], expect)
