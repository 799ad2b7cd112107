"""Multi-GPU use: one process per GPU, the mesh replicated, the queries sharded.

Queries are independent given the mesh, so nothing on the data path is
exchanged.  The collectives here are setup and bookkeeping only:

* :func:`broadcast_mesh` -- rank ``src`` runs natinterp3d's constructor once
  and broadcasts the packed arrays; every rank gets an ``Interpolator`` over
  the identical mesh (natinterp3d's constructor may perturb degenerate
  vertices with ``rand()``, so building on every rank could differ);
* :func:`shard_bounds` -- the contiguous query range of a rank;
* :func:`sharded_weights` -- each rank computes the CSR rows of its range and
  an all-gather of the per-rank non-zero counts turns its local row pointers
  into the global ones (the matrix is the row-wise concatenation);
* :func:`sharded_interpolate` -- each rank's block of ``W @ values``,
  optionally all-gathered into the full result;
* :func:`allreduce_grad` -- identity in the forward pass, sum over ranks of the
  gradient in the backward pass: wrapped around ``values`` before a
  differentiable interpolation of each rank's query shard, every rank ends
  with d loss / d values of the whole batch (d/dqueries stays per shard);
* :func:`shard_problems` / :func:`sharded_batch_interpolate` -- independent
  problems split over ranks by query count (no exchange on the data path).

Works with any ``torch.distributed`` backend (NCCL between GPUs, gloo on CPU).
"""
import numpy as np
import torch
import torch.distributed as dist

__all__ = ['broadcast_mesh', 'shard_bounds', 'sharded_weights', 'sharded_interpolate',
           'allreduce_grad', 'shard_problems', 'sharded_batch_interpolate']


def _tensor_device(group):
    backend = dist.get_backend(group)
    if backend == 'nccl':
        return torch.device('cuda', torch.cuda.current_device())
    return torch.device('cpu')


def shard_bounds(M, rank, world):
    """Contiguous [lo, hi) of M items for ``rank`` of ``world`` (sizes differ by at most 1)."""
    base, extra = divmod(int(M), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def broadcast_mesh(keys=None, group=None, src=0, device=None):
    """Build the mesh on rank ``src`` (from ``keys``) and give every rank an
    Interpolator over the same packed mesh."""
    from .natinterp3d import Interpolator
    rank = dist.get_rank(group)
    tdev = _tensor_device(group)
    if rank == src:
        it = Interpolator(keys, device=device)
        vx, tv, tn = it.mesh_arrays
        head = torch.tensor([vx.shape[0], tv.shape[0]] + list(it.centroid.view(np.int64)),
                            dtype=torch.int64, device=tdev)
    else:
        head = torch.zeros(5, dtype=torch.int64, device=tdev)
    dist.broadcast(head, src, group=group)
    nv, nt = int(head[0]), int(head[1])
    centroid = head[2:].cpu().numpy().view(np.float64).copy()
    if rank == src:
        bufs = [torch.from_numpy(a).to(tdev) for a in (vx, tv, tn)]
    else:
        bufs = [torch.empty((nv, 3), dtype=torch.float64, device=tdev),
                torch.empty((nt, 4), dtype=torch.int32, device=tdev),
                torch.empty((nt, 4), dtype=torch.int32, device=tdev)]
    for b in bufs:
        dist.broadcast(b, src, group=group)
    if rank == src:
        return it
    arrays = [b.cpu().numpy() for b in bufs]
    return Interpolator.from_mesh(centroid, *arrays, device=device)


def sharded_weights(queries, row_fn, group=None):
    """CSR block of this rank's query shard with global row pointers.

    ``row_fn(q_local) -> (rowptr, cols, vals)`` (numpy or tensors, local
    rowptr starting at 0) computes the rows; returns (global_row0,
    global_rowptr_block, cols, vals, total_nnz)."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard_bounds(len(queries), rank, world)
    rowptr, cols, vals = row_fn(queries[lo:hi])
    rowptr = np.asarray(rowptr.cpu() if isinstance(rowptr, torch.Tensor) else rowptr, np.int64)
    tdev = _tensor_device(group)
    mine = torch.tensor([int(rowptr[-1])], dtype=torch.int64, device=tdev)
    counts = [torch.zeros(1, dtype=torch.int64, device=tdev) for _ in range(world)]
    dist.all_gather(counts, mine, group=group)
    counts = [int(c.item()) for c in counts]
    offset = sum(counts[:rank])
    total = sum(counts)
    if total > np.iinfo(np.int32).max:
        raise OverflowError('Total number of nonzero weights exceeds int32 limit')
    return lo, (rowptr + offset).astype(np.int32), cols, vals, total


def sharded_interpolate(queries, interp_fn, group=None, gather=False):
    """This rank's block of the interpolation (``interp_fn(q_local) -> tensor``);
    with ``gather`` every rank receives the full [M, ...] result."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    M = len(queries)
    lo, hi = shard_bounds(M, rank, world)
    out = interp_fn(queries[lo:hi])
    if not gather:
        return lo, out
    tdev = _tensor_device(group)
    out_t = out if isinstance(out, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(out))
    out_t = out_t.to(tdev)
    width = tuple(out_t.shape[1:])
    # equal-sized blocks for the collective: pad to the largest shard, trim after
    rows = max(b - a for a, b in (shard_bounds(M, r, world) for r in range(world)))
    padded = torch.zeros((rows,) + width, dtype=out_t.dtype, device=tdev)
    padded[:out_t.shape[0]] = out_t
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    blocks = []
    for r in range(world):
        a, b = shard_bounds(M, r, world)
        blocks.append(parts[r][:b - a])
    return 0, torch.cat(blocks)


class _AllReduceGrad(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, group):
        ctx.group = group
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous().clone()
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=ctx.group)
        return g, None


def allreduce_grad(values, group=None):
    """``values`` unchanged; its gradient is summed over the ranks of ``group``
    (each rank differentiates its own query shard: d loss / d values is the
    sum of the shards' W_r^T g_r)."""
    return _AllReduceGrad.apply(values, group)


def shard_problems(costs, world):
    """Problem indices per rank, balanced by cost (e.g. query counts): the
    costliest problem goes to the least loaded rank, ties to the lower rank;
    each rank's list is in ascending problem order."""
    costs = np.asarray(costs, np.float64)
    load = np.zeros(int(world))
    parts = [[] for _ in range(int(world))]
    for p in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = int(np.argmin(load))
        parts[r].append(p)
        load[r] += costs[p]
    return [sorted(x) for x in parts]


def sharded_batch_interpolate(keys_list, queries_list, values_list, group=None, device=None,
                              batch_factory=None, gather=True):
    """Independent problems over the ranks of ``group``: each rank builds and
    evaluates its share (``batch_factory(keys) -> object with
    .interpolate(queries_list, values_list)``, by default a
    :class:`~natinterp3d_b200.batch.BatchInterpolator`).  Returns
    {problem index: result} for this rank's problems, or for all problems
    when ``gather`` (an object all-gather of the host results)."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    mine = shard_problems([len(q) for q in queries_list], world)[rank]
    out = {}
    if mine:
        if batch_factory is None:
            from .batch import BatchInterpolator

            def batch_factory(keys):
                return BatchInterpolator(keys, device=device)
        b = batch_factory([keys_list[p] for p in mine])
        res = b.interpolate([queries_list[p] for p in mine], [values_list[p] for p in mine])
        out = {p: np.asarray(r) for p, r in zip(mine, res)}
    if not gather:
        return out
    parts = [None] * world
    dist.all_gather_object(parts, out, group=group)
    full = {}
    for d in parts:
        full.update(d)
    return full
