"""Differentiable Sibson interpolation for PyTorch.

``interpolate(interpolator, queries, values)`` returns ``W(queries) @ values``
and back-propagates into both arguments:

* d/dvalues = W^T @ grad_out, a deterministic transpose product (CSC built by
  a stable sort on the GPU, no floating-point atomics);
* d/dqueries from the analytic derivative of the Sibson coordinates with
  respect to the query position (the GPU kernel differentiates the
  virtual-tet volumes, the only terms that move with the query).  The
  forward keeps every row's cavity record (788 bytes a row) so that the
  backward starts from it; beyond RECORDS_MAX_BYTES of records, or on meshes
  with other than the default fast predicates, the backward locates and
  floods each query's cavity again (same results, bit for bit).

The weights are computed in float64 on the device and cast to the query dtype;
the product and the output use the promoted dtype of (queries, values).  Rows
are summed in natinterp3d's stored column order, so for float64 queries the
output equals ``Interpolator.interpolate`` bit for bit; for float32 queries
natinterp3d's interpolate sums in sorted column order instead and the two can
differ in the last bits.
Sibson coordinates are continuous but not differentiable exactly at data
sites; such rows (and empty rows) get a zero query gradient.
"""
import torch

__all__ = ['interpolate', 'SibsonInterpolation']

# largest record buffer the forward keeps for the backward (bytes)
RECORDS_MAX_BYTES = 16 << 30


class _SibsonFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, queries, values, interp):
        dm = interp.device_mesh
        q = queries.detach().contiguous()
        v = values.detach()
        keep = (queries.requires_grad and dm.predicates == 'fast'
                and dm.records_bytes(q.shape[0]) <= RECORDS_MAX_BYTES)
        res = dm.weights_csr(q, interp.centroid, vals_dtype=torch.float64, return_totals=True,
                             keep_records=keep)
        rowptr, cols, w64, totals = res[:4]
        ctx.records = res[4] if keep else None
        # weights take the query dtype (as get_weights does); the product uses
        # the promoted dtype of (weights, values), summed in stored column order
        vals = w64.to(q.dtype)
        out = dm.spmm(rowptr, cols, vals, v)
        ctx.interp = interp
        ctx.value_shape = values.shape
        ctx.save_for_backward(q, v, rowptr, cols, vals, w64, totals)
        return out.reshape((q.shape[0],) + tuple(values.shape[1:]))

    @staticmethod
    def backward(ctx, grad_out):
        q, v, rowptr, cols, vals, w64, totals = ctx.saved_tensors
        dm = ctx.interp.device_mesh
        g = grad_out.contiguous()
        gq = gv = None
        if ctx.needs_input_grad[0]:
            gq = dm.query_grad(q, v, g, ctx.interp.centroid, rowptr, w64, totals,
                               records=ctx.records)
        ctx.records = None
        if ctx.needs_input_grad[1]:
            gv = dm.spmm_t(rowptr, cols, vals, g.reshape(q.shape[0], -1), dm.n_keys)
            gv = gv.reshape(ctx.value_shape).to(v.dtype)
        return gq, gv, None


def interpolate(interpolator, queries, values):
    """W(queries) @ values with gradients for queries [M, 3] and values [N] or [N, D]
    (CUDA tensors on the interpolator's device)."""
    return _SibsonFn.apply(queries, values, interpolator)


class SibsonInterpolation(torch.nn.Module):
    """Module wrapper: ``SibsonInterpolation(keys)(queries, values)``."""

    def __init__(self, keys, device=None):
        super().__init__()
        from .natinterp3d import Interpolator
        import numpy as np
        self.interpolator = Interpolator(np.asarray(keys, dtype=np.float64), device=device)

    def forward(self, queries, values):
        return interpolate(self.interpolator, queries, values)
