"""Differentiable projectors (the reference's autograd.py:17-119).

The forward and back projectors are an exact adjoint pair, so each is the
other's backward.  Differences from the reference, both additive:

* a leading batch axis is accepted: (B, rows, cols, slices) volumes
  project to (B, views, rows, channels) sinograms, one launch per volume;
* ``view_chunk``: with a memory cap the sinogram is produced and consumed in
  chunks of views -- the backward of :func:`forward_project_differentiable`
  back-projects the incoming gradient chunk by chunk and sums, and
  :func:`weighted_residual_loss` recomputes each chunk of A x in its own
  backward instead of keeping the whole sinogram alive.
"""

import torch

from ._lib import MBIR_LAYOUT_VRC


def _full_indices(model):
    return model.full_indices_device()


class _ForwardProjectFunction(torch.autograd.Function):
    """A: voxel cylinders at fixed indices -> sinogram; backward is A^T."""

    @staticmethod
    def forward(ctx, voxel_values, model, pixel_indices):
        ctx.model = model
        ctx.pixel_indices = pixel_indices
        return model.projector.forward(voxel_values, pixel_indices)

    @staticmethod
    def backward(ctx, grad_sinogram):
        grad = ctx.model.projector.back(grad_sinogram.contiguous(), ctx.pixel_indices)
        return grad, None, None


class _BackProjectFunction(torch.autograd.Function):
    """A^T: sinogram -> voxel cylinders at fixed indices; backward is A."""

    @staticmethod
    def forward(ctx, sinogram, model, pixel_indices):
        ctx.model = model
        ctx.pixel_indices = pixel_indices
        return model.projector.back(sinogram, pixel_indices)

    @staticmethod
    def backward(ctx, grad_values):
        return ctx.model.projector.forward(grad_values.contiguous(), ctx.pixel_indices), None, None


def _volumes(volume):
    return (volume.unsqueeze(0), True) if volume.dim() == 3 else (volume, False)


def forward_project_differentiable(model, volume):
    """Differentiable full-volume forward projection; (rows, cols, slices)
    or (B, rows, cols, slices) in, (V, R, C) or (B, V, R, C) out."""
    model._require_cuda()
    vols, single = _volumes(volume.to(device=model.torch_device, dtype=torch.float32))
    idx = _full_indices(model)
    outs = []
    for b in range(vols.shape[0]):
        vals = vols[b].reshape(-1, vols.shape[-1])[idx]
        outs.append(_ForwardProjectFunction.apply(vals, model, idx))
    return outs[0] if single else torch.stack(outs)


def back_project_differentiable(model, sinogram):
    """Differentiable full back projection; (V, R, C) or (B, V, R, C) in."""
    model._require_cuda()
    recon_shape = model.get_params('recon_shape')
    sinos = sinogram.to(device=model.torch_device, dtype=torch.float32)
    single = sinos.dim() == 3
    if single:
        sinos = sinos.unsqueeze(0)
    idx = _full_indices(model)
    outs = []
    for b in range(sinos.shape[0]):
        cyl = _BackProjectFunction.apply(sinos[b], model, idx)
        vol = torch.zeros(recon_shape[0] * recon_shape[1], cyl.shape[-1], dtype=cyl.dtype,
                          device=cyl.device).index_put((idx,), cyl)
        outs.append(vol.reshape(tuple(recon_shape[:2]) + (cyl.shape[-1],)))
    return outs[0] if single else torch.stack(outs)


class _ChunkedResidualLoss(torch.autograd.Function):
    """sum_v w (A_v x - y_v)^2 over view chunks, recomputing A_v x in the
    backward so no full sinogram of the forward pass is kept."""

    @staticmethod
    def forward(ctx, voxel_values, model, pixel_indices, y, weights, view_chunk):
        ctx.model, ctx.idx, ctx.view_chunk = model, pixel_indices, view_chunk
        ctx.save_for_backward(voxel_values, y, weights)
        total = torch.zeros((), dtype=torch.float64, device=voxel_values.device)
        V = y.shape[0]
        for v0 in range(0, V, view_chunk):
            vc = min(view_chunk, V - v0)
            r = model.projector.forward(voxel_values, pixel_indices, view_start=v0,
                                        view_count=vc) - y[v0:v0 + vc]
            total += (r * r * weights[v0:v0 + vc]).sum(dtype=torch.float64)
        return total

    @staticmethod
    def backward(ctx, grad_out):
        voxel_values, y, weights = ctx.saved_tensors
        model, idx, view_chunk = ctx.model, ctx.idx, ctx.view_chunk
        grad = torch.zeros_like(voxel_values)
        V = y.shape[0]
        for v0 in range(0, V, view_chunk):
            vc = min(view_chunk, V - v0)
            r = model.projector.forward(voxel_values, idx, view_start=v0, view_count=vc) \
                - y[v0:v0 + vc]
            g = (2.0 * grad_out) * weights[v0:v0 + vc] * r
            grad += model.projector.back(g.contiguous(), idx, view_start=v0,
                                         layout=MBIR_LAYOUT_VRC)
        return grad, None, None, None, None, None


def weighted_residual_loss(model, volume, y, weights=None, max_chunk_bytes=2 << 30):
    """sum w (A x - y)^2 for one volume (or a sum over a batch), with the
    sinogram formed in view chunks of at most ``max_chunk_bytes``.  The
    projections are FP32; the loss is accumulated and returned in FP64."""
    model._require_cuda()
    vols, _ = _volumes(volume.to(device=model.torch_device, dtype=torch.float32))
    ys = y.to(device=model.torch_device, dtype=torch.float32)
    if ys.dim() == 3:
        ys = ys.unsqueeze(0)
    V, R, C = ys.shape[1:]
    ws = torch.ones_like(ys) if weights is None else \
        weights.to(device=model.torch_device, dtype=torch.float32).expand_as(ys)
    chunk = max(1, min(V, int(max_chunk_bytes // max(1, 4 * R * C))))
    idx = _full_indices(model)
    loss = 0
    for b in range(vols.shape[0]):
        vals = vols[b].reshape(-1, vols.shape[-1])[idx]
        loss = loss + _ChunkedResidualLoss.apply(vals, model, idx, ys[b].contiguous(),
                                                 ws[b].contiguous(), chunk)
    return loss


class TorchProjector(torch.nn.Module):
    """The forward operator as an nn.Module; ``adjoint`` is the back projector."""

    def __init__(self, model):
        super().__init__()
        self.model = model

    def forward(self, volume):
        return forward_project_differentiable(self.model, volume)

    def adjoint(self, sinogram):
        return back_project_differentiable(self.model, sinogram)
