"""Differentiable projectors (GPU): the autograd gradient equals the
adjoint (reference test_adjoint.py:37-57 bar, rel-max 1e-5), agrees with
central finite differences in FP64 directions, and the view-chunked
residual loss equals the unchunked one with the same gradient."""

import numpy as np
import pytest
import torch

import mbirtorch_b200 as mb

pytestmark = pytest.mark.gpu


def _par(shape=(24, 16, 16)):
    m = mb.ParallelBeamModel(shape, np.linspace(0, np.pi, shape[0], endpoint=False))
    m.set_params(no_warning=True, verbose=0)
    return m


def _cone(shape=(24, 16, 16)):
    m = mb.ConeBeamModel(shape, np.linspace(0, 2 * np.pi, shape[0], endpoint=False),
                         source_detector_dist=96.0, source_iso_dist=64.0)
    m.set_params(no_warning=True, verbose=0)
    return m


@pytest.mark.parametrize("make", [_par, _cone])
def test_gradient_equals_back_projection(make):
    torch.manual_seed(0)
    m = make()
    rs = m.get_params('recon_shape')
    vol = torch.rand(tuple(rs), device='cuda', requires_grad=True)
    y = torch.rand(tuple(m.get_params('sinogram_shape')), device='cuda')
    (mb.forward_project_differentiable(m, vol) * y).sum().backward()
    expected = m.back_project(y, output_sharded=True)
    rel = float((vol.grad - expected).abs().max() / expected.abs().max())
    assert rel < 1e-5


@pytest.mark.parametrize("make", [_par, _cone])
def test_back_projection_gradient_is_forward(make):
    torch.manual_seed(1)
    m = make()
    sino = torch.rand(tuple(m.get_params('sinogram_shape')), device='cuda', requires_grad=True)
    x = torch.rand(tuple(m.get_params('recon_shape')), device='cuda')
    (mb.back_project_differentiable(m, sino) * x).sum().backward()
    expected = m.forward_project(x, output_sharded=True)
    rel = float((sino.grad - expected).abs().max() / expected.abs().max())
    assert rel < 1e-5


@pytest.mark.parametrize("make", [_par, _cone])
def test_weighted_loss_gradient_vs_finite_differences(make):
    """Directional derivatives of sum w (Ax - y)^2 at eps = 1e-3 against
    the autograd gradient (the loss is quadratic, so central differences
    are exact up to rounding)."""
    g = torch.Generator(device='cuda').manual_seed(2)
    m = make()
    rs = tuple(m.get_params('recon_shape'))
    ss = tuple(m.get_params('sinogram_shape'))
    x = torch.rand(rs, device='cuda', generator=g)
    y = torch.rand(ss, device='cuda', generator=g)
    w = torch.rand(ss, device='cuda', generator=g) + 0.5
    xr = x.clone().requires_grad_(True)
    loss = mb.weighted_residual_loss(m, xr, y, w)
    loss.backward()
    mask = torch.as_tensor(mb.get_2d_ror_mask(rs), device='cuda')[..., None].float()
    for _ in range(8):
        d = torch.randn(rs, device='cuda', generator=g) * mask
        eps = 1e-3
        lp = float(mb.weighted_residual_loss(m, x + eps * d, y, w))
        lm = float(mb.weighted_residual_loss(m, x - eps * d, y, w))
        fd = (lp - lm) / (2 * eps)
        an = float((xr.grad.double() * d.double()).sum())
        assert abs(fd - an) <= 2e-3 * max(abs(an), 1e-6), (fd, an)


def test_chunked_loss_equals_unchunked_and_batches():
    torch.manual_seed(3)
    m = _par((40, 12, 16))
    rs = tuple(m.get_params('recon_shape'))
    ss = tuple(m.get_params('sinogram_shape'))
    xb = torch.rand((3,) + rs, device='cuda', requires_grad=True)
    y = torch.rand((3,) + ss, device='cuda')
    l_small = mb.weighted_residual_loss(m, xb, y, max_chunk_bytes=4 * ss[1] * ss[2] * 7)
    l_small.backward()
    g_small = xb.grad.clone()
    xb.grad = None
    sino = mb.forward_project_differentiable(m, xb)
    assert sino.shape == (3,) + ss
    l_full = ((sino - y) ** 2).sum()
    l_full.backward()
    assert abs(float(l_small.detach()) - float(l_full.detach())) / float(l_full.detach()) < 1e-5
    assert float((g_small - xb.grad).abs().max() / xb.grad.abs().max()) < 1e-5
    proj = mb.TorchProjector(m)
    assert proj(xb[0]).shape == ss and proj.adjoint(sino[0]).shape == rs
