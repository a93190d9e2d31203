"""Differentiable projectors (GPU): the autograd gradient equals the
adjoint (reference test_adjoint.py:37-57 bar, rel-max 1e-5) and the
reference's own autograd gradient (tests/golden/autograd.npz), agrees with
central finite differences on 64 random directions at the differentiable-
projector configuration (4 volumes of 128^3, parallel and cone), and the
view-chunked residual loss equals the unchunked one with the same gradient."""

import numpy as np
import pytest
import torch

import mbirtorch_b200 as mb
from conftest import load_golden

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


@pytest.mark.parametrize("tag", ["par", "cone"])
def test_gradient_matches_reference_autograd(tag):
    """The gradient of sum w (A x - y)^2 through forward_project_
    differentiable against the reference's own autograd gradient at the same
    inputs (autograd.py:17-119 run on the CPU)."""
    d = load_golden('autograd.npz')
    m = _par() if tag == 'par' else _cone()
    assert tuple(m.get_params('recon_shape')) == tuple(d[f'{tag}_recon_shape'])
    x = torch.as_tensor(d[f'{tag}_x'], device='cuda').requires_grad_(True)
    y = torch.as_tensor(d[f'{tag}_y'], device='cuda')
    w = torch.as_tensor(d[f'{tag}_w'], device='cuda')
    s = mb.forward_project_differentiable(m, x)
    loss = (w * (s - y) ** 2).sum()
    loss.backward()
    ref = d[f'{tag}_grad']
    got = x.grad.cpu().numpy()
    assert float(np.abs(got - ref).max() / np.abs(ref).max()) < 1e-5
    assert abs(float(loss) - float(d[f'{tag}_loss'])) / float(d[f'{tag}_loss']) < 1e-5


def _cfg4(kind):
    """The differentiable-projector configuration: parallel (256 views, 128 x
    192 detector) or cone (256 views, 128 x 192, magnification 1.5), 128^3."""
    if kind == 'parallel':
        m = mb.ParallelBeamModel((256, 128, 192), np.linspace(0, np.pi, 256, endpoint=False))
    else:
        m = mb.ConeBeamModel((256, 128, 192), np.linspace(0, 2 * np.pi, 256, endpoint=False),
                             source_detector_dist=1152.0, source_iso_dist=768.0)
        m.set_params(no_warning=True, delta_det_channel=1.5, delta_det_row=1.5)
        m.auto_set_recon_geometry(no_warning=True)
    m.set_params(no_warning=True, verbose=0, recon_shape=(128, 128, 128))
    return m


def _field(gen, n):
    """Gaussian-smoothed N(0, 1) fields of 128^3 (separable 9-tap kernel)."""
    x = torch.randn((n, 1, 128, 128, 128), generator=gen, device='cuda')
    k = torch.exp(-0.5 * (torch.arange(-4, 5, device='cuda', dtype=torch.float32) / 2.0) ** 2)
    k = k / k.sum()
    for dim in range(3):
        shape = [1, 1, 1, 1, 1]
        shape[2 + dim] = 9
        pad = [0, 0, 0, 0, 0, 0]
        pad[2 * (2 - dim)] = pad[2 * (2 - dim) + 1] = 4
        x = torch.nn.functional.conv3d(torch.nn.functional.pad(x, pad, mode="replicate"),
                                       k.view(shape))
    return x[:, 0].contiguous()


@pytest.mark.parametrize("kind", ["parallel", "cone"])
def test_batched_gradient_vs_finite_differences_64_directions(kind):
    """Configuration 4: a batch of 4 smoothed-noise volumes of 128^3, the
    loss sum w (A x - y)^2 with y from a second seeded batch, the sinogram in
    view chunks of at most 2 GB.  Central differences at eps = 1e-3 on 64
    seeded random directions, with the perturbed losses summed in FP64,
    against the autograd gradient's directional derivatives."""
    gen = torch.Generator(device='cuda').manual_seed(40)
    m = _cfg4(kind)
    x = _field(gen, 4)
    with torch.no_grad():
        y = mb.forward_project_differentiable(m, _field(gen, 4))
    w = 0.5 + torch.rand(y.shape, generator=gen, device='cuda')
    xr = x.clone().requires_grad_(True)
    mb.weighted_residual_loss(m, xr, y, w).backward()
    grad = xr.grad.double()
    eps = 1e-3
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            d = torch.randn(x.shape, generator=gen, device='cuda')
            lp = float(mb.weighted_residual_loss(m, x + eps * d, y, w))
            lm = float(mb.weighted_residual_loss(m, x - eps * d, y, w))
            fd = (lp - lm) / (2 * eps)
            an = float((grad * d.double()).sum())
            worst = max(worst, abs(fd - an) / max(abs(an), 1e-12))
    assert worst <= 1e-3, worst
