"""Host-side logic of mbirtorch_b200 against the reference's own values
(CPU only: model geometry, tap radii, auto-regularization, DC damping
profile, partitions and RNG order, parameter semantics)."""

import warnings

import numpy as np
import pytest

import mbirtorch_b200 as mb
from _cases import PROJECTOR_NAMES, build_model, load_projector_case
from conftest import load_golden


@pytest.mark.parametrize("name", PROJECTOR_NAMES)
def test_model_geometry_matches_reference(name):
    d = load_projector_case(name)
    m = build_model(d)
    assert tuple(m.get_params('recon_shape')) == tuple(int(v) for v in d['recon_shape'])
    assert m.get_psf_radius() == int(d['psf_radius'])
    g = m._geometry()
    assert g.num_views == int(d['sinogram_shape'][0])
    if 'bp_psf_radius' in d.files:
        assert m.get_psf_radii() == (int(d['psf_radius']), int(d['bp_psf_radius']))
        assert np.isclose(m.get_magnification(), float(d['magnification']))
        assert np.isclose(m.get_params('recon_slice_offset'), float(d['recon_slice_offset']))
        np.testing.assert_array_equal(m._view_params_array(), d['view_params'])
    else:
        np.testing.assert_array_equal(m._view_params_array(), d['view_params'])


def _parallel(shape):
    m = mb.ParallelBeamModel(shape, np.linspace(0, np.pi, shape[0], endpoint=False))
    m.set_params(no_warning=True, verbose=0)
    return m


def test_auto_regularization_parallel_matches_reference():
    d = load_golden('direct.npz')
    m = _parallel(d['par_sino'].shape)
    r = m.auto_set_regularization_params(d['par_sino'])
    np.testing.assert_allclose([r['sigma_y'], r['sigma_x'], r['sigma_prox']], d['par_reg'],
                               rtol=1e-6)
    r = m.auto_set_regularization_params(d['par_sino'], weights=d['par_w'])
    np.testing.assert_allclose([r['sigma_y'], r['sigma_x'], r['sigma_prox']], d['par_reg_w'],
                               rtol=1e-6)


@pytest.mark.parametrize("tag", ["cone", "curved", "helical"])
def test_cone_geometry_regularization_damping_match_reference(tag):
    d = load_golden('direct.npz')
    s = d[f'{tag}_sino']
    V = s.shape[0]
    if tag == 'helical':
        ang, zs = np.linspace(0, 4 * np.pi, V, endpoint=False), np.linspace(-2.0, 2.0, V)
    else:
        ang, zs = np.linspace(0, 2 * np.pi, V, endpoint=False), None
    m = mb.ConeBeamModel(s.shape, ang, 64.0, 32.0, helical_z_shifts=zs,
                         use_curved_detector=(tag == 'curved'))
    m.set_params(no_warning=True, verbose=0)
    assert tuple(m.get_params('recon_shape')) == tuple(int(v) for v in d[f'{tag}_recon_shape'])
    assert np.isclose(m.get_params('recon_slice_offset'), float(d[f'{tag}_rso']))
    assert m.get_psf_radii() == tuple(int(v) for v in d[f'{tag}_psf'])
    r = m.auto_set_regularization_params(s)
    np.testing.assert_allclose([r['sigma_y'], r['sigma_x'], r['sigma_prox']], d[f'{tag}_reg'],
                               rtol=1e-6)
    np.testing.assert_array_equal(m._dc_damping_profile(), d[f'{tag}_dc'])


@pytest.mark.parametrize("tag,seed", [("a", 3), ("b", 5)])
def test_partitions_and_rng_order_match_reference(tag, seed):
    d = load_golden('partitions.npz')
    np.random.seed(seed)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        parts = mb.gen_set_of_pixel_partitions(tuple(d[f'{tag}_shape']),
                                               list(d[f'{tag}_gran']))
    for i, p in enumerate(parts):
        np.testing.assert_array_equal(p.numpy(), d[f'{tag}_part{i}'])
    np.testing.assert_array_equal(np.random.randint(0, 2 ** 30, size=4), d[f'{tag}_after'])
    np.testing.assert_array_equal(
        mb.gen_partition_sequence([2, 4, 6] + [7, 8, 9, 10] * 25, 120), d['seq'])
    np.testing.assert_array_equal(mb.get_2d_ror_mask((18, 13)), d['mask_18x13'])


def test_set_params_semantics():
    m = _parallel((12, 4, 16))
    with pytest.raises(ValueError):
        m.set_params(not_a_param=1)
    with pytest.raises(NameError):
        m.get_params('not_a_param')
    assert m.get_params('auto_regularize_flag') is True
    with pytest.warns(UserWarning):
        m.set_params(sigma_y=2.0)
    assert m.get_params('auto_regularize_flag') is False
    m.set_params(no_warning=True, sharpness=0.5)
    assert m.get_params('auto_regularize_flag') is True
    assert m.get_params(['p', 'q', 'T']) == [2.0, 1.2, 1.0]
    assert m.get_params('granularity') == [1, 2, 4, 8, 16, 32, 64, 128, 128, 128, 128]


def test_parallel_verify_rejects_bad_params():
    m = _parallel((12, 4, 16))
    m.set_params(no_warning=True, voxel_slice_aspect=2.0)
    with pytest.raises(ValueError):
        m.verify_valid_params()


def test_cone_rejects_mismatched_z_shifts():
    with pytest.raises(ValueError):
        mb.ConeBeamModel((10, 4, 8), np.zeros(10), 10.0, 5.0, helical_z_shifts=np.zeros(9))


def test_compute_without_cuda_fails_loudly():
    """No CPU fallback: compute on a machine without CUDA raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    m = _parallel((12, 4, 16))
    with pytest.raises(RuntimeError, match="CUDA"):
        m.forward_project(np.zeros(m.get_params('recon_shape'), np.float32))


def test_storage_precision_names():
    m = _parallel((12, 4, 16))
    for s in ('float32', 'bfloat16', 'float16', 'bf16', 'fp16'):
        m.set_storage_precision(s)
    with pytest.raises(ValueError):
        m.set_storage_precision('int8')


def test_denoiser_noise_estimate_and_regularization_match_reference():
    """The denoiser's host statistics (noise estimate, auto-regularization
    on the row subsample) against the reference's values."""
    from conftest import load_golden
    from mbirtorch_b200.denoising import _subsample_to_host
    d = load_golden('denoise.npz')
    noisy = d['noisy']
    den = mb.QGGMRFDenoiser(noisy.shape)
    den.set_params(no_warning=True, verbose=0)
    assert abs(den.estimate_image_noise_std(noisy) - float(d['sigma_est'])) \
        <= 1e-6 * float(d['sigma_est'])
    for tag, sigma in (('given', 0.1), ('auto', None)):
        sigma = den.estimate_image_noise_std(noisy) if sigma is None else sigma
        den.set_params(no_warning=True, sigma_noise=sigma)
        rows = den.subsample_views(np.arange(noisy.shape[0]))
        step = int(rows[1] - rows[0]) if rows.size > 1 else 1
        reg = den.auto_set_regularization_params(_subsample_to_host(noisy, row_step=step))
        np.testing.assert_allclose([reg['sigma_y'], reg['sigma_x'], reg['sigma_prox']],
                                   d[f'{tag}_reg'], rtol=1e-6)
