"""QGGMRFDenoiser on the GPU: the reference's seeded denoise runs (given and
estimated sigma_noise) and the FP64 oracle, and a noise-reduction check
(test_denoiser.py of the reference)."""

import numpy as np
import pytest

import mbirtorch_b200 as mb
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["given", "auto"])
def test_denoise_matches_reference_and_oracle(tag):
    from oracle import denoise as oden
    from oracle import vcd as ovcd
    d = load_golden('denoise.npz')
    noisy = d['noisy']
    den = mb.QGGMRFDenoiser(noisy.shape)
    den.set_params(no_warning=True, verbose=0)
    np.random.seed(13)
    out, dd = den.denoise(noisy, sigma_noise=0.1 if tag == 'given' else None, max_iterations=4,
                          stop_threshold_change_pct=0.0, logfile_path=None, print_logs=False)
    rp = dd['recon_params']
    assert rel_l2(out, d[f'{tag}_out']) <= 1e-4
    np.testing.assert_allclose(rp['alpha_values'], d[f'{tag}_alpha'], rtol=1e-4)
    np.testing.assert_allclose(rp['stop_threshold_change_pct'], d[f'{tag}_nmae_pct'], rtol=1e-4)
    np.random.seed(13)
    part = ovcd.pixel_partition(noisy.shape, 16, use_ror_mask=False)
    reg = rp['regularization_params']
    oout, _, _ = oden.denoise(noisy, reg['sigma_y'], reg['sigma_x'], part, 4)
    assert rel_l2(out, oout) <= 1e-5


def test_denoise_reduces_noise_and_stops_at_threshold():
    shape = (32, 32, 32)
    clean = np.zeros(shape, dtype=np.float32)
    clean[8:-8, 8:-8, 8:-8] = 1.0
    noisy = clean + 0.1 * np.random.RandomState(2).randn(*shape).astype(np.float32)
    den = mb.QGGMRFDenoiser(shape)
    den.set_params(no_warning=True, verbose=0)
    np.random.seed(0)
    out, _ = den.denoise(noisy, sigma_noise=0.1, max_iterations=5, stop_threshold_change_pct=0.0,
                         logfile_path=None, print_logs=False)
    assert np.linalg.norm(out - clean) < 0.6 * np.linalg.norm(noisy - clean)
    np.random.seed(0)
    _, dd = den.denoise(noisy, sigma_noise=0.1, max_iterations=50, stop_threshold_change_pct=5.0,
                        logfile_path=None, print_logs=False)
    rp = dd['recon_params']
    assert rp['num_iterations'] < 50 and rp['stop_threshold_change_pct'][-1] < 5.0
