"""FP64 QGGMRF-denoiser oracle (TEST INFRASTRUCTURE ONLY).

Restates the reference's denoiser sweep (mbirtorch v0.0.2):

  * vcd_subset_denoiser ..... denoising.py:35-83 (identity forward model:
    forward gradient -fmc * e, forward Hessian 1; step clamped to
    [eps_f32, 1.5])
  * the sweep ............... denoising.py:390-425 (one fixed partition, its
    subsets in stored order every iteration; nmae = sum |alpha d| / ||x||_1)

The regularization scalars (sigma_y = sigma_noise, sigma_x) are inputs.
"""

import numpy as np

from .qggmrf import F32_EPS, b_from_nbr_wts, gradient_and_hessian


def denoise(noisy, sigma_y, sigma_x, partition, max_iterations, init_image=None,
            p=2.0, q=1.2, T=1.0, nbr_wts=(1.0, 1.0, 1.0)):
    """Returns (image (N, M, S), alpha per iteration, nmae per iteration)."""
    shape = noisy.shape
    S = shape[2]
    noisy = np.asarray(noisy, np.float64).reshape(-1, S)
    x = noisy.copy() if init_image is None else np.asarray(init_image, np.float64).reshape(-1, S)
    e = noisy - x
    fmc = 1.0 / sigma_y ** 2
    b = b_from_nbr_wts(list(nbr_wts))
    alphas, nmaes = [], []
    for _ in range(max_iterations):
        ell1, alpha_sum = 0.0, 0.0
        for idx in np.asarray(partition):
            idx = idx.astype(np.int64)
            g_p, h_p = gradient_and_hessian(x, shape, idx, b, sigma_x, p, q, T)
            e_sub = e[idx]
            d = -((-fmc * e_sub + g_p) / (1.0 + h_p))
            pl, pq = np.sum(g_p * d), np.sum(h_p * d ** 2)
            fl, fq = fmc * np.sum(e_sub * d), fmc * np.sum(d * d)
            alpha = min(max((fl - pl) / (fq + pq + F32_EPS), F32_EPS), 1.5)
            ds = alpha * d
            x[idx] += ds
            e[idx] = e_sub - ds
            ell1 += np.sum(np.abs(ds))
            alpha_sum += alpha
        alphas.append(alpha_sum / len(partition))
        nmaes.append(ell1 / np.sum(np.abs(x)))
    return x.reshape(shape), np.array(alphas), np.array(nmaes)
