"""qGGMRF prior gradient/Hessian in FP64 numpy (TEST INFRASTRUCTURE ONLY).

Restates mbirtorch ``qggmrf.py`` (reference v0.0.2):
  * ``b_from_nbr_wts``  -- get_b_from_nbr_wts, qggmrf.py:22-32
  * ``two_b_tilde``     -- b_tilde_by_definition x 2, qggmrf.py:35-74
  * ``gradient_and_hessian`` -- qggmrf_gradient_and_hessian_at_indices,
    qggmrf.py:77-183 (single volume, reflected slice ends, clamped in-plane
    neighbours)
"""

import numpy as np

F32_EPS = float(np.finfo(np.float32).eps)


def b_from_nbr_wts(nbr_wts):
    """[row, col, slice] weights -> normalized 6-tuple ordered
    (row+1, row-1, col+1, col-1, slice+1, slice-1)."""
    b = np.array([nbr_wts, nbr_wts], dtype=np.float64).T.flatten()
    return tuple(b / np.sum(b))


def two_b_tilde(delta, sigma_x, p, q, T):
    """rho'(delta)/delta with |delta| floored at T*sigma_x*eps_f32."""
    a_min = T * sigma_x * F32_EPS
    abs_delta = np.maximum(np.abs(delta), a_min)
    delta_scale = abs_delta / (T * sigma_x)
    ds_q_minus_p = delta_scale ** (q - p)
    ds_p_minus_2 = abs_delta ** (p - 2)
    numerator = ds_p_minus_2 / (2 * sigma_x ** p)
    numerator = numerator * ds_q_minus_p * ((q / p) + ds_q_minus_p)
    return 2.0 * numerator / (1 + ds_q_minus_p) ** 2


def gradient_and_hessian(flat_recon, recon_shape, pixel_indices, b, sigma_x,
                         p, q, T):
    """Surrogate gradient and Hessian diagonal at the cylinders
    ``pixel_indices`` of ``flat_recon`` (N*N, S).  Returns two (P, S) arrays."""
    flat_recon = np.asarray(flat_recon, dtype=np.float64)
    idx = np.asarray(pixel_indices, dtype=np.int64)
    num_rows, num_cols = int(recon_shape[0]), int(recon_shape[1])
    cyl = flat_recon[idx]
    zero = np.zeros((cyl.shape[0], 1))
    delta = np.concatenate((zero, cyl[:, 1:] - cyl[:, :-1], zero), axis=1)
    bt2 = two_b_tilde(delta, sigma_x, p, q, T)
    bt2d = bt2 * delta
    grad = -b[4] * bt2d[:, 1:] + b[5] * bt2d[:, :-1]
    hess = b[4] * bt2[:, 1:] + b[5] * bt2[:, :-1]
    row, col = idx // num_cols, idx % num_cols
    for (dr, dc), bv in (((1, 0), b[0]), ((-1, 0), b[1]),
                         ((0, 1), b[2]), ((0, -1), b[3])):
        r = np.clip(row + dr, 0, num_rows - 1)
        c = np.clip(col + dc, 0, num_cols - 1)
        d = cyl - flat_recon[r * num_cols + c]
        w = bv * two_b_tilde(d, sigma_x, p, q, T)
        grad = grad + w * d
        hess = hess + w
    return grad, hess
