"""qGGMRF prior: parameter helpers and the host-side loss.

The prior's gradient and Hessian at subset cylinders run inside the fused
VCD kernels (csrc/vcd.cuh, ``vcd_direction_kernel``); this module holds the
host pieces of the reference's qggmrf.py (reference v0.0.2):

* :func:`get_b_from_nbr_wts` (qggmrf.py:22-32)
* :func:`qggmrf_loss` (qggmrf.py:209-252), a numpy debug path
"""

import numpy as np


def get_b_from_nbr_wts(qggmrf_nbr_wts):
    """[row, col, slice] weights -> 6 direction weights (row+1, row-1,
    col+1, col-1, slice+1, slice-1), normalized to sum to 1."""
    b = np.array([qggmrf_nbr_wts, qggmrf_nbr_wts]).T.flatten()
    b = b / np.sum(b)
    return tuple(b)


def qggmrf_loss(full_recon, qggmrf_params):
    """qGGMRF prior loss of a whole (rows, cols, slices) volume (numpy)."""
    b, sigma_x, p, q, T = qggmrf_params
    vol = np.asarray(full_recon)
    per_axis = [(b[j] + b[j + 1]) / (2 * sum(b)) for j in (0, 2, 4)]

    def rho(delta):
        a_min = T * sigma_x * np.finfo(np.float32).eps
        ad = np.clip(np.abs(delta), a_min, None)
        ds = ad / (T * sigma_x)
        dqp = ds ** (q - p)
        num = (ad ** p) / (p * sigma_x ** p) * dqp
        return num / (1 + dqp)

    loss = 0.0
    for axis in (0, 1, 2):
        loss += float(np.sum(per_axis[axis] * rho(np.diff(vol, axis=axis))))
    return loss
