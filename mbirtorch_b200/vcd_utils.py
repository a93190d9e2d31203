"""Host-side VCD helpers: ROR mask, pixel partitions, sequence, weights.

These run in numpy on the host exactly as in the reference (vcd_utils.py,
reference v0.0.2), because the seeded global ``np.random`` call order --
one permutation, then one choice per multi-subset partition -- fixes which
pixels each subset holds, and a reconstruction reproduces the reference's
trajectory only if that order is kept.
"""

import warnings

import numpy as np
import torch


def get_2d_ror_mask(recon_shape, *, use_ror_mask=True, crop_radius_pixels=0,
                    crop_radius_fraction=0.0):
    """Boolean (rows, cols) region-of-reconstruction mask (vcd_utils.py:18-79):
    the inscribed ellipse by default, all ones for ``use_ror_mask=False``, or
    a validated custom 0/1 array."""
    if use_ror_mask is False:
        if crop_radius_pixels != 0 and crop_radius_fraction != 0.0:
            raise ValueError('crop_radius_pixels and crop_radius_fraction must be zero '
                             'if use_ror_mask is set to False.')
        return np.ones(recon_shape[:2], dtype=bool)
    if use_ror_mask is True:
        if crop_radius_pixels != 0 and crop_radius_fraction != 0.0:
            raise ValueError('Only one of crop_radius_pixels and crop_radius_fraction '
                             'can be nonzero.')
        nr, nc = recon_shape[:2]
        rc, cc = (nr - 1) / 2, (nc - 1) / 2
        rr = rc - max(int(rc * crop_radius_fraction), crop_radius_pixels, 0)
        cr = cc - max(int(cc * crop_radius_fraction), crop_radius_pixels, 0)
        X, Y = np.meshgrid(np.arange(nc) - cc, np.arange(nr) - rc)
        return (X / cr) ** 2 + (Y / rr) ** 2 <= 1.0
    if crop_radius_pixels != 0 and crop_radius_fraction != 0.0:
        raise ValueError('crop_radius_pixels and crop_radius_fraction must be zero '
                         'if use_ror_mask is a custom array.')
    mask = np.asarray(use_ror_mask)
    if mask.shape != tuple(recon_shape[:2]):
        raise ValueError(f"Custom use_ror_mask must have shape recon_shape[:2]. "
                         f"Got mask.shape={mask.shape}, expected {tuple(recon_shape[:2])}.")
    if not np.all((mask == 0) | (mask == 1)):
        raise ValueError("Custom use_ror_mask must contain only 0s and 1s.")
    return mask


def get_support_radius(recon_shape, delta_voxel_row, delta_voxel_col, use_ror_mask=True):
    nr, nc = recon_shape[:2]
    hr, hc = 0.5 * nr * delta_voxel_row, 0.5 * nc * delta_voxel_col
    if use_ror_mask is True:
        return float(max(hr, hc))
    return float(np.hypot(hr, hc))


def gen_pixel_partition(recon_shape, num_subsets, use_ror_mask=True, rng=None):
    """(num_subsets, n) int32 pixel indices, sorted within each subset, equal
    sized (vcd_utils.py:97-156).  RNG use: one np.random.permutation of the
    ROR pixels, then one np.random.choice (without replacement) of the padding
    indices from the non-final subsets; a single subset draws nothing.
    ``rng`` (a numpy RandomState) replaces the global generator with the same
    call order; None uses numpy's global state, as the reference does."""
    rng = np.random if rng is None else rng
    nr, nc = recon_shape[:2]
    indices = np.arange(nr * nc, dtype=np.int32)
    if use_ror_mask is not False:
        indices = indices[get_2d_ror_mask(recon_shape, use_ror_mask=use_ror_mask).flatten() == 1]
    if num_subsets > len(indices):
        num_subsets = len(indices)
        warnings.warn('\nThe number of partition subsets is greater than the number of '
                      'pixels in the region of reconstruction.  \nReducing the number '
                      'of subsets to equal the number of indices.')
    if num_subsets == 1:
        return np.sort(indices).reshape(1, -1)
    per = int(np.ceil(len(indices) / num_subsets))
    n_extra = num_subsets * per - len(indices)
    indices = rng.permutation(indices)
    n_non_final = (num_subsets - 1) * per
    extra = rng.choice(indices[:n_non_final], size=n_extra, replace=False)
    indices = np.concatenate((indices, extra))
    return np.sort(indices.reshape(num_subsets, indices.size // num_subsets), axis=1)


def gen_set_of_pixel_partitions(recon_shape, granularity, device=None, use_ror_mask=True):
    """One partition per granularity entry, as int64 tensors on ``device``."""
    return [torch.as_tensor(np.ascontiguousarray(
        gen_pixel_partition(recon_shape, n, use_ror_mask=use_ror_mask)),
        dtype=torch.int64, device=device) for n in granularity]


def gen_partition_sequence(partition_sequence, max_iterations):
    seq = np.array(partition_sequence)
    if max_iterations > seq.size:
        return np.concatenate((seq, np.full(max_iterations - seq.size, seq[-1])))
    return seq[:max_iterations]


def gen_full_indices(recon_shape, use_ror_mask=True):
    return gen_pixel_partition(recon_shape, num_subsets=1, use_ror_mask=use_ror_mask)[0]


def gen_weights(sinogram, weight_type):
    """Noise-model weights (vcd_utils.py:205-260), computed where the input is."""
    xp = torch if isinstance(sinogram, torch.Tensor) else np
    if weight_type == 'unweighted':
        return xp.ones_like(sinogram)
    if weight_type == 'transmission':
        return xp.exp(-sinogram)
    if weight_type == 'transmission_root':
        return xp.exp(-sinogram / 2)
    if weight_type == 'emission':
        return 1.0 / (xp.abs(sinogram) + 0.1)
    raise Exception(f"gen_weights: undefined weight_type {weight_type}")


def estimate_background_cluster_boundaries(sinogram):
    """(left, right) value boundaries of the histogram peak nearest 0
    (vcd_utils.py:263-305)."""
    hist, edges = np.histogram(np.asarray(sinogram).ravel(), bins=400)
    centers = 0.5 * (edges[:-1] + edges[1:])
    peaks = []
    if len(hist) > 1 and hist[0] > hist[1]:
        peaks.append(0)
    for i in range(1, len(hist) - 1):
        if hist[i] >= hist[i - 1] and hist[i] > hist[i + 1]:
            peaks.append(i)
    if not peaks:
        peak = int(np.argmin(np.abs(centers)))
    else:
        peak = min(peaks, key=lambda i: abs(centers[i]))
    cutoff = 0.1 * hist[peak]
    lo = peak
    while lo > 0 and hist[lo] > cutoff:
        lo -= 1
    hi = peak
    while hi < len(hist) - 1 and hist[hi] > cutoff:
        hi += 1
    return centers[lo], centers[hi]
