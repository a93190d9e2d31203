"""FP64 VCD reconstruction oracle (TEST INFRASTRUCTURE ONLY).

Restates the reference's VCD engine on the CPU, calling the C projectors of
``oracle_proj.c``.  Followed (mbirtorch v0.0.2, file:line):

  * ROR mask / partitions ..... vcd_utils.py:18-79, 97-202 (same global
    np.random call order: permutation, then choice; one permutation of the
    subset order per iteration, tomography_model.py:2662-2697)
  * subset update ............. tomography_model.py:54-87, 2508-2657
  * cone DC damping ........... cone_beam.py:45-55, 424-496
  * direct recon filter ....... tomography_utils.py:18-78,
    parallel_beam.py:294-319, cone_beam.py:661-751
  * initial error state ....... tomography_model.py:1666-1712
  * iteration statistics ...... tomography_model.py:2325-2393, 2927-2987

The regularization scalars (sigma_y, sigma_x) are inputs: they come from the
host-side auto-regularization, which is checked separately against the
reference's own values.
"""

import numpy as np

from . import projectors as P
from .qggmrf import F32_EPS, b_from_nbr_wts, gradient_and_hessian


# ── partitions (host numpy, RNG order is load-bearing) ──────────────────────
def ror_mask(recon_shape):
    nr, nc = recon_shape[:2]
    rc, cc = (nr - 1) / 2, (nc - 1) / 2
    cols = np.arange(nc) - cc
    rows = np.arange(nr) - rc
    X, Y = np.meshgrid(cols, rows)
    return (X / cc) ** 2 + (Y / rc) ** 2 <= 1.0


def pixel_partition(recon_shape, num_subsets, use_ror_mask=True):
    nr, nc = recon_shape[:2]
    indices = np.arange(nr * nc, dtype=np.int32)
    if use_ror_mask:
        indices = indices[ror_mask(recon_shape).flatten() == 1]
    if num_subsets > len(indices):
        num_subsets = len(indices)
    if num_subsets == 1:
        return np.sort(indices).reshape(1, -1)
    per = int(np.ceil(len(indices) / num_subsets))
    extra = num_subsets * per - len(indices)
    indices = np.random.permutation(indices)
    non_final = (num_subsets - 1) * per
    extra_idx = np.random.choice(indices[:non_final], size=extra, replace=False)
    indices = np.concatenate((indices, extra_idx))
    return np.sort(indices.reshape(num_subsets, -1), axis=1)


def full_indices(recon_shape, use_ror_mask=True):
    return pixel_partition(recon_shape, 1, use_ror_mask)[0].astype(np.int64)


def partition_sequence(seq, max_iterations):
    seq = np.array(seq)
    if max_iterations > seq.size:
        return np.concatenate((seq, np.full(max_iterations - seq.size, seq[-1])))
    return seq[:max_iterations]


# ── geometry adapters ──────────────────────────────────────────────────────
class Problem:
    """One model's geometry for the oracle: kind 'parallel' or 'cone',
    an :class:`oracle.OracleGeometry`, and the per-view parameters (angles for
    parallel, (V, 2) [angle, z_shift] for cone)."""

    def __init__(self, kind, geom, view_params, recon_shape, source_iso_dist=None):
        self.kind = kind
        self.geom = geom
        self.view_params = np.asarray(view_params, dtype=np.float64)
        self.recon_shape = tuple(int(s) for s in recon_shape)
        self.source_iso_dist = source_iso_dist

    def forward(self, values, idx):
        if self.kind == 'parallel':
            return P.parallel_forward(self.geom, self.view_params, values, idx)
        return P.cone_forward(self.geom, self.view_params, values, idx)

    def back(self, sino, idx, coeff_power=1):
        if self.kind == 'parallel':
            return P.parallel_back(self.geom, self.view_params, sino, idx,
                                   coeff_power)
        return P.cone_back(self.geom, self.view_params, sino, idx, coeff_power)

    def z_shifts(self):
        if self.kind == 'parallel':
            return np.zeros(self.view_params.shape[0])
        return self.view_params[:, 1]


def dc_damping_profile(prob, cfg=(0.25, 100.0, 0.7, 0.5)):
    """Per-slice s_k of cone_beam.py:424-477 (FP64, cast to f32 like the
    reference)."""
    a, b, p, c = cfg
    g = prob.geom
    nz = prob.recon_shape[2]
    L = prob.recon_shape[0] * g.delta_voxel
    dz = g.delta_voxel_slice
    z = (np.arange(nz) - (nz - 1) / 2.0) * dz + g.recon_slice_offset
    R = prob.source_iso_dist
    zs = prob.z_shifts()

    def profile(t):
        return (c * t ** p + a * b ** p) / (t ** p + b ** p)

    if zs.max() - zs.min() == 0:
        s = profile(L * np.abs(z - zs[0]) / (R * dz))
    else:
        t = L * np.abs(z[:, None] - zs[None, :]) / (R * dz)
        s = profile(t).mean(axis=1)
    return s.astype(np.float32).astype(np.float64)


# ── direct recon (FBP / FDK) ────────────────────────────────────────────────
def ramp_filter(num_channels):
    n = np.arange(-num_channels + 1, num_channels)
    f = 0.5 * np.sinc(n) - 0.25 * np.sinc(n / 2) ** 2
    return f.astype(np.float32).astype(np.float64)


def row_filter(sino, filt):
    V, R, C = sino.shape
    rows = sino.reshape(-1, C)
    out = np.empty_like(rows)
    for i in range(rows.shape[0]):
        out[i] = np.convolve(rows[i], filt, mode='full')[C - 1:2 * C - 1]
    return out.reshape(V, R, C)


def direct_recon(prob, sino):
    g = prob.geom
    V, R, C = sino.shape
    sino = np.asarray(sino, dtype=np.float64)
    if prob.kind == 'parallel':
        scale = 1.0 / (g.delta_voxel * g.delta_voxel_row)
        filt = ramp_filter(C) * np.float32(scale * (np.pi / V))
        filtered = row_filter(sino, filt)
    else:
        m, n = np.meshgrid(np.arange(R), np.arange(C), indexing='ij')
        v = (m - (R - 1) / 2.0) * g.delta_det_row - g.det_row_offset
        u = (n - (C - 1) / 2.0) * g.delta_det_channel - g.det_channel_offset
        sdd = g.source_detector_dist
        wmap = (sdd / np.sqrt(sdd ** 2 + u ** 2 + v ** 2)).astype(np.float32)
        vol = g.delta_voxel * g.delta_voxel_row * g.delta_voxel_slice
        alpha = g.delta_det_row / (vol * g.magnification)
        filt = ramp_filter(C) * np.float32(alpha * (np.pi / V))
        filtered = row_filter(sino * wmap[None], filt)
    idx = full_indices(prob.recon_shape)
    cyl = prob.back(filtered, idx)
    nr, nc, ns = prob.recon_shape
    vol3 = np.zeros((nr * nc, ns))
    vol3[idx] = cyl
    vol3 = vol3.reshape(nr, nc, ns)
    zs = prob.z_shifts()
    if prob.kind == 'cone' and zs.max() - zs.min() > 0:
        k = np.arange(ns)
        z_k = g.delta_voxel_slice * (k - (ns - 1) / 2.0) + g.recon_slice_offset
        half = 0.5 * R * g.delta_det_row / g.magnification
        cov = np.sum(np.abs(z_k[:, None] - zs[None, :]) <= half, axis=1)
        zw = np.where(cov > 0, V / np.maximum(cov, 1), 0.0).astype(np.float32)
        vol3 = vol3 * zw[None, None, :]
    return vol3


# ── the VCD subset update and recon loop ────────────────────────────────────
class SubsetUpdater:
    """FP64 restatement of create_vcd_subset_updater's callable."""

    def __init__(self, prob, fm_hessian_flat, weights, sigma_y, sigma_x,
                 p=2.0, q=1.2, T=1.0, nbr_wts=(1.0, 1.0, 1.0), max_alpha=1.5,
                 positivity=False, dc_profile=None, prox_input=None, sigma_prox=None):
        """With ``prox_input`` ((N*N, S)) the prior is the proximal map's:
        gradient (x - v) / sigma_prox^2 and Hessian 1 / sigma_prox^2
        (qggmrf.py:186-206, tomography_model.py:2525-2537)."""
        self.prob = prob
        self.prox = None if prox_input is None else np.asarray(prox_input, np.float64)
        self.prox_c = None if prox_input is None else 1.0 / sigma_prox ** 2
        self.H = np.asarray(fm_hessian_flat, dtype=np.float64)
        self.w = None if weights is None else np.asarray(weights, np.float64)
        self.fm_c = 1.0 / sigma_y ** 2
        self.b = b_from_nbr_wts(list(nbr_wts))
        self.sigma_x, self.p, self.q, self.T = sigma_x, p, q, T
        self.max_alpha = max_alpha
        self.positivity = positivity
        self.dc = dc_profile

    def direction(self, g_f, g_p, h_f, h_p):
        if self.dc is None:
            return -((g_f + g_p) / (h_f + h_p))
        g = g_f + g_p
        h_inv = 1.0 / (h_f + h_p)
        gbar = np.sum(h_inv * g, axis=0) / np.sum(h_inv, axis=0)
        return -(g - ((1.0 - self.dc) * gbar)[None, :]) * h_inv

    def __call__(self, flat_recon, error, idx):
        prob, fm_c = self.prob, self.fm_c
        if self.prox is not None:
            g_p = self.prox_c * (flat_recon[idx] - self.prox[idx])
            h_p = self.prox_c
        else:
            g_p, h_p = gradient_and_hessian(flat_recon, prob.recon_shape, idx,
                                            self.b, self.sigma_x, self.p, self.q,
                                            self.T)
        ew = error if self.w is None else self.w * error
        g_f = -fm_c * prob.back(ew, idx)
        h_f = fm_c * self.H[idx]
        delta = self.direction(g_f, g_p, h_f, h_p)
        pl = np.sum(g_p * delta)
        pq = np.sum(h_p * delta * delta)
        Ad = prob.forward(delta, idx)
        if self.w is None:
            fl = fm_c * np.sum(error * Ad)
            fq = fm_c * np.sum(Ad * Ad)
        else:
            fl = fm_c * np.sum(self.w * error * Ad)
            fq = fm_c * np.sum(Ad * Ad * self.w)
        alpha = (fl - pl) / (fq + pq + F32_EPS)
        alpha = min(max(alpha, F32_EPS), self.max_alpha)
        if self.positivity:
            delta = np.maximum(-flat_recon[idx] / (alpha + F32_EPS), delta)
            Ad = prob.forward(delta, idx)
        ds = alpha * delta
        np.add.at(flat_recon, idx, ds)
        sumsq = np.sum(ds * ds, axis=0)
        error -= alpha * Ad
        ell1 = np.sum(np.abs(ds))
        return ell1, alpha, sumsq


def initial_state(prob, sino, init_recon, weights, scale_to_sinogram=True):
    idx = full_indices(prob.recon_shape)
    ns = prob.recon_shape[2]
    flat = np.asarray(init_recon, np.float64).reshape(-1, ns)
    fwd = prob.forward(flat[idx], idx)
    wf = fwd if weights is None else weights * fwd
    den = np.sum(wf * fwd)
    alpha = np.sum(wf * sino) / den if (den > 0 and scale_to_sinogram) else 1.0
    return sino - alpha * fwd, alpha * flat


def hessian_diagonal(prob, weights, sino_shape):
    idx = full_indices(prob.recon_shape)
    w = np.ones(sino_shape) if weights is None else weights
    cyl = prob.back(w, idx, coeff_power=2)
    nr, nc, ns = prob.recon_shape
    H = np.zeros((nr * nc, ns))
    H[idx] = cyl
    return H


def recon(prob, sino, sigma_y, sigma_x, partitions, seq, weights=None,
          init_recon=None, dc_profile=None, max_alpha=1.5, positivity=False,
          p=2.0, q=1.2, T=1.0, nbr_wts=(1.0, 1.0, 1.0), prox_input=None, sigma_prox=None):
    """FP64 VCD recon.  ``partitions`` must be drawn by the caller, and the
    global np.random state must be where the reference leaves it after the
    partitions: each iteration draws one subset permutation from it.

    Returns (recon (N, N, S), stats dict with fm_rmse, nmae, alpha)."""
    sino = np.asarray(sino, np.float64)
    weights = None if weights is None else np.asarray(weights, np.float64)
    scale = init_recon is None
    if init_recon is None:
        init_recon = direct_recon(prob, sino)
    error, flat = initial_state(prob, sino, init_recon, weights, scale)
    H = hessian_diagonal(prob, weights, sino.shape)
    prox_flat = None if prox_input is None else \
        np.asarray(prox_input, np.float64).reshape(-1, prob.recon_shape[2])
    upd = SubsetUpdater(prob, H, weights, sigma_y, sigma_x, p=p, q=q, T=T,
                        nbr_wts=nbr_wts, max_alpha=max_alpha,
                        positivity=positivity, dc_profile=dc_profile,
                        prox_input=prox_flat, sigma_prox=sigma_prox)
    N = sino.size
    avg_w = 1.0 if weights is None else float(np.mean(weights))
    stats = {'fm_rmse': [], 'nmae': [], 'alpha': []}
    for it in range(len(seq)):
        part = np.asarray(partitions[seq[it]])
        order = np.random.permutation(part.shape[0])
        ell1_tot, alpha_sum = 0.0, 0.0
        for k in order:
            ell1, alpha, _ = upd(flat, error, part[k].astype(np.int64))
            ell1_tot += ell1
            alpha_sum += alpha
        wsq = np.sum(error * error) if weights is None else np.sum(error * error * weights)
        stats['fm_rmse'].append(np.sqrt(wsq / (avg_w * N)) / sigma_y)
        l1 = np.sum(np.abs(flat))
        stats['nmae'].append(ell1_tot / l1 if l1 else float('nan'))
        stats['alpha'].append(alpha_sum / part.shape[0])
    nr, nc, ns = prob.recon_shape
    return flat.reshape(nr, nc, ns), stats
