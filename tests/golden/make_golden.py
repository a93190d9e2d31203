"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run where the reference package (mbirtorch 0.0.2) source tree is at hand,
naming its directory in MBIRTORCH_REFERENCE:

    MBIRTORCH_REFERENCE=<path to the mbirtorch checkout> \
        python tests/golden/make_golden.py

The script calls the reference's OWN torch bodies and public methods on
small seeded inputs (CPU, compile_mode='off') and stores inputs and outputs
in compressed .npz files next to this script.  The fixtures are the anchor
for the FP64 oracle (tests/test_oracle_golden.py) and, through it, for the
sm_100a kernels.  Nothing at run time reads the reference: only these files.

Cases
  projectors_*.npz  parallel (square, row aspect 3, channel offset 0.7) and
                    cone (flat, curved, helical, offsets) forward and back
                    bodies, coeff_power 1 and 2, full and subset pixel sets
  qggmrf.npz        qggmrf_gradient_and_hessian_at_indices on random volumes
  partitions.npz    gen_set_of_pixel_partitions / sequence under a seed
  autoreg.npz       auto_set_regularization_params on phantom sinograms
  direct.npz        recon_direct (FBP, FDK, helical FDK)
  recon_*.npz       seeded VCD recon traces (parallel, cone, weighted)
  prox_*.npz        seeded prox_map (proximal-map prior) traces, parallel
                    (automatic sigma_prox) and cone (given sigma_prox)
  denoise.npz       QGGMRFDenoiser: noise estimate and seeded denoise runs
                    (given and estimated sigma_noise)
  autograd.npz      the reference's autograd gradient of a weighted residual
                    loss through forward_project_differentiable (parallel,
                    cone)
  recon_simple_parallel_128.npz
                    the one-call parallel recon at the reference's CPU
                    configuration: a 128 x 128 x 16 ellipsoid phantom, 180
                    views on [0, pi), 16 x 192 detector, Gaussian noise at 1%
                    of the largest projection, 10 VCD iterations

Pass case-function names to regenerate only those, e.g.
    MBIRTORCH_REFERENCE=... python tests/golden/make_golden.py prox_cases
"""

import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("MBIRTORCH_REFERENCE")
if not REF:
    sys.exit("set MBIRTORCH_REFERENCE to the directory of the mbirtorch 0.0.2 checkout")
if REF not in sys.path:
    sys.path.insert(0, REF)

import mbirtorch  # noqa: E402
from mbirtorch import cone_beam, parallel_beam, qggmrf, vcd_utils  # noqa: E402
from mbirtorch.utilities import add_ellipsoid  # noqa: E402

torch.set_num_threads(min(8, os.cpu_count() or 1))


def _quiet(model):
    model.set_params(no_warning=True, verbose=0)
    return model


def phantom(recon_shape, seed, n_ellipsoids=10):
    """Sum of seeded ellipsoids on [-1, 1] grids (utilities.add_ellipsoid)."""
    rng = np.random.default_rng(seed)
    nr, nc, ns = recon_shape
    x = np.linspace(-1, 1, nc)
    y = np.linspace(-1, 1, nr)
    z = np.linspace(-1, 1, ns)
    X, Y = np.meshgrid(x, y)
    vol = np.zeros(recon_shape, np.float32)
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.5, 0.5, 3)
        a = rng.uniform(0.05, 0.4, 3)
        vol = add_ellipsoid(vol, (X, Y), z, c[0], c[1], c[2], a[0], a[1], a[2],
                            angle=rng.uniform(0, 180),
                            intensity=rng.uniform(0.1, 1.0))
    return vol.astype(np.float32)


def _geom_dict(model):
    """The model's geometry scalars in the reference's parameter names."""
    names = ['delta_det_channel', 'delta_det_row', 'det_channel_offset',
             'det_row_offset', 'delta_voxel', 'voxel_row_aspect',
             'voxel_slice_aspect']
    vals = model.get_params(names)
    d = dict(zip(names, [float(v) for v in vals]))
    d['sinogram_shape'] = np.array(model.get_params('sinogram_shape'))
    d['recon_shape'] = np.array(model.get_params('recon_shape'))
    return d


def projector_case(name, model, geometry, seed, ctor):
    """Run the reference torch bodies on random values/sinograms.  ``ctor``
    records how the model was built (constructor arguments and set_params),
    so a test can build the same model in another implementation."""
    rng = np.random.default_rng(seed)
    args = model._view_batch_args()
    rs = model.get_params('recon_shape')
    ss = model.get_params('sinogram_shape')
    vp_name = model.get_params('view_params_name')
    view_params = torch.as_tensor(np.asarray(model.get_params(vp_name)),
                                  dtype=torch.float32)
    full = vcd_utils.gen_full_indices(rs).astype(np.int64)
    subset = np.sort(rng.choice(full, size=max(1, full.size // 7), replace=False))
    if geometry == 'parallel':
        fwd, back = (parallel_beam._parallel_forward_view_batch,
                     parallel_beam._parallel_back_view_batch)
    else:
        fwd, back = cone_beam._cone_forward_view_batch, cone_beam._cone_back_view_batch
    out = dict(view_params=view_params.numpy(), **_geom_dict(model),
               psf_radius=np.array(args['psf_radius']),
               ctor=np.array(json.dumps(ctor)))
    if geometry == 'cone':
        out['bp_psf_radius'] = np.array(args['bp_psf_radius'])
        out['source_detector_dist'] = np.array(args['source_detector_dist'])
        out['magnification'] = np.array(args['magnification'])
        out['recon_slice_offset'] = np.array(args['recon_slice_offset'])
        out['use_curved_detector'] = np.array(int(args['use_curved_detector']))
    for tag, idx in (('full', full), ('subset', subset)):
        values = rng.standard_normal((idx.size, rs[2])).astype(np.float32)
        sino = rng.standard_normal(tuple(ss)).astype(np.float32)
        idx_t = torch.as_tensor(idx)
        with torch.no_grad():
            f = fwd(torch.as_tensor(values), idx_t, view_params, **args)
            b1 = back(torch.as_tensor(sino), idx_t, view_params, coeff_power=1, **args)
            b2 = back(torch.as_tensor(sino), idx_t, view_params, coeff_power=2, **args)
        out[f'{tag}_indices'] = idx
        out[f'{tag}_values'] = values
        out[f'{tag}_sino'] = sino
        out[f'{tag}_fwd'] = f.contiguous().numpy()
        out[f'{tag}_back1'] = b1.numpy()
        out[f'{tag}_back2'] = b2.numpy()
    np.savez_compressed(os.path.join(HERE, f'projectors_{name}.npz'), **out)
    print('wrote projectors', name, out['full_fwd'].shape)


PROJECTOR_CASES = [
    # name, geometry, seed, constructor arguments, set_params
    ('par_square', 'parallel', 1,
     dict(sinogram_shape=(30, 6, 24), angles=('linspace', 0.0, np.pi, 30)), {}),
    ('par_aspect3', 'parallel', 2,
     dict(sinogram_shape=(20, 5, 28), angles=('linspace', 0.0, np.pi, 20)),
     dict(voxel_row_aspect=3.0)),
    ('par_offset', 'parallel', 3,
     dict(sinogram_shape=(25, 4, 22), angles=('linspace', 0.1, np.pi + 0.1, 25)),
     dict(det_channel_offset=0.7, delta_det_channel=0.8)),
    ('cone_flat', 'cone', 4,
     dict(sinogram_shape=(24, 16, 16), angles=('linspace', 0.0, 2 * np.pi, 24),
          source_detector_dist=64.0, source_iso_dist=32.0), {}),
    ('cone_curved', 'cone', 5,
     dict(sinogram_shape=(24, 16, 16), angles=('linspace', 0.0, 2 * np.pi, 24),
          source_detector_dist=64.0, source_iso_dist=32.0, use_curved_detector=True), {}),
    ('cone_helical', 'cone', 6,
     dict(sinogram_shape=(40, 12, 18), angles=('linspace', 0.0, 4 * np.pi, 40),
          source_detector_dist=70.0, source_iso_dist=35.0,
          helical_z_shifts=('linspace_closed', -3.0, 3.0, 40)), {}),
    ('cone_offsets', 'cone', 7,
     dict(sinogram_shape=(20, 14, 20), angles=('linspace', 0.0, 2 * np.pi, 20),
          source_detector_dist=90.0, source_iso_dist=45.0),
     dict(det_row_offset=0.6, det_channel_offset=-0.4, delta_det_row=1.3,
          delta_det_channel=1.1, voxel_slice_aspect=1.5)),
]


def expand(spec):
    """('linspace', a, b, n) -> endpoint-free linspace; 'linspace_closed'
    includes the end point; anything else passes through."""
    if isinstance(spec, tuple) and spec and spec[0] == 'linspace':
        return np.linspace(spec[1], spec[2], spec[3], endpoint=False)
    if isinstance(spec, tuple) and spec and spec[0] == 'linspace_closed':
        return np.linspace(spec[1], spec[2], spec[3])
    return spec


def build_reference_model(geometry, ctor, setp):
    kw = {k: expand(v) for k, v in ctor.items()}
    shape = kw.pop('sinogram_shape')
    angles = kw.pop('angles')
    if geometry == 'parallel':
        m = mbirtorch.ParallelBeamModel(shape, angles, compile_mode='off', **kw)
    else:
        m = mbirtorch.ConeBeamModel(shape, angles, compile_mode='off', **kw)
    _quiet(m)
    if setp:
        m.set_params(no_warning=True, **setp)
    return m


def projector_cases():
    for name, geometry, seed, ctor, setp in PROJECTOR_CASES:
        model = build_reference_model(geometry, ctor, setp)
        projector_case(name, model, geometry, seed,
                       dict(geometry=geometry, ctor=ctor, set_params=setp))


def qggmrf_case():
    rng = np.random.default_rng(11)
    rs = (12, 10, 7)
    flat = rng.standard_normal((rs[0] * rs[1], rs[2])).astype(np.float32)
    flat[5] = flat[5, 0]   # a constant cylinder: zero slice deltas
    idx = np.sort(rng.choice(rs[0] * rs[1], size=40, replace=False)).astype(np.int64)
    out = dict(flat=flat, recon_shape=np.array(rs), indices=idx)
    for tag, (nbr, sx, p, q, T) in {
            'default': ([1.0, 1.0, 1.0], 0.7, 2.0, 1.2, 1.0),
            'aniso': ([1.0, 2.0, 0.5], 0.3, 2.0, 1.1, 2.0),
            'p15': ([1.0, 1.0, 1.0], 1.3, 1.5, 1.2, 1.0)}.items():
        b = qggmrf.get_b_from_nbr_wts(nbr)
        g, h = qggmrf.qggmrf_gradient_and_hessian_at_indices(
            torch.as_tensor(flat), rs, torch.as_tensor(idx), (b, sx, p, q, T))
        out[f'{tag}_params'] = np.array(nbr + [sx, p, q, T])
        out[f'{tag}_grad'] = g.numpy()
        out[f'{tag}_hess'] = h.numpy()
    np.savez_compressed(os.path.join(HERE, 'qggmrf.npz'), **out)
    print('wrote qggmrf')


def partition_case():
    out = {}
    for tag, rs, gran, seed in (('a', (20, 20, 3), [1, 2, 4, 8, 16], 3),
                                ('b', (17, 23, 2), [1, 3, 7, 64], 5)):
        np.random.seed(seed)
        parts = vcd_utils.gen_set_of_pixel_partitions(rs, gran)
        after = np.random.randint(0, 2 ** 30, size=4)   # RNG position afterwards
        for i, p in enumerate(parts):
            out[f'{tag}_part{i}'] = p.numpy()
        out[f'{tag}_after'] = after
        out[f'{tag}_shape'] = np.array(rs)
        out[f'{tag}_gran'] = np.array(gran)
    out['seq'] = vcd_utils.gen_partition_sequence([2, 4, 6] + [7, 8, 9, 10] * 25, 120)
    out['seq_short'] = vcd_utils.gen_partition_sequence([0, 1, 2], 2)
    out['mask_18x13'] = vcd_utils.get_2d_ror_mask((18, 13))
    np.savez_compressed(os.path.join(HERE, 'partitions.npz'), **out)
    print('wrote partitions')


def _parallel_data(seed, sino_shape=(30, 6, 24)):
    ang = np.linspace(0, np.pi, sino_shape[0], endpoint=False)
    m = _quiet(mbirtorch.ParallelBeamModel(sino_shape, ang, compile_mode='off'))
    rs = m.get_params('recon_shape')
    ph = phantom(rs, seed)
    sino = m.forward_project(ph)
    rng = np.random.default_rng(seed + 100)
    sino = (sino + rng.normal(0, 0.01 * sino.max(), sino.shape)).astype(np.float32)
    return m, ang, ph, sino


def _cone_data(seed, sino_shape=(24, 16, 16), helical=False, curved=False):
    V = sino_shape[0]
    if helical:
        ang = np.linspace(0, 4 * np.pi, V, endpoint=False)
        zsh = np.linspace(-2.0, 2.0, V)
    else:
        ang = np.linspace(0, 2 * np.pi, V, endpoint=False)
        zsh = None
    m = _quiet(mbirtorch.ConeBeamModel(sino_shape, ang, source_detector_dist=64.0,
                                       source_iso_dist=32.0, helical_z_shifts=zsh,
                                       use_curved_detector=curved, compile_mode='off'))
    rs = m.get_params('recon_shape')
    ph = phantom(rs, seed)
    sino = m.forward_project(ph)
    # Poisson counts at I0 = 1e4, converted back to line integrals.
    rng = np.random.default_rng(seed + 200)
    counts = rng.poisson(1e4 * np.exp(-0.05 * sino))
    sino = (-np.log(np.maximum(counts, 1) / 1e4) / 0.05).astype(np.float32)
    return m, ang, zsh, ph, sino


def autoreg_and_direct_cases():
    out = {}
    m, ang, ph, sino = _parallel_data(21)
    reg = m.auto_set_regularization_params(sino)
    out['par_sino'] = sino
    out['par_reg'] = np.array([reg['sigma_y'], reg['sigma_x'], reg['sigma_prox']])
    out['par_fbp'] = m.recon_direct(sino)
    w = vcd_utils.gen_weights(sino / max(1.0, sino.max()), 'transmission').astype(np.float32)
    reg = m.auto_set_regularization_params(sino, weights=w)
    out['par_w'] = w
    out['par_reg_w'] = np.array([reg['sigma_y'], reg['sigma_x'], reg['sigma_prox']])
    for tag, kw in (('cone', {}), ('curved', {'curved': True}), ('helical', {'helical': True})):
        mc, ang, zsh, ph, s = _cone_data(22, **kw)
        reg = mc.auto_set_regularization_params(s)
        out[f'{tag}_sino'] = s
        out[f'{tag}_reg'] = np.array([reg['sigma_y'], reg['sigma_x'], reg['sigma_prox']])
        out[f'{tag}_fdk'] = mc.recon_direct(s)
        out[f'{tag}_recon_shape'] = np.array(mc.get_params('recon_shape'))
        out[f'{tag}_rso'] = np.array(mc.get_params('recon_slice_offset'))
        out[f'{tag}_psf'] = np.array(mc.get_psf_radii())
        out[f'{tag}_dc'] = mc._dc_damping_slice_profile()[0][0].numpy()
    np.savez_compressed(os.path.join(HERE, 'direct.npz'), **out)
    print('wrote direct/autoreg')


def recon_cases():
    # Parallel, unweighted, default init (FBP scaled), 4 iterations.
    m, ang, ph, sino = _parallel_data(31)
    np.random.seed(7)
    rec, d = m.recon(sino, max_iterations=4, stop_threshold_change_pct=0,
                     logfile_path=None, print_logs=False)
    rp = d['recon_params']
    np.savez_compressed(os.path.join(HERE, 'recon_parallel.npz'), sino=sino, angles=ang,
                        recon=rec, fm_rmse=np.array(rp['fm_rmse']),
                        alpha=np.array(rp['alpha_values']),
                        stop=np.array(rp['stop_threshold_change_pct']),
                        reg=np.array([rp['regularization_params'][k]
                                      for k in ('sigma_y', 'sigma_x', 'sigma_prox')]),
                        seed=np.array(7), max_iterations=np.array(4))
    # Parallel, weighted, with positivity.
    w = vcd_utils.gen_weights(sino / max(1.0, sino.max()), 'transmission').astype(np.float32)
    m2, _, _, _ = _parallel_data(31)
    m2.set_params(no_warning=True, positivity_flag=True)
    np.random.seed(8)
    rec2, d2 = m2.recon(sino, weights=w, max_iterations=3, stop_threshold_change_pct=0,
                        logfile_path=None, print_logs=False)
    rp2 = d2['recon_params']
    np.savez_compressed(os.path.join(HERE, 'recon_parallel_weighted.npz'), sino=sino,
                        angles=ang, weights=w, recon=rec2,
                        fm_rmse=np.array(rp2['fm_rmse']),
                        alpha=np.array(rp2['alpha_values']),
                        reg=np.array([rp2['regularization_params'][k]
                                      for k in ('sigma_y', 'sigma_x', 'sigma_prox')]),
                        seed=np.array(8), max_iterations=np.array(3))
    # Cone (flat and helical), DC damping on (the default), 3 iterations.
    for tag, kw in (('cone', {}), ('cone_helical', {'helical': True})):
        mc, ang, zsh, ph, s = _cone_data(32, **kw)
        np.random.seed(9)
        rec3, d3 = mc.recon(s, max_iterations=3, stop_threshold_change_pct=0,
                            logfile_path=None, print_logs=False)
        rp3 = d3['recon_params']
        np.savez_compressed(os.path.join(HERE, f'recon_{tag}.npz'), sino=s, angles=ang,
                            z_shifts=np.zeros_like(ang) if zsh is None else zsh,
                            recon=rec3, fm_rmse=np.array(rp3['fm_rmse']),
                            alpha=np.array(rp3['alpha_values']),
                            reg=np.array([rp3['regularization_params'][k]
                                          for k in ('sigma_y', 'sigma_x', 'sigma_prox')]),
                            seed=np.array(9), max_iterations=np.array(3))
    print('wrote recons')


def prox_cases():
    # prox_map on a smoothed, perturbed phantom as the proximal input.
    m, ang, ph, sino = _parallel_data(41)
    rng = np.random.default_rng(43)
    v = (ph + rng.normal(0, 0.05, ph.shape)).astype(np.float32)
    np.random.seed(11)
    rec, d = m.prox_map(v, sino, max_iterations=3, stop_threshold_change_pct=0,
                        logfile_path=None, print_logs=False)
    rp = d['recon_params']
    np.savez_compressed(os.path.join(HERE, 'prox_parallel.npz'), sino=sino, angles=ang,
                        prox_input=v, recon=rec, fm_rmse=np.array(rp['fm_rmse']),
                        alpha=np.array(rp['alpha_values']),
                        reg=np.array([rp['regularization_params'][k]
                                      for k in ('sigma_y', 'sigma_x', 'sigma_prox')]),
                        sigma_prox=np.array(np.nan), seed=np.array(11), max_iterations=np.array(3))
    mc, ang, zsh, ph, s = _cone_data(42)
    v = (ph + rng.normal(0, 0.05, ph.shape)).astype(np.float32)
    np.random.seed(12)
    rec, d = mc.prox_map(v, s, sigma_prox=0.05, max_iterations=3, stop_threshold_change_pct=0,
                         logfile_path=None, print_logs=False)
    rp = d['recon_params']
    np.savez_compressed(os.path.join(HERE, 'prox_cone.npz'), sino=s, angles=ang,
                        z_shifts=np.zeros_like(ang), prox_input=v, recon=rec,
                        fm_rmse=np.array(rp['fm_rmse']), alpha=np.array(rp['alpha_values']),
                        reg=np.array([rp['regularization_params'][k]
                                      for k in ('sigma_y', 'sigma_x', 'sigma_prox')]),
                        sigma_prox=np.array(0.05), seed=np.array(12), max_iterations=np.array(3))
    print('wrote prox')


def denoise_case():
    shape = (24, 20, 10)
    clean = phantom(shape, 51)
    noisy = (clean + np.random.default_rng(52).normal(0, 0.1, shape)).astype(np.float32)
    den = mbirtorch.QGGMRFDenoiser(shape, compile_mode='off')
    den.configure_devices(devices=['cpu'])
    den.set_params(no_warning=True, verbose=0)
    out = {'noisy': noisy, 'sigma_est': np.array(den.estimate_image_noise_std(noisy))}
    for tag, sigma in (('given', 0.1), ('auto', None)):
        np.random.seed(13)
        d, dd = den.denoise(noisy, sigma_noise=sigma, max_iterations=4,
                            stop_threshold_change_pct=0.0, logfile_path=None, print_logs=False)
        rp = dd['recon_params']
        out[f'{tag}_out'] = d
        out[f'{tag}_alpha'] = np.array(rp['alpha_values'])
        out[f'{tag}_nmae_pct'] = np.array(rp['stop_threshold_change_pct'])
        out[f'{tag}_reg'] = np.array([rp['regularization_params'][k]
                                      for k in ('sigma_y', 'sigma_x', 'sigma_prox')])
    np.savez_compressed(os.path.join(HERE, 'denoise.npz'), **out)
    print('wrote denoise')


def recon_simple_parallel_case():
    """recon_simple_parallel at the reference's CPU configuration.  The
    phantom (128 x 128 x 16, unit voxels) is projected by a model of that
    recon shape; the one-call recon then runs at its default grid."""
    shape = (180, 16, 192)
    ang = np.linspace(0, np.pi, shape[0], endpoint=False)
    mp = _quiet(mbirtorch.ParallelBeamModel(shape, ang, compile_mode='off'))
    mp.set_params(no_warning=True, recon_shape=(128, 128, 16))
    ph = phantom((128, 128, 16), 61)
    clean = mp.forward_project(ph)
    rng = np.random.default_rng(62)
    sino = (clean + rng.normal(0, 0.01 * clean.max(), clean.shape)).astype(np.float32)
    # the data are rounded to float16 values (stored as float32 here), so the
    # fixture can hold them in half the bytes and still reproduce the input
    sino = sino.astype(np.float16).astype(np.float32)
    np.random.seed(63)
    import time
    t = time.perf_counter()
    rec, d = mbirtorch.recon_simple_parallel(sino, ang, max_iterations=10)
    secs = time.perf_counter() - t
    rp = d['recon_params']
    mask = vcd_utils.get_2d_ror_mask(rec.shape[:2]).astype(bool)
    np.savez_compressed(os.path.join(HERE, 'recon_simple_parallel_128.npz'),
                        sino_f16=sino.astype(np.float16), angles=ang,
                        recon_shape=np.array(rec.shape),
                        recon_ror=rec[mask].astype(np.float32),
                        fm_rmse=np.array(rp['fm_rmse']), alpha=np.array(rp['alpha_values']),
                        num_iterations=np.array(rp['num_iterations']),
                        reg=np.array([rp['regularization_params'][k]
                                      for k in ('sigma_y', 'sigma_x', 'sigma_prox')]),
                        seed=np.array(63), max_iterations=np.array(10),
                        reference_cpu_seconds=np.array(secs),
                        reference_cpu_threads=np.array(torch.get_num_threads()))
    print(f'wrote recon_simple_parallel_128 ({secs:.1f} s on the CPU)')


def autograd_case():
    """The reference's own autograd (forward_project_differentiable) on a
    parallel and a cone model: the gradient of sum w (A x - y)^2 at a seeded
    volume, with its inputs."""
    out = {}
    for tag in ('par', 'cone'):
        shape = (24, 16, 16)
        if tag == 'par':
            m = _quiet(mbirtorch.ParallelBeamModel(
                shape, np.linspace(0, np.pi, shape[0], endpoint=False), compile_mode='off'))
        else:
            m = _quiet(mbirtorch.ConeBeamModel(
                shape, np.linspace(0, 2 * np.pi, shape[0], endpoint=False),
                source_detector_dist=96.0, source_iso_dist=64.0, compile_mode='off'))
        m.configure_devices(devices=['cpu'])
        rs = tuple(m.get_params('recon_shape'))
        g = torch.Generator().manual_seed(71)
        x = torch.rand(rs, generator=g, dtype=torch.float32)
        y = torch.rand(shape, generator=g, dtype=torch.float32)
        w = torch.rand(shape, generator=g, dtype=torch.float32) + 0.5
        xr = x.clone().requires_grad_(True)
        from mbirtorch.autograd import forward_project_differentiable
        s = forward_project_differentiable(m, xr)
        loss = (w * (s - y) ** 2).sum()
        loss.backward()
        out[f'{tag}_x'], out[f'{tag}_y'], out[f'{tag}_w'] = x.numpy(), y.numpy(), w.numpy()
        out[f'{tag}_grad'] = xr.grad.numpy()
        out[f'{tag}_loss'] = np.array(float(loss))
        out[f'{tag}_recon_shape'] = np.array(rs)
    np.savez_compressed(os.path.join(HERE, 'autograd.npz'), **out)
    print('wrote autograd')


CASES = ['projector_cases', 'qggmrf_case', 'partition_case', 'autoreg_and_direct_cases',
         'recon_cases', 'prox_cases', 'denoise_case', 'recon_simple_parallel_case',
         'autograd_case']

if __name__ == '__main__':
    for name in (sys.argv[1:] or CASES):
        globals()[name]()
