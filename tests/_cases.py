"""Helpers shared by the CPU and GPU tests: rebuild the golden fixtures'
geometries as oracle geometries and as mbirtorch_b200 models."""

import glob
import json
import os

import numpy as np

from conftest import GOLDEN

PROJECTOR_FILES = sorted(glob.glob(os.path.join(GOLDEN, "projectors_*.npz")))
PROJECTOR_NAMES = [os.path.basename(f)[len("projectors_"):-4] for f in PROJECTOR_FILES]


def expand(spec):
    """['linspace', a, b, n] -> endpoint-free linspace; 'linspace_closed'
    includes the end point; anything else passes through."""
    if isinstance(spec, (list, tuple)) and spec and spec[0] == 'linspace':
        return np.linspace(spec[1], spec[2], int(spec[3]), endpoint=False)
    if isinstance(spec, (list, tuple)) and spec and spec[0] == 'linspace_closed':
        return np.linspace(spec[1], spec[2], int(spec[3]))
    if isinstance(spec, list):
        return tuple(spec)
    return spec


def load_projector_case(name):
    return np.load(os.path.join(GOLDEN, f"projectors_{name}.npz"))


def oracle_geometry(d):
    """OracleGeometry from a projector fixture's stored geometry scalars."""
    from oracle import OracleGeometry
    ss, rs = d['sinogram_shape'], d['recon_shape']
    dv = float(d['delta_voxel'])
    g = OracleGeometry(
        num_det_rows=int(ss[1]), num_det_channels=int(ss[2]),
        num_recon_rows=int(rs[0]), num_recon_cols=int(rs[1]), num_slices=int(rs[2]),
        delta_det_channel=float(d['delta_det_channel']),
        delta_det_row=float(d['delta_det_row']),
        det_channel_offset=float(d['det_channel_offset']),
        det_row_offset=float(d['det_row_offset']),
        delta_voxel=dv, delta_voxel_row=dv * float(d['voxel_row_aspect']),
        delta_voxel_slice=dv * float(d['voxel_slice_aspect']),
        psf_radius=int(d['psf_radius']))
    if 'bp_psf_radius' in d.files:
        g.bp_psf_radius = int(d['bp_psf_radius'])
        g.source_detector_dist = float(d['source_detector_dist'])
        g.magnification = float(d['magnification'])
        g.recon_slice_offset = float(d['recon_slice_offset'])
        g.use_curved_detector = bool(d['use_curved_detector'])
    return g


def is_cone(d):
    return 'bp_psf_radius' in d.files


def oracle_forward(d, values, idx):
    import oracle
    g = oracle_geometry(d)
    vp = d['view_params'].astype(np.float64)
    if is_cone(d):
        return oracle.cone_forward(g, vp, values, idx)
    return oracle.parallel_forward(g, vp, values, idx)


def oracle_back(d, sino, idx, coeff_power=1):
    import oracle
    g = oracle_geometry(d)
    vp = d['view_params'].astype(np.float64)
    if is_cone(d):
        return oracle.cone_back(g, vp, sino, idx, coeff_power)
    return oracle.parallel_back(g, vp, sino, idx, coeff_power)


def build_model(d, **extra):
    """The same model in mbirtorch_b200 (constructor + set_params)."""
    import mbirtorch_b200 as mb
    spec = json.loads(str(d['ctor']))
    kw = {k: expand(v) for k, v in spec['ctor'].items()}
    shape = kw.pop('sinogram_shape')
    angles = kw.pop('angles')
    if spec['geometry'] == 'parallel':
        m = mb.ParallelBeamModel(shape, angles, **extra, **kw)
    else:
        m = mb.ConeBeamModel(shape, angles, **extra, **kw)
    m.set_params(no_warning=True, verbose=0)
    if spec['set_params']:
        m.set_params(no_warning=True, **spec['set_params'])
    return m


def oracle_problem(m):
    """The oracle's view of an mbirtorch_b200 model: same geometry scalars,
    view parameters and recon shape."""
    from oracle import OracleGeometry, vcd
    g = m._geometry()
    og = OracleGeometry(
        num_det_rows=g.num_det_rows, num_det_channels=g.num_det_channels,
        num_recon_rows=g.num_recon_rows, num_recon_cols=g.num_recon_cols,
        num_slices=g.num_slices, delta_det_channel=g.delta_det_channel,
        delta_det_row=g.delta_det_row, det_channel_offset=g.det_channel_offset,
        det_row_offset=g.det_row_offset, delta_voxel=g.delta_voxel,
        delta_voxel_row=g.delta_voxel_row, delta_voxel_slice=g.delta_voxel_slice,
        recon_slice_offset=g.recon_slice_offset, magnification=g.magnification,
        source_detector_dist=g.source_detector_dist,
        use_curved_detector=bool(g.use_curved_detector), psf_radius=g.psf_radius,
        bp_psf_radius=g.bp_psf_radius)
    kind = 'cone' if g.geometry == 1 else 'parallel'
    return vcd.Problem(kind, og, m._view_params_array(), m.get_params('recon_shape'),
                       source_iso_dist=m.get_params('source_iso_dist') if kind == 'cone'
                       else None)
