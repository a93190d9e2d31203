"""Availability probe and per-device value self-checks of the sm_100a kernels.

The counterpart of the reference's kernel_availability.py:86-133 (the
process-wide probe) and :204-219 (the per-kernel, per-device gate).  Both
answer with a ``(usable, reason)`` pair and never raise: a caller that only
asks whether the kernels are there must not be broken by the asking.

* :func:`kernels_available` -- once per process: the library loads, its ABI
  version is the one this package binds, CUDA is present, and device 0 is a
  compute-capability 10.0 part (the library carries sm_100a code only).
* :func:`projectors_usable` -- once per device: a tiny parallel and a tiny
  cone problem run through the projector pair on that device and must satisfy
  the adjoint identity <A x, y> = <x, A^T y>, give the same sum when a cone
  volume is projected as two slice bands, and repeat bit for bit.  There is no
  second implementation in this package to compare against (no CPU or eager
  fallback exists), so the checks are properties the projectors must have.

Unlike the reference, a ``False`` here does not select another code path:
this package has none.  :func:`require_usable` turns the answer into a
``RuntimeError`` carrying the reason; the reference-side integration (the
``_view_batch_bodies()`` seam) uses the pair to keep its own torch bodies.
"""

import os

import numpy as np
import torch

from . import _lib

#: Set to 1 to report the kernels unavailable (a bisection handle, as the
#: reference's MBIRTORCH_DISABLE_TRITON).
DISABLE_ENV_VAR = 'MBIRTORCH_B200_DISABLE'

#: Relative tolerance of the value self-checks (the reference's figure).
SELF_CHECK_REL_TOL = 1e-4

ABI_VERSION = 10100

_PROBE_RESULT = None
_DEVICE_RESULTS = {}


def kernels_available():
    """(usable, reason): whether the sm_100a library can run in this
    process.  Cached; never raises."""
    global _PROBE_RESULT
    if _PROBE_RESULT is None:
        _PROBE_RESULT = _probe()
    return _PROBE_RESULT


def _probe():
    if os.environ.get(DISABLE_ENV_VAR, '0') == '1':
        return False, f'disabled by {DISABLE_ENV_VAR}=1'
    try:
        version = int(_lib.query(None, 'mbir_abi_version'))
        if version != ABI_VERSION:
            return False, f'libmbir_b200.so has ABI {version}, this package binds {ABI_VERSION}'
        if not torch.cuda.is_available():
            return False, 'not a CUDA platform (torch.cuda is unavailable)'
        major, minor = torch.cuda.get_device_capability(0)
        if (major, minor) != (10, 0):
            return False, (f'device 0 is compute capability {major}.{minor}; the library '
                           'carries sm_100a code only')
        return True, f'available (ABI {version}, {torch.cuda.get_device_name(0)})'
    except Exception as e:  # noqa: BLE001 -- every failure becomes a reason
        return False, f'library failed to load: {type(e).__name__}: {e}'


def projectors_usable(device):
    """(usable, reason): whether the projector pair reproduces its required
    properties on ``device``.  Cached per device; never raises."""
    ok, reason = kernels_available()
    if not ok:
        return ok, reason
    key = str(torch.device(device))
    if key not in _DEVICE_RESULTS:
        _DEVICE_RESULTS[key] = _self_check(key)
    return _DEVICE_RESULTS[key]


def require_usable(device):
    """Raise ``RuntimeError`` with the reason when the kernels cannot run on
    ``device``."""
    ok, reason = projectors_usable(device)
    if not ok:
        raise RuntimeError(f'mbirtorch_b200 kernels unusable on {device}: {reason}')


def _rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-30)


def _cells(device):
    """The two tiny problems, built like the reference's self-check cells
    (kernel_availability.py:222-275): 4 views, a 10 x 10 detector, the
    models' default recon geometry (so the tap radii follow from it), and
    one pixel left out of the full index set (so no launch tile is full)."""
    from .cone_beam import ConeBeamModel
    from .parallel_beam import ParallelBeamModel
    from .vcd_utils import gen_full_indices
    cell = (4, 10, 10)
    par = ParallelBeamModel(cell, np.linspace(0, np.pi, cell[0], endpoint=False))
    cone = ConeBeamModel(cell, np.linspace(0, 2 * np.pi, cell[0], endpoint=False),
                         source_detector_dist=4.0 * cell[2], source_iso_dist=2.0 * cell[2])
    out = []
    for name, m in (('parallel', par), ('cone', cone)):
        m.set_params(no_warning=True, verbose=0)
        m.configure_devices(devices=[str(device)])
        idx = torch.as_tensor(np.asarray(gen_full_indices(m.get_params('recon_shape')))[:-1],
                              dtype=torch.int64, device=device)
        out.append((name, m.projector, idx))
    return out


def _self_check(device_key):
    try:
        device = torch.device(device_key)
        gen = torch.Generator().manual_seed(0)
        worst = 0.0
        for name, proj, idx in _cells(device):
            g = proj.geom
            x = torch.rand((idx.shape[0], g.num_slices), generator=gen).to(device)
            y = torch.rand(proj.sino_shape, generator=gen).to(device)
            ax = proj.forward(x, idx)
            aty = proj.back(y, idx)
            lhs = float(torch.sum(ax.double() * y.double()))
            rhs = float(torch.sum(x.double() * aty.double()))
            worst = max(worst, _rel(lhs, rhs))
            if not torch.equal(ax, proj.forward(x, idx)) or not torch.equal(aty,
                                                                           proj.back(y, idx)):
                return False, f'{name} projectors are not repeatable on {device_key}'
            if name == 'cone':
                k = g.num_slices // 3
                bands = proj.forward(x[:, :k].contiguous(), idx, slice_start=0) + \
                    proj.forward(x[:, k:].contiguous(), idx, slice_start=k)
                worst = max(worst, float((bands - ax).abs().max()) /
                            max(float(ax.abs().max()), 1e-30))
        torch.cuda.synchronize(device)
        if worst > SELF_CHECK_REL_TOL:
            return False, (f'projector self-check on {device_key}: relative gap {worst:.3g} '
                           f'above {SELF_CHECK_REL_TOL:g}')
        return True, f'projector self-check passed on {device_key} (worst gap {worst:.2g})'
    except Exception as e:  # noqa: BLE001
        return False, f'projector self-check failed to run: {type(e).__name__}: {e}'
