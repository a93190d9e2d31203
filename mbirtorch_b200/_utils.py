"""Parameter records and defaults.

The parameter names, default values and recompile flags are part of the
public API a user of the reference relies on (``get_params`` /
``set_params``), so they are kept identical to mbirtorch's ``_utils.py``
(reference v0.0.2, _utils.py:56-115).
"""

import copy
from dataclasses import dataclass
from typing import Any

FILE_FORMAT_NUMBER = 1.0


@dataclass
class Param:
    val: Any
    recompile_flag: bool = True


def _defaults():
    p = Param
    return {
        # forward model
        'geometry_type': p(None, False),
        'file_format': p(FILE_FORMAT_NUMBER, False),
        'sinogram_shape': p(None, True),
        'delta_det_channel': p(1.0, True),
        'delta_det_row': p(1.0, True),
        'det_row_offset': p(0.0, True),
        'det_channel_offset': p(0.0, True),
        'sigma_y': p(1.0, False),
        'alu_unit': p(None, False),
        'alu_value': p(1.0, False),
        # recon model
        'recon_shape': p(None, True),
        'delta_voxel': p(None, True),
        'voxel_row_aspect': p(1.0, True),
        'voxel_slice_aspect': p(1.0, True),
        'sigma_x': p(1.0, False),
        'sigma_prox': p(1.0, False),
        'p': p(2.0, False),
        'q': p(1.2, False),
        'T': p(1.0, False),
        'qggmrf_nbr_wts': p([1.0, 1.0, 1.0], False),
        # reconstruction
        'auto_regularize_flag': p(True, False),
        'positivity_flag': p(False, False),
        'snr_db': p(30.0, False),
        'sharpness': p(1.0, False),
        'granularity': p([1, 2, 4, 8, 16, 32, 64, 128, 128, 128, 128], False),
        'partition_sequence': p([2, 4, 6] + [7, 8, 9, 10] * 25, False),
        'verbose': p(1, False),
        'max_alpha': p(1.5, False),
        'use_ror_mask': p(True, False),
    }


_DEFAULTS = _defaults()

recon_param_names = ['num_iterations', 'granularity', 'partition_sequence', 'fm_rmse',
                     'prior_loss', 'regularization_params', 'stop_threshold_change_pct',
                     'alpha_values', 'delta_norm_per_slice']

AUTO_REGULARIZATION_PARAM_NAMES = ('sigma_y', 'sigma_x', 'sigma_prox')


def get_default_params():
    return copy.deepcopy(_DEFAULTS)
