"""Parameter storage and the run logger.

Semantics follow the reference's ParameterHandler (parameter_handler.py:
260-344):

* ``get_params(name)`` returns one value, ``get_params([names])`` a list;
  an unknown name raises NameError.
* ``set_params(**kw)``: an unknown name raises ValueError unless
  ``no_warning`` (the construction path, which adds it as a new
  recompile-flagged parameter).  Setting sigma_y / sigma_x / sigma_prox
  directly turns auto-regularization off (with a warning); setting
  sharpness or snr_db turns it back on.  A recompile-flagged change
  rebuilds the device projector.  No validity check runs here; it is
  deferred to reconstruction entry.
"""

import io
import itertools
import logging
import os
import warnings

import numpy as np

from . import _utils
from ._utils import Param

_counter = itertools.count(1)


class ParameterHandler:

    def __init__(self):
        self.params = _utils.get_default_params()
        self.logger_name = f'mbirtorch_b200.{type(self).__name__}.{next(_counter)}'
        self.logger = logging.getLogger(self.logger_name)
        self.logger.propagate = False
        self.logger.handlers.clear()
        h = logging.StreamHandler()
        h.setFormatter(logging.Formatter('%(message)s'))
        self.logger.addHandler(h)
        self.logger.setLevel(logging.INFO)
        self.log_buffer = None
        self._log_file_handler = None

    # ── logging ─────────────────────────────────────────────────────────────
    def setup_logger(self, logfile_path='~/.mbirtorch/logs/recon.log', print_logs=True):
        """Route this model's run log to a string buffer (kept in the recon
        dict), optionally the console, and optionally a file."""
        verbose = self.get_params('verbose')
        level = logging.WARNING if verbose <= 0 else (logging.INFO if verbose == 1
                                                      else logging.DEBUG)
        self.close_log_file()
        self.logger.handlers.clear()
        self.logger.setLevel(level)
        fmt = logging.Formatter('%(message)s')
        self.log_buffer = io.StringIO()
        bh = logging.StreamHandler(self.log_buffer)
        bh.setFormatter(fmt)
        self.logger.addHandler(bh)
        if print_logs:
            ch = logging.StreamHandler()
            ch.setFormatter(fmt)
            self.logger.addHandler(ch)
        if logfile_path:
            path = os.path.abspath(os.path.expanduser(logfile_path))
            os.makedirs(os.path.dirname(path), exist_ok=True)
            fh = logging.FileHandler(path, mode='w')
            fh.setFormatter(fmt)
            self.logger.addHandler(fh)
            self._log_file_handler = fh

    def close_log_file(self):
        fh = getattr(self, '_log_file_handler', None)
        if fh is not None:
            fh.flush()
            fh.close()
            self.logger.removeHandler(fh)
            self._log_file_handler = None

    # ── access ──────────────────────────────────────────────────────────────
    def get_params(self, parameter_names):
        if isinstance(parameter_names, str):
            if parameter_names not in self.params:
                raise NameError(f"'{parameter_names}' not a recognized parameter")
            return self.params[parameter_names].val
        out = []
        for name in parameter_names:
            if name not in self.params:
                raise NameError(f"'{name}' not a recognized parameter")
            out.append(self.params[name].val)
        return out

    @staticmethod
    def normalize_scalar(val):
        return val.item() if isinstance(val, np.generic) else val

    def set_params(self, no_warning=False, no_compile=False, **kwargs):
        recompile = False
        reg_change = False
        meta_change = False
        for key, val in kwargs.items():
            flag = True
            if key in self.params:
                flag = self.params[key].recompile_flag
            elif not no_warning:
                valid = '\n'.join(f'   {k}' for k in self.params)
                raise ValueError(f'{key} is not a recognized parameter\n'
                                 f'Valid parameters are: \n{valid}\n')
            self.params[key] = Param(self.normalize_scalar(val), flag)
            if flag:
                recompile = True
            elif key in ('sigma_y', 'sigma_x', 'sigma_prox'):
                reg_change = True
            elif key in ('sharpness', 'snr_db'):
                meta_change = True
        if reg_change and not no_warning:
            self.set_params(auto_regularize_flag=False)
            warnings.warn('You are directly setting regularization parameters, sigma_x, '
                          'sigma_y or sigma_prox. This is an advanced feature that will '
                          'disable auto-regularization.')
        if meta_change and self.get_params('auto_regularize_flag') is False:
            self.set_params(auto_regularize_flag=True)
            if not no_warning:
                warnings.warn('You have re-enabled auto-regularization by setting sharpness '
                              'or snr_db. It was previously disabled')
        if recompile and not no_compile:
            self.refresh_device_bindings()

    def refresh_device_bindings(self):
        """Geometry changed: drop the cached device projector."""

    def verify_valid_params(self):
        shape = self.get_params('sinogram_shape')
        if len(shape) != 3:
            raise ValueError(f'sinogram_shape must be (views, rows, channels); got {shape}')

    def print_params(self):
        verbose, vp_name = self.get_params(['verbose', 'view_params_name'])
        print('----')
        for key, entry in self.params.items():
            if verbose < 3 and key == vp_name:
                val = np.asarray(entry.val)
                print(f'{key} = array(shape={val.shape}, dtype={val.dtype})')
            else:
                print(f'{key} = {entry.val}')
        print('----')
