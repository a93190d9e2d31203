"""Direct-recon (FBP / FDK) row filter.

The reference filters each detector row with a (2C-1)-tap space-domain ramp
in 'valid' mode through torch.fft (tomography_utils.py:18-78).  Here the
same filter runs through cuFFT on the device (torch.fft, a library FFT), in
one batched call; the back projection that follows is the sm_100a kernel.
"""

import numpy as np
import torch


def generate_direct_recon_filter(num_channels, filter_name="ramp"):
    """The (2C-1)-tap space-domain ramp filter (float32)."""
    if filter_name not in ("ramp",):
        raise ValueError("Unsupported filter. Supported filters are: ramp.")
    n = np.arange(-num_channels + 1, num_channels)
    f = 0.5 * np.sinc(n) - 0.25 * np.sinc(n / 2) ** 2
    return f.astype(np.float32)


def apply_row_filter(block, filter_arr, row_weight=None, rows_per_batch=1 << 16):
    """'valid' convolution of every detector row of ``block`` (V, R, C) with
    ``filter_arr`` (2C-1,), after an optional (R, C) pre-weight."""
    V, R, C = block.shape
    L = C + filter_arr.shape[0] - 1
    n_fft = 1 << int(np.ceil(np.log2(L)))
    filt_f = torch.fft.rfft(filter_arr.to(torch.float32), n=n_fft)
    rows = block.reshape(-1, C)
    out = torch.empty_like(rows)
    for r0 in range(0, rows.shape[0], rows_per_batch):
        win = rows[r0:r0 + rows_per_batch]
        if row_weight is not None:
            det_rows = torch.arange(r0, r0 + win.shape[0], device=block.device) % R
            win = win * row_weight[det_rows]
        full = torch.fft.irfft(torch.fft.rfft(win, n=n_fft, dim=1) * filt_f, n=n_fft, dim=1)
        out[r0:r0 + win.shape[0]] = full[:, C - 1:2 * C - 1]
    return out.reshape(V, R, C)
