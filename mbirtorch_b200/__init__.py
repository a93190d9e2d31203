"""mbirtorch_b200: the MBIR reconstruction hot path of mbirtorch on B200.

The parallel-beam and cone-beam (flat, curved, helical) projector pair and
the VCD voxel-subset update with its qGGMRF prior run as hand-written
sm_100a CUDA kernels behind a plain C ABI (include/mbir_b200.h,
``libmbir_b200.so``).  This package is the host side: it keeps mbirtorch's
model API (``TomographyModel``, ``ParallelBeamModel``, ``ConeBeamModel``,
``recon``, ``forward_project``/``back_project``, ``recon_simple_*``, the
autograd entry points) so a user of that API can switch.
"""

__version__ = "0.1.0"

from .autograd import (TorchProjector, back_project_differentiable,  # noqa: F401
                       forward_project_differentiable, weighted_residual_loss)
from .cone_beam import ConeBeamModel, recon_simple_cone  # noqa: F401
from .denoising import QGGMRFDenoiser  # noqa: F401
from .parallel_beam import ParallelBeamModel, recon_simple_parallel  # noqa: F401
from .qggmrf import get_b_from_nbr_wts, qggmrf_loss  # noqa: F401
from .tomography_model import TomographyModel  # noqa: F401
from .vcd_utils import (gen_full_indices, gen_partition_sequence, gen_pixel_partition,  # noqa
                        gen_set_of_pixel_partitions, gen_weights, get_2d_ror_mask)

__all__ = [
    "ParallelBeamModel", "ConeBeamModel", "TomographyModel", "QGGMRFDenoiser",
    "recon_simple_parallel",
    "recon_simple_cone", "TorchProjector", "forward_project_differentiable",
    "back_project_differentiable", "weighted_residual_loss", "gen_weights",
    "gen_full_indices", "gen_pixel_partition", "gen_set_of_pixel_partitions",
    "gen_partition_sequence", "get_2d_ror_mask", "get_b_from_nbr_wts", "qggmrf_loss",
]
