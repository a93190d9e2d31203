"""CPU oracle for the mbirtorch reconstruction hot path -- TEST INFRASTRUCTURE.

This package restates the reference algorithm (mbirtorch v0.0.2) on the CPU
in FP64 so that the sm_100a kernels of ``mbirtorch_b200`` can be checked
against it.  It checks results and is never the thing measured or shipped: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import it, and nothing in ``mbirtorch_b200`` does.

Parity of the oracle itself is pinned against golden vectors produced by the
reference's own torch bodies (``tests/golden/make_golden.py``, checked by
``tests/test_oracle_golden.py``).

Contents:
  * ``oracle_proj.c`` -- the four projector bodies (parallel/cone, forward/
    back), compiled with gcc into ``oracle/_build/liboracle.so``.
  * :mod:`oracle.projectors` -- ctypes wrappers with numpy in/out.
  * :mod:`oracle.qggmrf` -- the qGGMRF surrogate gradient/Hessian.
  * :mod:`oracle.vcd` -- partitions, the VCD subset update and a small recon
    driver, calling the C projectors.
"""

from .projectors import (OracleGeometry, build, cone_back, cone_forward,  # noqa: F401
                         library_path, parallel_back, parallel_forward)
