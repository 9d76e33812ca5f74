"""ysim_b200 -- B200 (sm_100a) implementation of ysim's per-substep cloth hot path.

The compute path is the CUDA library ysim_b200/lib/libysim_b200.so behind the C
ABI in include/ysim_b200.h; this package is its Python host binding.  There is
no CPU fallback: if the library is missing the import of ``ysim_b200.scene``
fails loudly.
"""
from . import generators  # noqa: F401

__all__ = ["generators", "scene", "build"]
