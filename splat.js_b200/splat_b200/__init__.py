"""splat_b200: B200-native Gaussian-splat training step for splat.js.

The compute path is the CUDA library ``libsplat_b200.so`` (C ABI declared in
include/splat_b200.h).  This package is the host-side mirror of the
reference's ``GSTrainer`` (src/gs/trainer.js) over that ABI.
"""
from . import scene  # noqa: F401
