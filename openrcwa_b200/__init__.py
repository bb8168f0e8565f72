"""B200-native RCWA diffraction-efficiency engine (host-side Python binding).

The compute path is the CUDA library ``openrcwa_b200/lib/librcwa_b200.so``
behind the C ABI of ``include/rcwa_b200.h``.
"""
from .abi import (Engine, Mlp, Plan, RcwaError, Stack, load, EXPORTS, RCWA_CONTINUOUS_XY,  # noqa: F401
                  RCWA_DISCONTINUOUS_X, RCWA_DISCONTINUOUS_Y, RCWA_PREC_FP64, RCWA_PREC_MIXED)
