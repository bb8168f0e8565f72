"""B200-native RCWA diffraction-efficiency engine (host-side Python binding).

The compute path is the CUDA library ``openrcwa_b200/lib/librcwa_b200.so``
behind the C ABI of ``include/rcwa_b200.h``.
"""
from .abi import (Engine, Mlp, Plan, RcwaError, Stack, TableStack, Tuner, load, EXPORTS, RCWA_CONTINUOUS_XY,  # noqa: F401
                  RCWA_DISCONTINUOUS_X, RCWA_DISCONTINUOUS_Y, RCWA_PREC_FP64, RCWA_PREC_MIXED,
                  RCWA_TUNE_LU, RCWA_TUNE_SCHUR, RCWA_TUNE_PRODUCT, RCWA_TUNING_OFF, RCWA_TUNING_TABLE,
                  RCWA_TUNING_AUTO, eig_cluster_size, lu_cluster_size, set_eig_cluster, set_lu_cluster,
                  set_qr_sweep_limit)
