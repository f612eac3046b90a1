"""nlsb200: B200-native Lanczos exponential integrators (KG / phi^4 / NLSE).

Host package over the C ABI of lib/libnlsb200.so (include/nlsb200.h).
"""
from ._lib import (BIN_DIR, FP32, FP64, KG_GAUTSCHI, KG_SV, LIB_PATH, NL_CQ, NL_DSINE, NL_POLY, NL_SAT, NL_SINE,
                   NL_SINH, NLSE_SEWI, NLSE_SS2, SP4_GAUTSCHI, SP4_SV, SYMBOLS, NlsError, build, lib)
from .solver import (Pool, Solver, Spec, downsample_fft, downsample_fft_3d, downsample_interpolation,
                     downsample_interpolation_3d, pinned_empty, reference_phi4_rm)

__all__ = ["Solver", "Pool", "Spec", "NlsError", "build", "lib", "LIB_PATH", "BIN_DIR",
           "SYMBOLS", "KG_GAUTSCHI", "KG_SV", "SP4_SV", "SP4_GAUTSCHI", "NLSE_SS2",
           "NLSE_SEWI", "FP32", "FP64", "reference_phi4_rm", "pinned_empty", "downsample_interpolation",
           "downsample_interpolation_3d", "downsample_fft", "downsample_fft_3d", "NL_POLY", "NL_SINE", "NL_DSINE", "NL_SINH", "NL_CQ", "NL_SAT"]
