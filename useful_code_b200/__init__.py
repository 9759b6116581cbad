"""B200-native Monte Carlo LIBOR-market-model pricing pipeline.

A drop-in for the GPU hot path of Kooderive (xcwork/Useful_Code): Sobol
generation and scrambling, Brownian bridge, pseudo-root correlation and
drift, predictor-corrector evolution, cash flows and discounting,
Longstaff–Schwartz regression and reductions.  The compute lives in the
CUDA library ``liblmm_b200.so`` (include/lmm_c.h); this package binds it:

* ``useful_code_b200._lib``      ctypes binding, typed from the C headers
* ``useful_code_b200.market``    model and product set-up (curves, vols,
  pseudo-roots, Sobol directions, scramblers, LS basis tables)
* ``useful_code_b200.pricer``    staged and fused Bermudan / European
  pricing pipelines driven through the C ABI

Importing fails if the CUDA library has not been built; there is no CPU
fallback.
"""
from ._lib import LIB, LmmError, call  # noqa: F401

__all__ = ["LIB", "LmmError", "call"]
