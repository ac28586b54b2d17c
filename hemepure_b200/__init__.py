"""hemepure_b200: B200-native D3Q19 collide-and-stream for HemePure's lb::LBM hot path.

The compute path is libhemeb200.so (hand-written CUDA for sm_100a behind a C
ABI, include/hemeb200.h); this package holds its Python binding, the synthetic
vessel generator, the build script and the serving layer.
"""

from .lbm import LBM, HemeLBError, Unstable, library  # noqa: F401

__all__ = ["LBM", "HemeLBError", "Unstable", "library"]
