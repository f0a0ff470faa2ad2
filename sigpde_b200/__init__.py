"""sigpde_b200 -- B200-native (sm_100a) signature-kernel engine.

`sigpde_b200.torch` keeps the `sigpde.torch` API of stojl/SigPDE; the hot
path runs in libsigk.so (hand-written CUDA, C ABI in include/sigk.h).
"""
__version__ = "0.1.0"

__all__ = ["torch"]
