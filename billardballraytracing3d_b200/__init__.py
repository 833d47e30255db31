"""B200-native (sm_100a) multi-bounce specular trace loop.

The product is libbbrt_cuda.so (built in-tree from csrc/ by build.py) behind
the C ABI of include/bbrt.h.  `api.Scene` drives that ABI from Python; the
C++ headers under include/bbrt/ mirror the reference's class API on top of
it.  `scenes` generates the synthetic patch sets and ray sources.
"""
from . import scenes  # noqa: F401

__all__ = ["scenes", "api", "build"]
