"""B200-native key search for onion-gen's device hot path.

The engine (``gpu.Engine``) is sm_100a CUDA behind the C ABI in
``include/onion_gen_b200.h``; ``filter`` and ``key`` expose the host side of
the hit path through the same library. Importing this package loads
``libonion_gen_b200.so`` and fails loudly if it is missing.
"""
from . import _native  # noqa: F401  (loads the library or raises)
from . import batch, filter, gpu, key, serve  # noqa: F401

__all__ = ["gpu", "batch", "serve", "filter", "key"]
