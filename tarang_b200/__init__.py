"""tarang_b200: B200-native pseudo-spectral time-step path of Tarang-4.0.

The product is the sm_100a library ``libtarang_gpu.so`` behind the C ABI in
``include/tarang_gpu.h``; this package binds it (``_lib``), mirrors the reference's
solver classes (``solver``), builds initial conditions (``ic``) and drives the serving loop.
"""

from . import _lib  # noqa: F401

__all__ = ["_lib", "solver", "ic", "build"]
