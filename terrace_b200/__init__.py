"""terrace_b200 -- B200-native (sm_100a) Terrace dynamic-graph hot path.

The product is libterrace_b200.so (C ABI: include/terrace_b200.h); this
package is its Python mirror of the reference Graph API.  Importing the
package does not load the library; constructing a Graph does, and raises if
the library was not built (there is no CPU fallback).
"""
from ._lib import (TRC_DEVICE_PTR, TRC_DROP_SELF_LOOPS, TRC_SYMMETRIZE, TRC_UNREACHED,  # noqa: F401
                   TrcError, LIB_PATH)
from .graph import Graph, rmat_generate  # noqa: F401
from .server import Server  # noqa: F401

__all__ = ["Graph", "Server", "rmat_generate", "TrcError", "TRC_UNREACHED", "LIB_PATH"]
