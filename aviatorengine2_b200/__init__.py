"""B200-native ray/path-tracing hot path of AviatorEngine2.

The compute lives in libae_b200.so (hand-written CUDA for sm_100a behind a C
ABI, include/ae_b200.h); this package is the host-side mirror of the
reference's renderer interface over that ABI.
"""
from . import _lib
from ._lib import AeError, lib
from .renderer import Context, Renderer, RendererSettings
from .serving import Server

__all__ = ["AeError", "Context", "Renderer", "RendererSettings", "Server", "lib", "_lib"]
