"""B200 wavefront path tracer with the scene-object API of andrea-luongo/open_rendering_framework.

The compute path is hand-written sm_100a CUDA behind the C ABI in include/orf_b200.h
(libpt_b200.so in this package).  ``_native`` binds that ABI; ``scene`` mirrors the reference's
Integrator / Camera / Background / Light / Material classes over it.
"""
from . import _native  # noqa: F401

__all__ = ["_native"]
