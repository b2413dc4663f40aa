"""B200-native IFE-PIC step (hot path of weqwoueu/pic-, PIC-IFE_GEC).

The compute lives in libpicgpu.so (CUDA, sm_100a) behind the C-ABI of
include/picgpu.h; this package binds it and mirrors the reference's main
loop on the host.
"""
from . import api  # noqa: F401
