"""cuopus_b200: batched libopus-exact Opus decoding on NVIDIA B200 (sm_100a).

The product is the native library cuopus_b200/lib/libcuopus.so (C ABI in
include/cuopus.h); cuopus_b200.cuopus_native is its Python surface, the same
as the reference's cuopus_native module.
"""
from . import cuopus_native  # noqa: F401
from .cuopus_native import (CuopusError, decode_ogg_multi, decode_ogg_to_cuda_tensor,  # noqa: F401
                            last_arena_overflow, probe, release_workspaces, warmup, workspace_bytes)
