"""The C ABI library loads on a machine without a GPU and exports every entry
point include/cuopus.h declares (no compute call is made here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cuopus.h")
LIB = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus.so")

REFERENCE_EIGHT = ["cuopus_probe", "cuopus_decode_f16k", "cuopus_decode_f16k_on", "cuopus_decode_f16k_multi",
                   "cuopus_warmup", "cuopus_last_arena_overflow", "cuopus_workspace_bytes",
                   "cuopus_release_workspaces"]


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cuopus_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_reference_surface():
    names = declared()
    for n in REFERENCE_EIGHT:
        assert n in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "libcuopus.so must be built (python -m cuopus_b200.build)"
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    assert set(declared()) <= exported


def test_python_surface_matches_reference_module():
    from cuopus_b200 import cuopus_native as cn
    for name in ("probe", "decode_ogg_to_cuda_tensor", "decode_ogg_multi", "warmup", "workspace_bytes",
                 "last_arena_overflow", "release_workspaces", "CuopusError"):
        assert hasattr(cn, name), name


def test_host_only_calls_without_gpu():
    """Calls that never touch the device work on a CPU-only machine."""
    from cuopus_b200 import cuopus_native as cn
    assert cn.workspace_bytes() >= 0
    assert cn.last_arena_overflow() in (False, True)
    assert cn.lib().cuopus_slot_bytes() > 0
    assert cn.lib().cuopus_default_width() in (1, 2, 4, 8, 16, 32)


def test_no_cpu_fallback_on_the_decode_path():
    """Without a GPU the decode entry points fail with a CUDA error code,
    never by decoding on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cuopus_b200 import cuopus_native as cn
    data = open(os.path.join(ROOT, "tests", "golden", "streams", "plain_a.opus"), "rb").read()
    n16 = cn.probe(data)
    lib = cn.lib()
    buf = (ctypes.c_float * n16)()
    out_len = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(256)
    rc = lib.cuopus_decode_f16k_on(data, len(data), ctypes.cast(buf, ctypes.c_void_p), n16,
                                   ctypes.byref(out_len), None, err, 256)
    assert rc == 2, (rc, err.value)
    assert out_len.value == 0


PHASES_HEADER = os.path.join(ROOT, "include", "cuopus_phases.h")
PHASES_LIB = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus_phases.so")


def test_stage_timer_build_exports_both_headers():
    """libcuopus_phases.so is the product library plus the stage timers; the
    product library itself carries no timers."""
    src = re.sub(r"/\*.*?\*/", "", open(PHASES_HEADER).read(), flags=re.S)
    timer_names = sorted(set(re.findall(r"\b(cuopus_[a-z0-9_]+)\s*\(", src)))
    assert timer_names == ["cuopus_phase_count", "cuopus_phase_read", "cuopus_phase_reset"]
    lib = ctypes.CDLL(PHASES_LIB)
    missing = [n for n in declared() + timer_names if not hasattr(lib, n)]
    assert not missing, missing
    from cuopus_b200 import cuopus_native as cn
    assert lib.cuopus_phase_count() == len(cn.PHASE_NAMES)
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    assert "cuopus_phase_read" not in out


def test_tail_scheduling_arguments_are_checked():
    """light_sms needs the queue schedule and every lane: other combinations
    are refused with RC 3 before any device work."""
    from cuopus_b200 import cuopus_native as cn
    lib = cn.lib()
    b = cn.Batch()
    for f in ("data", "off", "len", "first", "npkts", "channels", "trim", "keep", "res"):
        setattr(b, f, 16)   # never dereferenced: the call is refused first
    b.nchains, b.width, b.block, b.light_sms, b.long_chains = 4, 32, 64, 2, 2
    err = ctypes.create_string_buffer(256)
    for schedule, scalar in ((2, 0), (0, 0), (1, 1)):
        b.schedule, b.scalar = schedule, scalar
        rc = lib.cuopus_decode_batch(ctypes.byref(b), None, None, err, 256)
        assert rc == 3 and b"tail scheduling" in err.value
