"""Coverage of the frame-level branches of opus_decode_frame (CPU only).

Redundancy frames in both directions (celt_to_silk = 1 before the SILK frame,
0 after it, src/opus_decoder.c:458-476 / :532-552), mode transitions that
conceal 5 ms of the previous mode and crossfade it in (:347, smooth_fade at
:205), and the silence frame the CELT layer decodes when hybrid switches to
SILK (:441-452): the host build of the decoder counts, frame by frame, which of
these branches ran (hc_frame_events).  The streams the GPU parity tests decode
must reach each of them, and the spliced chains of tests/branches.py reach the
transitions without redundancy that encoded streams never contain; those
chains decode to libopus's samples here and on the GPU (test_gpu_parity.py).
"""
import ctypes
import os
import sys

import numpy as np
import pytest

from oracle import corpus, ogg_port, ref_decode

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from branches import spliced_chains  # noqa: E402
from test_host_parity import host_decode  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOSTCHECK = os.path.join(ROOT, "cuopus_b200", "lib", "libcuopus_hostcheck.so")
EV = ["frames", "redundancy_celt_to_silk", "redundancy_silk_to_celt", "transition_crossfade", "hybrid_to_silk_silence",
      "concealment_frames", "transition_to_celt", "transition_from_celt"]


@pytest.fixture(scope="module")
def hc():
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.fail(str(e))
    lib = ctypes.CDLL(HOSTCHECK)
    lib.hc_frame_events.argtypes = [ctypes.c_void_p]
    return lib


def _events(hc):
    a = (ctypes.c_ulonglong * 8)()
    hc.hc_frame_events(a)
    return dict(zip(EV, [int(v) for v in a]))


def _decode_streams(hc, specs):
    _events(hc)
    for spec in specs:
        ix = ogg_port.demux(corpus.make_stream(spec))
        host_decode(hc, ix["packets"], [(0, len(ix["packets"]))], ix["channels"])
    return _events(hc)


def test_gpu_test_streams_reach_redundancy_transitions_and_silence(hc):
    """The mixed streams of test_gpu_parity.py (the segmented-chain set at
    every width, and the 24 whole streams) contain redundancy frames in both
    directions, SILK -> CELT crossfades, hybrid -> SILK silence frames and
    concealment frames."""
    specs = [dict(kind="mixed", seed=6000 + w + s, seconds=4.0, channels=1 + s % 2)
             for w in (32, 16, 8, 4, 1) for s in range(4)]
    rng = np.random.default_rng(77)
    for s in range(24):
        ch = int(rng.integers(1, 3))
        specs.append(dict(kind="mixed", seed=7000 + s, seconds=float(rng.uniform(0.5, 6)), channels=ch))
    ev = _decode_streams(hc, specs)
    for k in ("redundancy_celt_to_silk", "redundancy_silk_to_celt", "transition_crossfade",
              "hybrid_to_silk_silence", "concealment_frames", "transition_to_celt"):
        assert ev[k] > 0, (k, ev)


@pytest.mark.parametrize("channels", [1, 2])
def test_spliced_mode_changes(hc, channels):
    """Every mode change without redundancy, CELT -> SILK / hybrid included:
    the host build decodes the spliced chains to libopus's samples, and the
    crossfades from and to CELT both run."""
    packets, chains = spliced_chains(channels)
    _events(hc)
    got = host_decode(hc, packets, chains, channels)
    ev = _events(hc)
    ref = ref_decode.decode_chains(packets, chains, channels)
    for i, (pcm, ns, rg, stop, _) in enumerate(got):
        assert stop == int(ref["status"][i]) == 0
        assert np.array_equal(ns, ref["nsamp"][i]) and np.array_equal(rg, ref["rng"][i]), i
        assert np.array_equal(pcm, ref["pcm"][i]), i
    assert ev["transition_from_celt"] >= 2 and ev["transition_to_celt"] >= 2, ev
    assert ev["hybrid_to_silk_silence"] >= 1, ev
