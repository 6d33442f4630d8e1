"""The decoder sources under UndefinedBehaviorSanitizer (CPU only).

The host same-source build (one lane per chain) is compiled again with
-fsanitize=undefined and aborts on the first report; it must decode mixed
SILK / hybrid / CELT streams, mono and stereo, with lost packets, DTX frames
and in-band FEC, to libopus's samples.  Integer overflow in a signed type, an
out-of-range shift or a misaligned access anywhere in the decoder fails it."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import corpus, ogg_port, ref_decode

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cuopus_b200", "csrc")


def _lossy(packets, seed, p_lost, p_dtx):
    rng = np.random.default_rng(seed)
    out = []
    for p in packets:
        u = rng.random()
        if u < p_lost:
            out.append(b"")
        elif u < p_lost + p_dtx and (p[0] & 3) == 0:
            out.append(p[:1])
        else:
            out.append(p)
    return out


@pytest.fixture(scope="module")
def hc_ubsan(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ is not installed")
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.skip(str(e))
    out = str(tmp_path_factory.mktemp("ubsan") / "libhc_ubsan.so")
    r = subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-w", "-fsanitize=undefined",
                        "-fno-sanitize-recover=all", "-I", CSRC, os.path.join(CSRC, "hostcheck.cpp"), "-o", out,
                        "-lpthread"], capture_output=True, text=True)
    if r.returncode != 0 and "ubsan" in (r.stderr + r.stdout).lower():
        pytest.skip("UBSan runtime unavailable: " + r.stderr[-200:])
    assert r.returncode == 0, r.stderr[-2000:]
    return out


def _decode_all(lib_path):
    """Decode the streams with the sanitised build; raises on a mismatch (a
    sanitizer report aborts the process)."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_host_parity import host_decode
    hc = ctypes.CDLL(lib_path)
    for seed in range(12):
        spec = dict(kind="mixed", seed=78000 + seed, seconds=2.5, channels=1 + seed % 2)
        if seed % 3 == 0:
            spec.update(inband_fec=1, loss_perc=20, dtx=1)
        ix = ogg_port.demux(corpus.make_stream(spec))
        pk = _lossy(ix["packets"], seed, 0.08 if seed % 2 else 0.0, 0.05)
        for fec in (0, 1):
            ref = ref_decode.decode_chains(pk, [(0, len(pk))], ix["channels"], fec=fec)
            pcm, ns, rg, stop, _ = host_decode(hc, pk, [(0, len(pk))], ix["channels"], fec=fec)[0]
            assert stop == int(ref["status"][0])
            assert np.array_equal(ns, ref["nsamp"][0]) and np.array_equal(rg, ref["rng"][0])
            assert np.array_equal(pcm, ref["pcm"][0]), (seed, fec)


def test_decoder_has_no_undefined_behaviour(hc_ubsan):
    """Run in a child process, so that a sanitizer report (which aborts) fails
    this test with the report instead of ending the test run."""
    import sys
    env = dict(os.environ, UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1",
               PYTHONPATH=os.pathsep.join([ROOT, os.environ.get("PYTHONPATH", "")]))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), hc_ubsan], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]


if __name__ == "__main__":
    import sys
    _decode_all(sys.argv[1])
