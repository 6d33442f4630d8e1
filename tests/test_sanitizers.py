"""The decoder and demuxer sources under the sanitizers (CPU only).

The host same-source build (one lane per chain) is compiled again with
-fsanitize=address,undefined (UBSan alone where g++ has no ASan runtime) and
aborts on the first report; it must decode mixed
SILK / hybrid / CELT streams, mono and stereo, with lost packets, DTX frames
and in-band FEC, and chains ending in random packets, to libopus's samples.
Integer overflow in a signed type, an out-of-range shift, a misaligned access
or a read or write out of bounds anywhere in the decoder fails it.
The host demuxer is built with AddressSanitizer as well and parses damaged
streams (tests/asan_demux_driver.cpp)."""
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


def _asan_runtime():
    """Path of g++'s AddressSanitizer runtime, or None.  A sanitised shared
    library loaded into Python needs it preloaded."""
    r = subprocess.run(["g++", "-print-file-name=libasan.so"], capture_output=True, text=True)
    path = r.stdout.strip()
    return path if os.path.isabs(path) and os.path.exists(path) else None


@pytest.fixture(scope="module")
def hc_ubsan(tmp_path_factory):
    """(library, LD_PRELOAD value): the host build under UBSan, and under
    AddressSanitizer too where g++ has its runtime."""
    if not shutil.which("g++"):
        pytest.skip("g++ is not installed")
    try:
        corpus.ref_lib()
    except OSError as e:
        pytest.skip(str(e))
    asan = _asan_runtime()
    out = str(tmp_path_factory.mktemp("ubsan") / "libhc_ubsan.so")
    r = subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-w",
                        "-fsanitize=address,undefined" if asan else "-fsanitize=undefined",
                        "-fno-sanitize-recover=all", "-I", CSRC, os.path.join(CSRC, "hostcheck.cpp"), "-o", out,
                        "-lpthread"], capture_output=True, text=True)
    if r.returncode != 0 and "ubsan" in (r.stderr + r.stdout).lower():
        pytest.skip("UBSan runtime unavailable: " + r.stderr[-200:])
    assert r.returncode == 0, r.stderr[-2000:]
    return out, asan


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
    # random packets (any TOC, framing code, padding and payload) after up to
    # three good ones: the decoder's status, counts and samples are libopus's
    rng = np.random.default_rng(79)
    for channels in (1, 2):
        good = ogg_port.demux(corpus.make_stream(dict(kind="mixed", seed=78100, seconds=1.0,
                                                      channels=channels)))["packets"]
        pk, chains = [], []
        for k in range(200):
            n_good = int(rng.integers(0, 4))
            chains.append((len(pk), n_good + 1))
            pk += good[:n_good]
            pk.append(rng.integers(0, 256, int(rng.integers(1, 400)), dtype=np.uint8).tobytes())
        ref = ref_decode.decode_chains(pk, chains, channels)
        got = host_decode(hc, pk, chains, channels)
        for c, (pcm, ns, rg, stop, _) in enumerate(got):
            assert stop == int(ref["status"][c]), (channels, c)
            assert np.array_equal(ns, ref["nsamp"][c]) and np.array_equal(rg, ref["rng"][c]), (channels, c)
            assert np.array_equal(pcm, ref["pcm"][c]), (channels, c)


def test_decoder_has_no_undefined_behaviour(hc_ubsan):
    """Run in a child process, so that a sanitizer report (which aborts) fails
    this test with the report instead of ending the test run."""
    import sys
    lib, asan = hc_ubsan
    env = dict(os.environ, UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1",
               PYTHONPATH=os.pathsep.join([ROOT, os.environ.get("PYTHONPATH", "")]))
    if asan:
        env.update(LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0")
    r = subprocess.run([sys.executable, os.path.abspath(__file__), lib], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]


def test_demuxer_on_damaged_streams_under_address_sanitizer(tmp_path):
    """The host demuxer and chain builder (ogg_demux.cpp) built with
    AddressSanitizer + UndefinedBehaviorSanitizer and run over 1,500 seeded
    damages of the golden streams, each in a heap buffer of exactly its size,
    under the default options, the page-CRC check and the granule
    warn-and-resync policy: no report, the demux with its pages split over
    three threads identical to the one-thread demux in every field, and under
    the default options the same streams accepted as by the oracle's port, with
    the same lengths."""
    import json
    import struct
    import sys
    if not shutil.which("g++"):
        pytest.skip("g++ is not installed")
    exe = str(tmp_path / "asan_demux")
    r = subprocess.run(["g++", "-O1", "-g", "-std=c++17", "-w", "-fsanitize=address,undefined",
                        "-fno-sanitize-recover=all", "-I", CSRC, os.path.join(CSRC, "ogg_demux.cpp"),
                        os.path.join(ROOT, "tests", "asan_demux_driver.cpp"), "-o", exe],
                       capture_output=True, text=True)
    if r.returncode != 0 and "asan" in (r.stderr + r.stdout).lower():
        pytest.skip("ASan runtime unavailable: " + r.stderr[-200:])
    assert r.returncode == 0, r.stderr[-2000:]
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_host_parity import _mutate, _port_index
    gold = os.path.join(ROOT, "tests", "golden")
    names = sorted(json.load(open(os.path.join(gold, "index.json"))))
    streams = {n: open(os.path.join(gold, "streams", n + ".opus"), "rb").read() for n in names}
    rng = np.random.default_rng(71)
    recs = [_mutate(rng, streams[names[i % len(names)]]) for i in range(1500)]
    recs += list(streams.values())
    path = tmp_path / "records"
    path.write_bytes(b"".join(struct.pack("<I", len(d)) + d for d in recs))
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    p = subprocess.run([exe, str(path)], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-4000:]
    lines = p.stdout.splitlines()
    assert len(lines) == 3 * len(recs)
    accepted = 0
    for i, d in enumerate(recs):
        seg, pre = (1.0, 250.0) if i % 2 else (0.5, 80.0)
        want = _port_index(d, seg, pre)
        got = lines[3 * i].split()
        if want is None:
            assert got == ["refused"], i
            continue
        accepted += 1
        ix, chains = want
        assert got == ["ok", str(ix["play48"]), str(ix["channels"]), str(len(ix["packets"])), str(len(chains)),
                       str(sum(c[3] for c in chains))], i
    assert accepted > 200


if __name__ == "__main__":
    import sys
    _decode_all(sys.argv[1])
