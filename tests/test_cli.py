"""cuopus_decode, the command-line tool: demux-only mode and the blob / chain
dumps (CPU), then decoding in every mode and the daemon protocol (GPU), all
against the golden tables and the oracle."""
import json
import os
import socket
import struct
import subprocess
import tempfile
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cuopus_b200", "bin", "cuopus_decode")
GOLD = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(GOLD, "index.json")) as _f:
    INDEX = json.load(_f)


def _path(name):
    return os.path.join(GOLD, "streams", name + ".opus")


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        pytest.fail("cuopus_decode must be built (python -m cuopus_b200.build)")
    return CLI


def test_usage(cli):
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.parametrize("name", ["mixed_stereo_b", "plain_a", "code3_120ms"])
def test_demux_dumps_match_reference_tables(cli, name, tmp_path):
    blob, chains = str(tmp_path / "b.blob"), str(tmp_path / "c.bin")
    r = subprocess.run([cli, "--ogg", _path(name), "-", "--seg", "0.5", "--preroll", "80", "--dump-blob", blob,
                        "--dump-chains", chains], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    g = INDEX[name]
    b = open(blob, "rb").read()
    assert b[:4] == b"CUOP"
    n = struct.unpack_from("<I", b, 4)[0]
    assert n == g["n_packets"]
    assert list(struct.unpack_from("<%dI" % n, b, 8)) == g["packet_len"]
    c = open(chains, "rb").read()
    assert c[:4] == b"CUC2"
    k = struct.unpack_from("<I", c, 4)[0]
    tab = np.frombuffer(c[8:], np.uint32).reshape(k, 4).tolist()
    assert tab == g["chains_0.5_80"]


def test_arguments(cli, tmp_path):
    """Options may come before or after the output path; bad values and
    unknown options are usage errors (exit 2)."""
    r = subprocess.run([cli, "--ogg", _path("plain_a"), "--seg", "0.5", "-"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "chains" in r.stdout
    for bad in (["--stride", "x"], ["--seg"], ["--bogus"]):
        r = subprocess.run([cli, "--ogg", _path("plain_a"), "-"] + bad, capture_output=True, text=True)
        assert r.returncode == 2, bad
    r = subprocess.run([cli, "--serve"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_bad_file(cli, tmp_path):
    p = tmp_path / "x.opus"
    p.write_bytes(b"not an ogg file")
    r = subprocess.run([cli, "--ogg", str(p), "-"], capture_output=True, text=True)
    assert r.returncode == 1


def test_daemon_protocol_without_decoding(cli):
    """The daemon's request handling that needs no device: PING, a request for
    a missing file, an unknown command and QUIT, and the refusal of a socket
    path that does not fit sockaddr_un."""
    d = tempfile.mkdtemp()
    r = subprocess.run([cli, "--serve", os.path.join(d, "x" * 200)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "socket path" in r.stderr
    sock = os.path.join(d, "s")
    env = dict(os.environ, CUOPUS_SERVE_IDLE_S="60")
    p = subprocess.Popen([cli, "--serve", sock], env=env, stderr=subprocess.PIPE, text=True)
    try:
        t0 = time.time()
        while not os.path.exists(sock) and time.time() - t0 < 60:
            time.sleep(0.1)
        time.sleep(0.2)
        assert _ask(sock, "PING") == "PONG 2"
        # a client that connects and sends nothing does not hold up the others,
        # and a line sent in pieces is read whole
        idle = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
        idle.connect(sock)
        part = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
        part.settimeout(60)
        part.connect(sock)
        part.sendall(b"PI")
        assert _ask(sock, "PING") == "PONG 2"
        time.sleep(0.1)
        part.sendall(b"NG\n")
        assert part.recv(64) == b"PONG 2\n"
        part.close()
        assert _ask(sock, "DECODE 1 250 32 /nonexistent %s" % os.path.join(d, "o")).startswith("ERR")
        bad = os.path.join(d, "bad.opus")
        with open(bad, "wb") as f:
            f.write(b"not an ogg stream")
        assert _ask(sock, "DECODE 1 250 32 %s %s" % (bad, os.path.join(d, "o"))).startswith("ERR")
        assert _ask(sock, "DECODE16F 1 250").startswith("ERR bad request")
        assert _ask(sock, "DECODE 1 x 32 a b").startswith("ERR bad request")
        assert _ask(sock, "BOGUS").startswith("ERR")
        idle.close()
        assert _ask(sock, "QUIT") == "BYE"
        assert p.wait(timeout=30) == 0
        assert not os.path.exists(sock)
    finally:
        if p.poll() is None:
            p.kill()


# ------------------------------------------------------------------ GPU

def _want_i16(name, seg=1.0, pre=250.0):
    from oracle import pipeline
    pcm, ch, _ = pipeline.i16(open(_path(name), "rb").read(), seg, pre)
    return pcm


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["mixed_stereo_a", "long_hybrid"])
def test_cli_ogg_int16(cuda, cli, name, tmp_path):
    out = str(tmp_path / "o.pcm")
    r = subprocess.run([cli, "--ogg", _path(name), out, "--stride", "16"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.int16)
    assert np.array_equal(got, _want_i16(name))


@pytest.mark.gpu
def test_cli_ogg_f16k(cuda, cli, tmp_path):
    from oracle import pipeline
    out = str(tmp_path / "o.f32")
    r = subprocess.run([cli, "--ogg", _path("plain_b"), out, "--f16k"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, np.float32)
    want = pipeline.f16k(open(_path("plain_b"), "rb").read())
    assert got.shape == want.shape and np.max(np.abs(got - want)) == 0.0


@pytest.mark.gpu
def test_cli_blob_mode(cuda, cli, tmp_path):
    blob, chains, out = str(tmp_path / "b"), str(tmp_path / "c"), str(tmp_path / "o.pcm")
    r = subprocess.run([cli, "--ogg", _path("mixed_mono_b"), "-", "--seg", "0.5", "--preroll", "80",
                        "--dump-blob", blob, "--dump-chains", chains], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([cli, blob, chains, out, "8"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert np.array_equal(np.fromfile(out, np.int16), _want_i16("mixed_mono_b", 0.5, 80.0))


def _ask(sock, line, timeout=120):
    s = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
    s.settimeout(timeout)
    s.connect(sock)
    s.sendall(line.encode() + b"\n")
    data = b""
    while not data.endswith(b"\n"):
        d = s.recv(4096)
        if not d:
            break
        data += d
    s.close()
    return data.decode().strip()


@pytest.mark.gpu
def test_cli_daemon_protocol(cuda, cli):
    from oracle import pipeline
    d = tempfile.mkdtemp()
    sock = os.path.join(d, "s")
    env = dict(os.environ, CUOPUS_SERVE_IDLE_S="60")
    p = subprocess.Popen([cli, "--serve", sock], env=env, stderr=subprocess.PIPE, text=True)
    try:
        t0 = time.time()
        while not os.path.exists(sock) and time.time() - t0 < 60:
            time.sleep(0.1)
        time.sleep(0.2)
        assert _ask(sock, "PING") == "PONG 2"
        out = os.path.join(d, "o.f32")
        rep = _ask(sock, "DECODE16F 1 250 16 %s %s" % (_path("plain_a"), out)).split()
        assert rep[0] == "OK" and len(rep) == 10, rep
        want = pipeline.f16k(open(_path("plain_a"), "rb").read())
        assert int(rep[1]) == want.size and int(rep[2]) == INDEX["plain_a"]["pcm_samples_48k"]
        assert np.array_equal(np.fromfile(out, np.float32), want)
        out2 = os.path.join(d, "o.pcm")
        rep = _ask(sock, "DECODE 1 250 32 %s %s" % (_path("mixed_stereo_b"), out2)).split()
        assert rep[0] == "OK", rep
        assert np.array_equal(np.fromfile(out2, np.int16), _want_i16("mixed_stereo_b"))
        assert _ask(sock, "DECODE 1 250 32 /nonexistent %s" % out2).startswith("ERR")
        assert _ask(sock, "BOGUS").startswith("ERR")
        assert _ask(sock, "QUIT") == "BYE"
        assert p.wait(timeout=30) == 0
    finally:
        if p.poll() is None:
            p.kill()
