"""Streams that exercise the frame-level branches of opus_decode_frame
(src/opus_decoder.c:237-668), shared by the CPU and GPU tests.

The encoder covers a switch from CELT to SILK or hybrid with a redundancy
frame, so an encoded stream never reaches the decoder's CELT -> SILK
transition without one (the 5 ms concealment crossfade of :347 / :458-476).
Splicing the packets of separate encodes -- a CELT encode followed by a SILK,
hybrid or CELT encode of another signal, and so on -- gives every mode change
without redundancy; any packet sequence is valid decoder input, and libopus
decodes the same sequence for the comparison.
"""
import numpy as np

from oracle import corpus

_MODES = {
    "silk": (corpus.MODE_SILK, corpus.BW_WB, 960, 24000),
    "hybrid": (corpus.MODE_HYBRID, corpus.BW_SWB, 960, 40000),
    "celt": (corpus.MODE_CELT, corpus.BW_FB, 960, 64000),
    "celt10": (corpus.MODE_CELT, corpus.BW_FB, 480, 48000),
}


def _encode(mode, channels, seed, seconds=0.6):
    rng = np.random.default_rng(seed)
    n = int(seconds * corpus.SR)
    x = corpus.synth("speech" if mode in ("silk", "hybrid") else "chord", n, rng)
    if channels == 2:
        x = np.stack([x, 0.7 * x + 0.3 * corpus.synth("pink", n, rng)], axis=1).reshape(-1)
    m, bw, fs, br = _MODES[mode]
    pk, _ = corpus.encode(corpus.to_i16(x), channels, [corpus.Seg(0, m, bw, fs, br)])
    return pk


# (first encode, second encode): CELT -> SILK / hybrid without redundancy,
# SILK / hybrid -> CELT without redundancy, hybrid -> SILK (the CELT layer's
# silence frame), and CELT 20 ms -> CELT 10 ms (no transition).
SPLICES = [("celt", "silk"), ("celt", "hybrid"), ("silk", "celt"), ("hybrid", "celt"), ("hybrid", "silk"),
           ("celt", "celt10"), ("silk", "hybrid")]


def spliced_chains(channels, seed=0):
    """One packet list holding every splice, and its chains: each chain is one
    splice, decoded from a fresh decoder (10 packets of the first encode, then
    10 of the second, taken from the middle of each)."""
    packets, chains = [], []
    for k, (a, b) in enumerate(SPLICES):
        pa = _encode(a, channels, 9100 + 10 * k + seed)
        pb = _encode(b, channels, 9105 + 10 * k + seed)
        chains.append((len(packets), 20))
        packets += pa[5:15] + pb[10:20]
    return packets, chains
