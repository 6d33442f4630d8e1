"""The N > 1 path on CPU: world-size-2 gloo ranks run the bench's rank logic
(every rank decodes its own batch of the same shape, no data exchange; the
step time is the max over ranks and rank 0 reports) with the oracle decoder
standing in for the GPU, and the chain tables every rank builds are the
same."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import sys
    import time

    import numpy as np
    import torch
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import ogg_port, ref_decode
        gold = os.path.join(ROOT, "tests", "golden", "streams")
        names = sorted(os.listdir(gold))
        d = open(os.path.join(gold, names[0]), "rb").read()
        ix = ogg_port.demux(d)
        chains = ogg_port.build_chains(ix, 1.0, 250.0)
        t0 = time.perf_counter()
        r = ref_decode.decode_chains(ix["packets"], chains, ix["channels"], nthreads=1)
        step = time.perf_counter() - t0
        t = torch.tensor([step], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tab = torch.tensor(np.array(chains, np.int64).reshape(-1))
        gathered = [torch.zeros_like(tab) for _ in range(world)]
        dist.all_gather(gathered, tab)
        same = all(torch.equal(g, tab) for g in gathered)
        digest = int(np.frombuffer(np.concatenate(r["pcm"]).tobytes(), np.uint8).sum())
        dg = torch.tensor([digest], dtype=torch.int64)
        dl = [torch.zeros_like(dg) for _ in range(world)]
        dist.all_gather(dl, dg)
        dist.barrier()
        if rank == 0:
            audio = ix["play48"] / 48000.0
            q.put(dict(max_step=float(t.item()), own=step, same_tables=same,
                       same_pcm=len(set(int(x) for x in dl)) == 1, value=world * audio / float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_weak_scaling():
    try:
        from oracle.corpus import ref_lib
        ref_lib()
    except OSError as e:
        pytest.skip(str(e))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out["same_tables"] and out["same_pcm"]
    assert out["max_step"] >= out["own"] > 0
    assert out["value"] > 0
