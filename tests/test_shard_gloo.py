"""The multi-GPU path on CPU: two gloo ranks split a job into contiguous frame
ranges, generate their own frames from offset counters, decode them (the
oracle stands in for the GPU decoder here), and reduce only counters; the
totals equal a single process decoding the whole job."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from wimax_ldpc_lib_b200.shard import shard_range

RATE, Z, FRAMES, EBNO = 0, 24, 203, 1.75


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _job(oracle, first, count):
    info, cw, llr, _ = oracle.framegen(RATE, Z, 99, first, count, EBNO)
    _, dec, _, it, sf = oracle.decode(RATE, Z, llr.astype(np.float32), 10)
    fe = (dec[:, :info.shape[1]] != info).any(axis=1)
    return [float(fe.sum()), float(it.sum()), float(sf.sum()), float(count)]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from oracle.oracle import Oracle
    from wimax_ldpc_lib_b200.shard import max_over_ranks, reduce_counters
    first, count = shard_range(FRAMES, rank, world)
    totals = reduce_counters(_job(Oracle(), first, count))
    slowest = max_over_ranks(float(rank + 1))
    if rank == 0:
        out.put((totals, slowest))
    dist.destroy_process_group()


def test_shard_ranges_cover_the_job():
    for total in (0, 1, 7, 262144, 262145):
        for world in (1, 2, 3, 8):
            spans = [shard_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and sum(c for _, c in spans) == total
            for (f0, c0), (f1, _) in zip(spans, spans[1:]):
                assert f0 + c0 == f1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_two_gloo_ranks_match_one_process(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    totals, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert totals == _job(oracle, 0, FRAMES)
    assert slowest == 2.0
