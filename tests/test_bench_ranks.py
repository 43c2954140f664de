"""Multi-rank combination of bench.py (CPU, gloo, two ranks).

Ranks running shards of one join add their pair counts and set hashes (a
wrapping 64-bit sum, so disjoint shards' hashes add up to the union's) and the
step time is the maximum over ranks.
"""
import os
import socket

import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, port, out):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    ms = [12.5, 30.0][rank]
    pairs = [1_000_000_007, 5][rank]
    h = [(1 << 64) - 5, 7][rank]          # the sum wraps past 2^64
    out[rank] = bench.combine_ranks(ms, pairs, h, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_combine_ranks_two_gloo_ranks():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:   # no fork of this (threaded) process
        out = m.dict()
        mp.spawn(_rank, args=(port, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        assert res[r] == (30.0, 1_000_000_012, 2)
