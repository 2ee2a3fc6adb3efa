"""Slab sharding across ranks (replicas, no data-path collective) on CPU.

The partition is pmilos' (pmilos.c:1181-1205); two gloo ranks each invert their
slab with the oracle restatement (the checker stands in for the GPU here) and
the results-only gather must reproduce the one-process inversion bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pmilos_b200.shard import slab


def test_slab_partition_matches_pmilos():
    for npix, world in [(10, 3), (4096, 8), (7, 7), (5, 8), (65536, 1)]:
        spans = [slab(npix, r, world) for r in range(world)]
        counts = [c for _, c in spans]
        assert sum(counts) == npix
        assert counts == sorted(counts, reverse=True) and max(counts) - min(counts) <= 1
        assert all(spans[r + 1][0] == spans[r][0] + spans[r][1] for r in range(world - 1))
    with pytest.raises(ValueError):
        slab(10, 3, 3)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_path):
    import datetime

    import torch.distributed as dist

    import pyoracle as po
    from gpu_common import case, oracle
    from pmilos_b200.shard import gather

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        c = case(1)
        s, n = slab(c["obs"].shape[0], rank, world)
        r = oracle(c).invert(c["obs"][s:s + n], c["guess"], fix=c["fix"], noise=(1.0 / 1000) ** 2)
        full = gather(r, c["obs"].shape[0])
        if rank == 0:
            np.savez(out_path, **full)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_one_process_result(tmp_path):
    from gpu_common import case, oracle

    out = str(tmp_path / "gathered.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    c = case(1)
    ref = oracle(c).invert(c["obs"], c["guess"], fix=c["fix"], noise=(1.0 / 1000) ** 2)
    assert np.array_equal(got["models"], ref["models"])
    assert np.array_equal(got["chisq"], ref["chisq"])
    assert np.array_equal(got["iters"], ref["iters"])
