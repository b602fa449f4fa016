"""The multi-GPU path of bench.py, run on the CPU: two gloo ranks take
disjoint sets of full blocks (weak scaling, no data exchange), agree on the
slowest rank's time and on the parity of every rank's lines, as
`bench.py --gpus N` does over NCCL."""
import socket
from datetime import timedelta

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        blocks = bench.rank_blocks(16, rank)
        slowest = bench.max_over_ranks(10.0 * (rank + 1), world, torch.device("cpu"))
        gathered = [None] * world
        dist.all_gather_object(gathered, blocks)
        # parity: both ranks match, then rank 1 alone reports a mismatch
        both = bench.combine_parity({"ok": True, "lines_checked": 4}, world, torch.device("cpu"))
        one_bad = bench.combine_parity({"ok": rank != 1, "lines_checked": 4}, world, torch.device("cpu"))
        q.put((rank, slowest, gathered, both["ok"], one_bad["ok"]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_blocks_and_take_the_slowest_time():
    import multiprocessing as mp
    import bench
    from pentago_b200.end import section_shape, section_sig
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shape = section_shape(section_sig(bench.SECTION))
    for rank, slowest, gathered, both_ok, one_bad_ok in results:
        assert slowest == 20.0
        assert both_ok and not one_bad_ok
        a, b = (set(map(tuple, g)) for g in gathered)
        assert len(a) == len(b) == 16 and not (a & b)
        for blk in a | b:
            assert all(0 <= c and 8 * (c + 1) <= s for c, s in zip(blk, shape)), blk


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1, None) == 3.5
    assert bench.rank_blocks(4, 0) == [bench.block_of(i) for i in range(4)]
