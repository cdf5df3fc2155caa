"""The N > 1 path on CPU: two gloo ranks split the work of one triangle
COUNT round-robin, each counts its share (with the oracle standing in for
the device kernel, which needs a GPU), and one all-reduce combines them.
Also checks the modulo-2^64 combine and the max-over-ranks timing."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, result_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist

    from emptyheaded_b200 import shard
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        u, v = O.gen_rmat(3, 12, 16 << 12)
        s, d, _ = O.preprocess(u, v)
        t = O.Trie(s, d)
        per = t.triangle_per_vertex()
        # heaviest-first work order, round-robin ownership
        order = np.argsort(-per.astype(np.int64), kind="stable")
        mine = sum(int(per[order[i]]) for i in shard.owned(len(order), rank, world))
        total = shard.combine_counts(mine)
        wrap = shard.combine_counts((1 << 63) + rank)  # sums past 2^64 wrap
        tmax = shard.max_over_ranks(1.5 + rank)
        with open(os.path.join(result_dir, "r%d.txt" % rank), "w") as f:
            f.write("%d %d %.3f %d" % (total, wrap, tmax, t.triangle()))
    finally:
        dist.destroy_process_group()


def test_two_rank_count_combine(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    rows = [open(os.path.join(tmp_path, "r%d.txt" % r)).read().split() for r in range(world)]
    for total, wrap, tmax, want in rows:
        assert int(total) == int(want) == 485514
        assert int(wrap) == ((1 << 64) + 1) & ((1 << 64) - 1)
        assert float(tmax) == 2.5


def test_owned_partition_covers_every_item():
    from emptyheaded_b200 import shard
    for n in (0, 1, 7, 100):
        for w in (1, 2, 3, 8):
            got = sorted(i for r in range(w) for i in shard.owned(n, r, w))
            assert got == list(range(n))
