"""Sharding of independent runs across ranks and the end-of-run gather, on
two gloo ranks (CPU): the multi-GPU path of a sweep without a GPU."""
import os
import socket

import pytest

from alpineem_b200.parallel import gather_results, max_over_ranks, shard, unshard


def test_shard_unshard():
    items = list(range(10))
    for world in (1, 2, 3, 4):
        parts = [shard(items, r, world) for r in range(world)]
        assert sorted(v for p in parts for v in p) == items
        assert unshard(parts, world) == items
    with pytest.raises(ValueError):
        shard(items, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        items = list(range(7))
        mine = shard(items, rank, world)
        parts = gather_results([x * x for x in mine])
        full = unshard(parts, world)
        job = max_over_ranks(0.25 + rank)
        with open(os.path.join(out_dir, "r%d.txt" % rank), "w") as f:
            f.write("%s %s %s\n" % (mine, full, job))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        line = (tmp_path / ("r%d.txt" % r)).read_text()
        assert ("[%s]" % ", ".join(str(x) for x in range(7)[r::world])) in line
        assert "[0, 1, 4, 9, 16, 25, 36]" in line
        assert line.strip().endswith("1.25")
