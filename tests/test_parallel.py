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


SWEEP = ["smoke", "pbc_sheets", "drude_pbc", "kmax_te", "kmax_tm"]


def _run_deck(name, directory):
    """One run of the sweep on a CPU rank: the deck checked through the C
    ABI (grid sizes) and run by the FP32 oracle; returns (sizes, the sum of
    the absolute values of every number in the .dat file)."""
    import subprocess
    import numpy as np
    import alpineem_b200 as ab
    import decks
    from datfile import dat_blocks
    from conftest import ORACLE_BUILD
    d = os.path.join(directory, name)
    os.makedirs(d, exist_ok=True)
    path, kmax = decks.write_deck(name, d)
    sizes = ab.check_deck(open(path).read(), kmax=kmax)
    binary = os.path.join(ORACLE_BUILD, "fdtd_oracle_kmax" if kmax else "fdtd_oracle")
    r = subprocess.run([binary, "inputs.txt"], cwd=d, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stdout[-1000:] + r.stderr[-1000:]
    blocks, _ = dat_blocks(os.path.join(d, decks.DECKS[name].get("name", "data.dat")))
    return list(sizes), float(sum(np.abs(b).sum() for _, b in blocks))


def _sweep_rank(rank, world, port, out_dir):
    import datetime
    import json
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300))
    try:
        mine = shard(SWEEP, rank, world)
        res = [_run_deck(n, os.path.join(out_dir, "rank%d" % rank)) for n in mine]
        full = unshard(gather_results(res), world)
        with open(os.path.join(out_dir, "sweep%d.json" % rank), "w") as f:
            json.dump({"mine": mine, "full": full}, f)
    finally:
        dist.destroy_process_group()


def test_sharded_sweep_equals_single_rank(tmp_path, oracle_bin):
    """A sweep of independent runs (five small decks: unit cells with sheets
    and Drude poles, constant-k TE/TM cells, a scattering case) sharded over
    two gloo ranks, run, gathered and put back in item order equals the same
    sweep run on one rank, result for result."""
    import json
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    mp.start_processes(_sweep_rank, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    single = [_run_deck(n, str(tmp_path / "single")) for n in SWEEP]
    for r in range(world):
        got = json.loads((tmp_path / ("sweep%d.json" % r)).read_text())
        assert got["mine"] == SWEEP[r::world]
        assert [tuple(s) for s, _ in got["full"]] == [tuple(s) for s, _ in single]
        assert [v for _, v in got["full"]] == [v for _, v in single]
