"""Checkpoint / resume (aem_checkpoint_save / aem_checkpoint_load).

A run stopped after k steps, saved to a file, and continued in a new handle
made from the same deck must end where the uninterrupted run ends: final
fields bit-identical and the .dat blocks equal (far-field series on a common
time axis at the parity tolerance, since their bins are summed with float
atomics in no fixed order).  k is odd and falls inside a 32-step far-field
batch, so the fused path's buffer swap parity and a partly filled batch
buffer are carried across.  Cases: the fused path (port antenna with far
field), the two-kernel TF/SF path with far field, and a constant-k unit cell
continued by CUDA-graph replay.  A file from another deck, or not a
checkpoint at all, is rejected."""
import numpy as np
import pytest

import decks
from test_gpu_graph import FIELDS, _compare

pytestmark = pytest.mark.gpu


def _sim(name, d):
    import alpineem_b200 as ab
    _, kmax = decks.write_deck(name, str(d))
    return ab.Simulation(str(d / "inputs.txt"), kmax=kmax, outdir=str(d)), kmax


def _finish(sim, mode):
    left = sim.steps[1] - sim.steps[0]
    if mode == "graph":
        sim.run_graph(left, 32)
    else:
        sim.run(left)
    sim.synchronize()
    fields = [sim.field(c) for c in FIELDS]
    sim.write_outputs()
    return fields


@pytest.mark.parametrize("name,k,mode", [("dipole_port", 37, "eager"), ("tfsf_sphere", 45, "eager"),
                                         ("kmax_te", 51, "graph")])
def test_resume_equals_uninterrupted(name, k, mode, tmp_path, gpu_lib):
    da, db = tmp_path / "whole", tmp_path / "resumed"
    da.mkdir()
    db.mkdir()
    sim, kmax = _sim(name, da)
    with sim:
        fa = _finish(sim, "eager")
    ck = str(tmp_path / "state.ckpt")
    sim, _ = _sim(name, db)
    with sim:
        sim.run(k)
        sim.checkpoint_save(ck)
        sim.run(5)  # steps after the save are discarded by the load below
        sim.checkpoint_load(ck)
        assert sim.steps[0] == k
    sim, _ = _sim(name, db)
    with sim:
        sim.checkpoint_load(ck)
        assert sim.steps[0] == k
        fb = _finish(sim, mode)
    _compare(name, da, db, fa, fb, kmax)


def test_checkpoint_rejects_other_files(tmp_path, gpu_lib):
    import alpineem_b200 as ab
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    ck = str(tmp_path / "a.ckpt")
    sim, _ = _sim("kmax_te", a)
    with sim:
        sim.run(3)
        sim.checkpoint_save(ck)
    junk = tmp_path / "junk.ckpt"
    junk.write_bytes(b"not a checkpoint at all")
    sim, _ = _sim("dipole_port", b)
    with sim:
        with pytest.raises(ab.AemError, match="not written by a run of this deck"):
            sim.checkpoint_load(ck)
        with pytest.raises(ab.AemError, match="not a checkpoint file"):
            sim.checkpoint_load(str(junk))
        with pytest.raises(ab.AemError, match="cannot open checkpoint"):
            sim.checkpoint_load(str(tmp_path / "missing.ckpt"))
        sim.run(2)
        assert sim.steps[0] == 2
