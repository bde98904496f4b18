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


def test_truncated_checkpoint_leaves_the_handle_unchanged(tmp_path, gpu_lib):
    """A truncated file is rejected before any buffer is overwritten: the
    handle keeps its own state and step count and runs on as if the load
    had not been tried."""
    import alpineem_b200 as ab
    a, b, c = tmp_path / "a", tmp_path / "b", tmp_path / "c"
    for p in (a, b, c):
        p.mkdir()
    ck = tmp_path / "state.ckpt"
    sim, _ = _sim("dipole_port", a)
    with sim:
        sim.run(20)
        sim.checkpoint_save(str(ck))
    data = ck.read_bytes()
    short = tmp_path / "short.ckpt"
    short.write_bytes(data[:len(data) - 100])
    sim, _ = _sim("dipole_port", b)
    with sim:
        sim.run(7)
        with pytest.raises(ab.AemError, match="truncated"):
            sim.checkpoint_load(str(short))
        assert sim.steps[0] == 7
        sim.run(13)
        got = [sim.field(f) for f in FIELDS]
    sim, _ = _sim("dipole_port", c)
    with sim:
        sim.run(20)
        want = [sim.field(f) for f in FIELDS]
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_checkpoint_does_not_depend_on_the_watchdog(tmp_path, gpu_lib):
    """The watchdog's flag is scratch, not run state: a checkpoint written
    with `watchdog K` on loads into a handle of the same deck without it,
    and the reverse, and both continue to the same fields."""
    import alpineem_b200 as ab
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    decks.write_deck("dipole_port", str(a))
    decks.write_deck("dipole_port", str(b))
    (a / "inputs.txt.b200").write_text("watchdog 10\n")
    ck_w, ck_n = str(tmp_path / "w.ckpt"), str(tmp_path / "n.ckpt")
    with ab.Simulation(str(a / "inputs.txt"), outdir=str(a)) as sw, ab.Simulation(str(b / "inputs.txt"), outdir=str(b)) as sn:
        sw.run(11)
        sn.run(11)
        sw.checkpoint_save(ck_w)
        sn.checkpoint_save(ck_n)
        sw.checkpoint_load(ck_n)
        sn.checkpoint_load(ck_w)
        sw.run(20)
        sn.run(20)
        for f in FIELDS:
            assert np.array_equal(sw.field(f), sn.field(f))
