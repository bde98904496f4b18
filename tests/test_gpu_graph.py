"""CUDA-graph replay and the batched-instance driver against eager runs.

The kernels of a replayed step read the step number from device memory;
everything else is the eager launch sequence, so the final fields must be
bit-identical and the .dat blocks equal.  The far-field bins are summed with
float atomics in no fixed order, so those series are compared on a common
time axis at the parity tolerance, like the oracle comparison."""
import os

import numpy as np
import pytest

import decks
from datfile import dat_blocks
from test_gpu_parity import TOL, _check_far_field

pytestmark = pytest.mark.gpu

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _run(name, d, mode, g):
    import alpineem_b200 as ab
    _, kmax = decks.write_deck(name, str(d))
    with ab.Simulation(str(d / "inputs.txt"), kmax=kmax, outdir=str(d)) as sim:
        total = sim.steps[1]
        if mode == "graph":
            sim.run_graph(total, g)
        else:
            sim.run(total)
        sim.synchronize()
        fields = [sim.field(c) for c in FIELDS]
        sim.write_outputs()
    return fields, kmax


def _compare(name, da, db, fa, fb, kmax):
    for c, (a, b) in enumerate(zip(fa, fb)):
        assert np.array_equal(a, b), "%s: field %s differs" % (name, FIELDS[c])
    fname = decks.DECKS[name].get("name", "data.dat")
    ba, la = dat_blocks(str(da / fname))
    bb, lb = dat_blocks(str(db / fname))
    assert len(la) == len(lb)
    peak = max(np.linalg.norm(b) for _, b in ba)
    for (ta, a), (tb, b) in zip(ba, bb):
        assert ta == tb and a.shape == b.shape
        if ta.startswith("far field rE") or ta.startswith("far field phase correction"):
            continue
        assert np.array_equal(a, b), "%s: block '%s' differs" % (name, ta)
    if not kmax:
        _check_far_field(name, str(da / fname), str(db / fname), peak)


# (deck, steps per graph): fused path with 32-step far-field batches,
# two-kernel path with far field, plane sums with sheets, complex kmax
@pytest.mark.parametrize("name,g", [("dipole_port", 64), ("tfsf_sphere", 32), ("pbc_sheets", 50), ("kmax_te", 40)])
def test_graph_equals_eager(name, g, tmp_path, gpu_lib):
    da, db = tmp_path / "eager", tmp_path / "graph"
    da.mkdir()
    db.mkdir()
    fa, kmax = _run(name, da, "eager", g)
    fb, _ = _run(name, db, "graph", g)
    _compare(name, da, db, fa, fb, kmax)


def test_batch_equals_single(tmp_path, gpu_lib):
    """Three kmax runs advanced together by aem_run_batch equal three runs on
    their own."""
    import alpineem_b200 as ab
    names = ["kmax_te", "kmax_tm", "kmax_te"]
    single = []
    for q, name in enumerate(names):
        d = tmp_path / ("single%d" % q)
        d.mkdir()
        single.append((d,) + _run(name, d, "eager", 1))
    dirs, sims = [], []
    try:
        for q, name in enumerate(names):
            d = tmp_path / ("batch%d" % q)
            d.mkdir()
            _, kmax = decks.write_deck(name, str(d))
            dirs.append(d)
            sims.append(ab.Simulation(str(d / "inputs.txt"), kmax=kmax, outdir=str(d)))
        total = sims[0].steps[1]
        ab.run_batch(sims, total, 25)
        for q, sim in enumerate(sims):
            sim.synchronize()
            fields = [sim.field(c) for c in FIELDS]
            sim.write_outputs()
            d1, f1, kmax = single[q]
            _compare(names[q], d1, dirs[q], f1, fields, kmax)
    finally:
        for s in sims:
            s.close()
