"""Failure detection, with every failure made on the host (no test faults,
traps or hangs a GPU):

* the watchdog (extension `watchdog K`) stops a run with AEM_ERR_DIVERGED
  (AemDiverged) at the first K-th step whose E or H holds a NaN or Inf:
  a NaN planted in a checkpoint file on the host, resumed eagerly and by
  graph replay; a time step 4x over the Courant limit (deck factor 0.25),
  whose fields overflow to Inf within tens of steps;
* the watchdog leaves a normal run bit-identical;
* an allocation failure injected on the host (AEM_FAIL_ALLOC_AT=n) makes the
  handle's creation fail with AEM_ERR_CUDA, after which handles are created
  and run normally;
* a truncated bulk geometry file and a missing one are rejected with the
  reference-style input error."""
import os
import struct

import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu


def _sim(name, tmp_path, ext=None, **change):
    import alpineem_b200 as ab
    d = dict(decks.DECKS[name], **change)
    return ab.Simulation(deck_text=decks.deck_text(d), ext_text=ext, kmax=bool(d.get("kmax")), outdir=str(tmp_path))


def _plant_nan(path):
    """Overwrite one value of the first stored buffer (Ex of the two-kernel
    path) in the middle of a checkpoint file with a quiet NaN."""
    with open(path, "r+b") as f:
        head = f.read(8 + 48)
        nbuf = struct.unpack("<6q", head[8:])[5]
        sizes = struct.unpack("<%dq" % nbuf, f.read(8 * nbuf))
        f.seek(8 + 48 + 8 * nbuf + (sizes[0] // 2 // 4) * 4)
        f.write(struct.pack("<I", 0x7FC00000))


@pytest.mark.parametrize("mode", ["eager", "graph"])
def test_watchdog_stops_on_a_planted_nan(mode, tmp_path, gpu_lib):
    import alpineem_b200 as ab
    ck = str(tmp_path / "state.ckpt")
    with _sim("kmax_te", tmp_path, "watchdog 10\n") as sim:
        sim.run(20)
        sim.checkpoint_save(ck)
    _plant_nan(ck)
    with _sim("kmax_te", tmp_path, "watchdog 10\n") as sim:
        sim.checkpoint_load(ck)
        with pytest.raises(ab.AemDiverged, match="non-finite value at step 30"):
            if mode == "graph":
                sim.run_graph(40, 10)
            else:
                sim.run(40)
        assert sim.steps[0] == 30


def test_unstable_time_step_diverges(tmp_path, gpu_lib):
    import alpineem_b200 as ab
    with _sim("dipole_port", tmp_path, "watchdog 5\n", factor=0.25) as sim:
        with pytest.raises(ab.AemDiverged, match="diverged"):
            sim.run(sim.steps[1])
        assert 5 <= sim.steps[0] < sim.steps[1] and sim.steps[0] % 5 == 0


def test_watchdog_leaves_a_normal_run_unchanged(tmp_path, gpu_lib):
    out = []
    for ext in (None, "watchdog 7\n"):
        d = tmp_path / ("w" if ext else "plain")
        d.mkdir()
        with _sim("dipole_port", d, ext) as sim:
            sim.run(sim.steps[1])
            out.append([sim.field(c) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_injected_allocation_failure(tmp_path, monkeypatch, gpu_lib):
    import alpineem_b200 as ab
    for n in (1, 3, 9):
        monkeypatch.setenv("AEM_FAIL_ALLOC_AT", str(n))
        with pytest.raises(ab.AemError, match="injected by AEM_FAIL_ALLOC_AT"):
            _sim("kmax_te", tmp_path)
    monkeypatch.delenv("AEM_FAIL_ALLOC_AT")
    with _sim("kmax_te", tmp_path) as sim:
        sim.run(5)
        assert sim.steps[0] == 5


def test_bulk_file_errors(tmp_path, gpu_lib):
    import alpineem_b200 as ab
    path, kmax = decks.write_deck("ellipsoids_small", str(tmp_path))
    bulk = os.path.join(str(tmp_path), decks.DECKS["ellipsoids_small"]["bulk"])
    data = open(bulk, "rb").read()
    with open(bulk, "wb") as f:
        f.write(data[: len(data) // 2])
    with pytest.raises(ab.AemError, match="too short"):
        ab.Simulation(path, kmax=kmax, outdir=str(tmp_path))
    os.remove(bulk)
    with pytest.raises(ab.AemError, match="cannot open bulk geometry file"):
        ab.Simulation(path, kmax=kmax, outdir=str(tmp_path))
