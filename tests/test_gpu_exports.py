"""Field exports against the oracle: the per-step full-field files
(<name>_full_*.bin, fdtd_solver.f90:6960-7003) and the 2-D video slices
(<name>_video_*.bin, fdtd_solver.f90:6833-6958 and :8788-8807).

Both are Fortran unformatted sequential files: every record is a 4-byte
length, the FP32 values (re, im pairs for the constant-k solver) and the
length again.  The record structure must match exactly; the values at the
parity tolerance of the field comparison (relative L2 <= 1e-4 per
component over all steps, a near-zero component judged against the largest
E or H component)."""
import numpy as np
import pytest

import decks
from datfile import rel_l2
from test_gpu_parity import TOL, _run_oracle

pytestmark = pytest.mark.gpu

FULL = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
VIDEO = ("Ex", "Hx", "Ey", "Hy", "Ez", "Hz")


def read_records(path, kmax):
    """The records of a Fortran unformatted sequential file as FP32 (or
    complex64) arrays; asserts the leading and trailing lengths agree."""
    raw = open(path, "rb").read()
    out, p = [], 0
    while p < len(raw):
        n = int(np.frombuffer(raw, np.int32, 1, p)[0])
        body = np.frombuffer(raw, np.float32, n // 4, p + 4)
        assert int(np.frombuffer(raw, np.int32, 1, p + 4 + n)[0]) == n, (path, p)
        out.append(body.view(np.complex64) if kmax else body)
        p += n + 8
    return out


def _compare(od, gd, base, names, kmax, expect_records, expect_len):
    recs = {}
    for c in names:
        o = read_records(str(od / ("%s_%s.bin" % (base, c))), kmax)
        g = read_records(str(gd / ("%s_%s.bin" % (base, c))), kmax)
        assert len(o) == len(g) == expect_records, (c, len(o), len(g))
        assert all(r.size == expect_len for r in o + g), c
        recs[c] = (np.concatenate(o), np.concatenate(g))
    epeak = max(np.linalg.norm(recs[c][0]) for c in names if c[0] == "E")
    hpeak = max(np.linalg.norm(recs[c][0]) for c in names if c[0] == "H")
    for c in names:
        o, g = recs[c]
        err = rel_l2(o, g, floor=1e-2 * (epeak if c[0] == "E" else hpeak))
        assert err <= TOL, "%s_%s: rel L2 %.3g" % (base, c, err)


def _decks(name, tmp_path):
    od, gd = tmp_path / "oracle", tmp_path / "gpu"
    od.mkdir()
    gd.mkdir()
    _, kmax = decks.write_deck(name, str(od))
    decks.write_deck(name, str(gd))
    return od, gd, kmax


@pytest.mark.parametrize("name,mode", [("full_dipole", "run"), ("full_dipole", "graph"), ("full_kmax", "run")])
def test_full_field_export(name, mode, tmp_path, oracle_bin, gpu_lib):
    """Every step's averaged fields; the graph driver falls back to eager
    steps (the host writes each step) and must give the same files."""
    import alpineem_b200 as ab
    od, gd, kmax = _decks(name, tmp_path)
    _run_oracle(oracle_bin["fdtd_oracle_kmax" if kmax else "fdtd_oracle"], str(od))
    with ab.Simulation(str(gd / "inputs.txt"), kmax=kmax, outdir=str(gd)) as sim:
        total = sim.steps[1]
        if mode == "graph":
            sim.run_graph(total, 16)
        else:
            sim.run(total // 3)   # a partial run, then the rest
            sim.run_all()
    # X - 1 - pbc_x = nx cells along x (likewise y, z) in every record
    d = decks.DECKS[name]
    cells = int(np.prod(d["n"]))
    fname = d.get("name", "data.dat")
    _compare(od, gd, fname[:-4] + "_full", FULL, kmax, d["steps"], cells)


def test_video_slices(tmp_path, oracle_bin, gpu_lib):
    """The y-normal video slice of every step, written at the end of the run."""
    import alpineem_b200 as ab
    od, gd, kmax = _decks("video", tmp_path)
    _run_oracle(oracle_bin["fdtd_oracle"], str(od))
    with ab.Simulation(str(gd / "inputs.txt"), kmax=kmax, outdir=str(gd)) as sim:
        sim.run_all()
    d = decks.DECKS["video"]
    nx, _, nz = d["n"]
    _compare(od, gd, "data_video", VIDEO, kmax, 1, nx * nz * d["steps"])
