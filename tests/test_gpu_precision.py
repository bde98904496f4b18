"""The error of every FP32 output against the FP64 build of the oracle.

The solver computes in FP32, as the reference does; the oracle's FP64 build
(fdtd_oracle_f64 / fdtd_oracle_kmax_f64) runs the same statements in double
precision.  For every parity deck, each numeric block of the FP32 GPU run's
<name>.dat is compared with the FP64 run's:
  * probe time series (incident wave, plane sums, port voltages, phase-centre
    incident): relative L2 <= 1e-4;
  * far-field series, on the common time axis (start bins may differ, see
    test_gpu_parity._check_far_field): relative L2 <= 1e-3.
A near-zero block is judged against the largest block of the run (floor
1e-3 of its norm), as in the parity test.  With AEM_PRECISION_REPORT set to
a file name, each deck's largest errors are appended to it as one JSON line.
"""
import json
import os

import numpy as np
import pytest

import decks
from datfile import dat_blocks, rel_l2
from test_gpu_parity import _run_oracle

pytestmark = pytest.mark.gpu

TOL_PROBE, TOL_FF = 1e-4, 1e-3


def _far_field_err(odat, gdat, peak):
    import postproc
    o, g = postproc.parse_dat(odat), postproc.parse_dat(gdat)
    dt, worst = o["time_step"], 0.0
    for q in range(2 * o["num_angles"]):
        a = q // 2
        s = int(round((o["time_corr"][a] - g["time_corr"][a]) / dt))
        so, sg = o["ff"][q], g["ff"][q]
        T = len(so)
        n0, n1 = max(0, -s), min(T, T - s)
        worst = max(worst, rel_l2(so[n0 + s:n1 + s], sg[n0:n1], floor=1e-3 * peak))
    return worst


@pytest.mark.parametrize("name", sorted(decks.DECKS))
def test_fp32_error_against_fp64(name, tmp_path, oracle_bin, gpu_lib):
    import alpineem_b200 as ab
    od, gd = tmp_path / "f64", tmp_path / "gpu"
    od.mkdir()
    gd.mkdir()
    _, kmax = decks.write_deck(name, str(od))
    decks.write_deck(name, str(gd))
    _run_oracle(oracle_bin["fdtd_oracle_kmax_f64" if kmax else "fdtd_oracle_f64"], str(od))
    with ab.Simulation(str(gd / "inputs.txt"), kmax=kmax, outdir=str(gd)) as sim:
        sim.run_all()
    fname = decks.DECKS[name].get("name", "data.dat")
    ob, _ = dat_blocks(str(od / fname))
    gb, _ = dat_blocks(str(gd / fname))
    assert len(ob) == len(gb)
    peak = max(np.linalg.norm(b) for _, b in ob)
    probe = 0.0
    for (ta, a), (tb, b) in zip(ob, gb):
        assert ta == tb and a.shape == b.shape
        if ta.startswith("far field rE") or ta.startswith("far field phase correction"):
            continue
        probe = max(probe, rel_l2(a, b, floor=1e-3 * peak))
    ff = 0.0 if kmax or not decks.DECKS[name].get("ff") else _far_field_err(str(od / fname), str(gd / fname), peak)
    rep = os.environ.get("AEM_PRECISION_REPORT")
    if rep:
        with open(rep, "a") as f:
            f.write(json.dumps({"deck": name, "probe_rel_l2": probe, "far_field_rel_l2": ff}) + "\n")
    assert probe <= TOL_PROBE, (name, probe)
    assert ff <= TOL_FF, (name, ff)


@pytest.mark.parametrize("name", ["tfsf_sphere", "drude_pbc", "kmax_te", "ellipsoids_small"])
def test_fp64_coefficient_tables(name, tmp_path, oracle_bin, gpu_lib):
    """Extension `coef_precision 64`: the material (Ga, Gb, Drude Ja, Jb) and
    CPML (b, c, kappa, den) tables are evaluated on the GPU in FP64 and
    rounded once.  The run then differs from the reference-arithmetic run
    (the tables changed) and its probe series stay within 1e-4 of the FP64
    oracle."""
    import alpineem_b200 as ab
    od, gd, rd = tmp_path / "f64", tmp_path / "gpu64", tmp_path / "gpu32"
    for p in (od, gd, rd):
        p.mkdir()
    _, kmax = decks.write_deck(name, str(od))
    decks.write_deck(name, str(gd))
    decks.write_deck(name, str(rd))
    ext = gd / "inputs.txt.b200"
    ext.write_text((ext.read_text() if ext.exists() else "") + "coef_precision 64\n")
    _run_oracle(oracle_bin["fdtd_oracle_kmax_f64" if kmax else "fdtd_oracle_f64"], str(od))
    for d in (gd, rd):
        with ab.Simulation(str(d / "inputs.txt"), kmax=kmax, outdir=str(d)) as sim:
            sim.run_all()
    fname = decks.DECKS[name].get("name", "data.dat")
    ob, _ = dat_blocks(str(od / fname))
    gb, _ = dat_blocks(str(gd / fname))
    rb, _ = dat_blocks(str(rd / fname))
    peak = max(np.linalg.norm(b) for _, b in ob)
    probe, changed = 0.0, False
    for (ta, a), (_, b), (_, c) in zip(ob, gb, rb):
        changed = changed or not np.array_equal(b, c)
        if ta.startswith("far field rE") or ta.startswith("far field phase correction"):
            continue
        probe = max(probe, rel_l2(a, b, floor=1e-3 * peak))
    rep = os.environ.get("AEM_PRECISION_REPORT")
    if rep:
        with open(rep, "a") as f:
            f.write(json.dumps({"deck": name + "_coef64", "probe_rel_l2": probe}) + "\n")
    assert changed, name
    assert probe <= TOL_PROBE, (name, probe)
