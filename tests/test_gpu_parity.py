"""GPU parity: the CUDA solver against the CPU oracle on the same decks.

For every deck in tests/decks.py both the FP32 oracle (a statement-by-
statement C restatement of main_fdtd/fdtd_solver.f90) and the sm_100a
solver run the full step count.  Compared:
  * every numeric block of <name>.dat (incident wave, reflected/transmitted
    plane sums, far-field E_theta/E_phi, port voltages, phase-centre
    incident, time corrections): relative L2 <= 1e-4, the tolerance the task
    sets for probe time series (FP32 both sides; the two differ only in
    rounding: GPU expf in the incident-wave function and reduction order);
  * all six final field arrays in the reference layout: relative L2 <= 1e-4;
  * the header lines token by token and <name>_geometry.bin byte for byte
    (where the deck does not switch it off).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import decks
from datfile import dat_blocks, header_values, read_oracle_dump, rel_l2

TOL = 1e-4
pytestmark = pytest.mark.gpu


def _run_oracle(binary, d, max_steps=None, dump_fields=True, dump_series=False):
    """Run the oracle on d/inputs.txt; optionally dump the final fields
    (ORACLE_DUMP) and the raw plane-sum series (ORACLE_SERIES_DIR)."""
    env = dict(os.environ)
    if dump_fields:
        env["ORACLE_DUMP"] = os.path.join(d, "fields.bin")
    if dump_series:
        env["ORACLE_SERIES_DIR"] = d
    if max_steps:
        env["ORACLE_MAX_STEPS"] = str(max_steps)
    r = subprocess.run([binary, "inputs.txt"], cwd=d, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout + r.stderr


def _check_far_field(name, odat, gdat, peak, tol=TOL):
    """Far-field series on a common time axis.  The reference writes each
    angle's series from its first non-zero bin (fdtd_solver.f90:8483-8534)
    and records that start in the time correction r/c - (start-1) dt, which
    the post-processor applies as a phase (post_processor.py:245-249).  The
    first non-zero bin is set by the smallest pulse-tail contributions, so
    two correct runs may start a few bins apart; aligned by their own time
    corrections, the series must agree (relative L2 <= TOL) and the shift
    must be a whole number of steps."""
    import postproc
    o, g = postproc.parse_dat(odat), postproc.parse_dat(gdat)
    dt = o["time_step"]
    for q in range(2 * o["num_angles"]):
        a = q // 2
        sh = (o["time_corr"][a] - g["time_corr"][a]) / dt  # start_g - start_o in steps
        s = int(round(sh))
        assert abs(sh - s) < 1e-3 * max(1.0, abs(sh)), (name, a, sh)
        so, sg = o["ff"][q], g["ff"][q]
        T = len(so)
        # GPU sample n is oracle sample n + s; compare where both windows hold data
        n0, n1 = max(0, -s), min(T, T - s)
        assert n1 - n0 >= T // 2, (name, q, s)
        err = rel_l2(so[n0 + s:n1 + s], sg[n0:n1], floor=1e-3 * peak)
        assert err <= tol, "%s: far field %d (angle %d) rel L2 %.3g (start shift %d)" % (name, q, a, err, s)


def _kmax_far_field(dat):
    """Constant-k far-field series of a .dat (complex, per angle theta then
    phi) and the per-angle time corrections."""
    blocks, _ = dat_blocks(dat)
    series, corr = [], None
    for t, b in blocks:
        if t.startswith("far field rE"):
            series.append(b[1:, 0] + 1j * b[1:, 1])  # row 0 holds theta, phi
        elif t.startswith("far field phase correction"):
            corr = b[:, 0]
    return series, corr


def _check_far_field_kmax(name, odat, gdat, dt, peak):
    """As _check_far_field, for the complex series of a constant-k run."""
    so_all, co = _kmax_far_field(odat)
    sg_all, cg = _kmax_far_field(gdat)
    assert len(so_all) == len(sg_all) > 0
    for q, (so, sg) in enumerate(zip(so_all, sg_all)):
        a = q // 2
        sh = (co[a] - cg[a]) / dt
        s = int(round(sh))
        assert abs(sh - s) < 1e-3 * max(1.0, abs(sh)), (name, a, sh)
        T = len(so)
        n0, n1 = max(0, -s), min(T, T - s)
        assert n1 - n0 >= T // 2, (name, q, s)
        err = rel_l2(so[n0 + s:n1 + s], sg[n0:n1], floor=1e-3 * peak)
        assert err <= TOL, "%s: far field %d (angle %d) rel L2 %.3g (start shift %d)" % (name, q, a, err, s)


@pytest.mark.parametrize("name", sorted(decks.DECKS))
def test_deck_parity(name, tmp_path, oracle_bin, gpu_lib):
    import alpineem_b200 as ab

    od, gd, md = tmp_path / "oracle", tmp_path / "gpu", tmp_path / "oracle_mid"
    for p in (od, gd, md):
        p.mkdir()
    _, kmax = decks.write_deck(name, str(od))
    decks.write_deck(name, str(gd))
    decks.write_deck(name, str(md))
    binary = oracle_bin["fdtd_oracle_kmax" if kmax else "fdtd_oracle"]
    _run_oracle(binary, str(od))
    # fields are compared half way through, while the pulse is in the grid
    # (after it leaves, only rounding-level residue remains)
    half = decks.DECKS[name]["steps"] // 2
    _run_oracle(binary, str(md), max_steps=half)

    with ab.Simulation(str(gd / "inputs.txt"), kmax=kmax, outdir=str(gd)) as sim:
        sim.run(half)
        gfields = [sim.field(c) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")]
        sim.run_all()

    fname = decks.DECKS[name].get("name", "data.dat")
    ob, olines = dat_blocks(str(od / fname))
    gb, glines = dat_blocks(str(gd / fname))
    assert len(olines) == len(glines)
    nh = 19 if kmax else 17
    assert [ln.split()[:3] for ln in olines[:nh]] == [ln.split()[:3] for ln in glines[:nh]]
    for a, b in zip(header_values(olines, nh), header_values(glines, nh)):
        np.testing.assert_allclose(np.array(a, float), np.array(b, float), rtol=1e-6)
    assert len(ob) == len(gb)
    peak = max(np.linalg.norm(b) for _, b in ob)
    for (ta, a), (tb, b) in zip(ob, gb):
        assert ta == tb and a.shape == b.shape, (ta, tb)
        if ta.startswith("far field rE") or ta.startswith("far field phase correction"):
            continue  # compared on a common time axis below
        # an all-but-zero block (e.g. cross polarisation of a symmetric case)
        # is judged against the largest block of the run
        err = rel_l2(a, b, floor=1e-3 * peak)
        assert err <= TOL, "%s: block '%s' rel L2 %.3g" % (name, ta, err)
    if not kmax:
        _check_far_field(name, str(od / fname), str(gd / fname), peak)
    elif decks.DECKS[name].get("ff"):
        dt = float(olines[4].split()[3])
        _check_far_field_kmax(name, str(od / fname), str(gd / fname), dt, peak)

    ofields = read_oracle_dump(str(md / "fields.bin"), kmax)
    # a component that stays near zero (e.g. Ex of an x-travelling wave) is
    # judged against the largest E (or H) component, 1e-2 of whose norm is
    # still far above FP32 rounding noise
    epeak = max(np.linalg.norm(f) for f in ofields[:3])
    hpeak = max(np.linalg.norm(f) for f in ofields[3:])
    for c, (a, b) in enumerate(zip(ofields, gfields)):
        assert a.shape == b.shape, (c, a.shape, b.shape)
        err = rel_l2(a, b, floor=1e-2 * (epeak if c < 3 else hpeak))
        assert err <= TOL, "%s: field %d rel L2 %.3g" % (name, c, err)

    geo = fname[:-4] + "_geometry.bin"
    if "geometry_bin no" in decks.DECKS[name].get("_ext", ""):
        assert not (gd / geo).exists()
    else:
        assert (od / geo).read_bytes() == (gd / geo).read_bytes()
