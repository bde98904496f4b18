"""Pins the CPU oracle to the reference's own golden data.

Each case under tests/golden/ is one of the reference's examples: its solver
decks (the inputs*.txt its master scripts write) and the CSVs the reference
committed from its own runs.  The oracle (FP32 build) runs every deck; the
post-processing restated in tests/postproc.py turns the .dat files into the
CSV quantities, which must match the committed CSVs.

Tolerance: relative L2 over the trusted band of the complex quantity
(amplitude and phase together) <= 1e-4.  The reference's own three committed
builds of the sphere case (main, -MP, -ACC) differ from each other by up to
3e-5 on the co-polarised column; the cross-polarised columns of the symmetric
cases are numerical noise (the reference's builds disagree with each other
there by several percent) and are not compared.

The slab cases finish in about a minute on 8 cores and always run; the 3-D
cases (sphere, image-plane half sphere, dipole antenna) take 5-15 minutes
each and run with ALPINEEM_SLOW=1.
"""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import postproc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-4
# checkout of the reference repository (for the one test that runs its
# post-processor script); the test is skipped without it
REF_ROOT = os.environ.get("ALPINEEM_REFERENCE", "")


def _run_case(case, tmp, binary):
    src = os.path.join(GOLDEN, case)
    for f in os.listdir(src):
        if not f.endswith(".csv"):
            shutil.copy(os.path.join(src, f), tmp)
    for deck in sorted(f for f in os.listdir(tmp) if f.startswith("inputs") and f.endswith(".txt")):
        r = subprocess.run([binary, deck], cwd=tmp, capture_output=True, text=True, timeout=3600)
        assert r.returncode == 0 and "ERROR" not in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
    return tmp


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _check(csv, freq, cols, which, tol=TOL):
    fref, ref = postproc.csv_complex(csv)
    got = postproc.match_rows(fref, freq, cols)
    for q in which:
        err = _rel(got[q], ref[q])
        assert err <= tol, "%s column %d: rel L2 %.3g" % (os.path.basename(csv), q, err)


@pytest.mark.parametrize("case", ["multilayer_slab", "drude_slab", "subpixel_slab"])
def test_slab_sparameters(case, tmp_path, oracle_bin):
    d = _run_case(case, str(tmp_path), oracle_bin["fdtd_oracle"])
    freq, S = postproc.plane_wave_sparams(os.path.join(d, "data.dat"), os.path.join(d, "clear.dat"),
                                          os.path.join(d, "metal.dat"))
    _check(os.path.join(GOLDEN, case, "S_parameters.csv"), freq, S, [0, 1])


@pytest.mark.slow
def test_pec_sphere_rcs(tmp_path, oracle_bin):
    d = _run_case("pec_sphere", str(tmp_path), oracle_bin["fdtd_oracle"])
    freq, F = postproc.scattering(os.path.join(d, "data.dat"), os.path.join(d, "clear.dat"))
    for csv in ("Scattering_Far_Field.csv", "Scattering_Far_Field-MP.csv", "Scattering_Far_Field-ACC.csv"):
        _check(os.path.join(GOLDEN, "pec_sphere", csv), freq, F, [0])


@pytest.mark.slow
def test_igp_half_sphere_rcs(tmp_path, oracle_bin):
    d = _run_case("igp_half_sphere", str(tmp_path), oracle_bin["fdtd_oracle"])
    freq, F = postproc.scattering(os.path.join(d, "data.dat"), os.path.join(d, "clear.dat"),
                                  full_clear=os.path.join(d, "IGP_full_clear.dat"))
    _check(os.path.join(GOLDEN, "igp_half_sphere", "Scattering_Far_Field.csv"), freq, F, [0])


@pytest.mark.slow
def test_dipole_antenna(tmp_path, oracle_bin):
    d = _run_case("dipole_antenna", str(tmp_path), oracle_bin["fdtd_oracle"])
    freq, S = postproc.antenna_sparams(os.path.join(d, "data.dat"))
    _check(os.path.join(GOLDEN, "dipole_antenna", "S_parameters.csv"), freq, S, [0])
    freq, G = postproc.antenna_gain(os.path.join(d, "data.dat"))
    # co-polarised (theta) column of every angle
    _check(os.path.join(GOLDEN, "dipole_antenna", "Realized_antenna_gain.csv"), freq, G,
           list(range(0, len(G), 2)))


@pytest.mark.skipif(not REF_ROOT or not os.path.isdir(REF_ROOT), reason="ALPINEEM_REFERENCE not set")
def test_postproc_restatement_matches_reference_script(tmp_path, oracle_bin):
    """The restated post-processing equals the reference's own script, run
    unchanged on the same oracle .dat files (matplotlib replaced by a no-op
    module because only its CSV output is used)."""
    d = _run_case("multilayer_slab", str(tmp_path), oracle_bin["fdtd_oracle"])
    stub = tmp_path / "stub" / "matplotlib"
    stub.mkdir(parents=True)
    (stub / "__init__.py").write_text("")
    (stub / "pyplot.py").write_text("def __getattr__(n):\n    return lambda *a, **k: None\n")
    script = os.path.join(REF_ROOT, "examples", "trans_and_refl_infinite_multilayered_slab", "post_processor.py")
    env = dict(os.environ, PYTHONPATH=str(tmp_path / "stub"), MPLBACKEND="Agg")
    r = subprocess.run([sys.executable, script], cwd=d, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    fref, ref = postproc.csv_complex(os.path.join(d, "S_parameters.csv"))
    freq, S = postproc.plane_wave_sparams(os.path.join(d, "data.dat"), os.path.join(d, "clear.dat"),
                                          os.path.join(d, "metal.dat"))
    got = postproc.match_rows(fref, freq, S)
    for q in (0, 1):
        assert _rel(got[q], ref[q]) < 1e-10
