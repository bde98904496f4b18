"""The drop-in executable (alpineem_b200/_lib/FDTD-B200, and the FDTD-B200-kmax
name that selects the constant-k grammar), run the way main_fdtd/master.py
runs the reference solver (`./<solver> inputs.txt` in the deck's
directory): it prints the reference's progress lines
(fdtd_solver.f90:8312-8317 and the setup / post-processing lines), writes
the same .dat as a run through the library (every block bit-equal: the
far-field bins, real and constant-k, are summed in a fixed order), and
leaves a JSON run record (aem_run.json)."""
import json
import os
import re
import subprocess

import pytest

import decks
from datfile import dat_blocks

pytestmark = pytest.mark.gpu

LINES = [r"Reading in the inputs file and setting up the simulation\.\.\.",
         r"Setup is finished\. Time to complete was \d+\.\d{3} seconds\.",
         r"Starting main FDTD algorithm\.\.\.",
         r"Finished main FDTD algorithm\. Time to complete was \d+\.\d{3} seconds\.",
         r"Average of \d+\.\d{2} Mcells per second\.",
         r"Post processing some data\.\.\.",
         r"Finished post processing\. Time to complete was \d+\.\d{3} seconds\."]


@pytest.mark.parametrize("name,exe", [("dipole_port", "FDTD-B200"), ("kmax_te", "FDTD-B200-kmax"),
                                      ("kmax_ff", "FDTD-B200-kmax")])
def test_executable_drop_in(name, exe, tmp_path, gpu_lib):
    import numpy as np
    import alpineem_b200 as ab
    de, dl = tmp_path / "exe", tmp_path / "lib"
    de.mkdir()
    dl.mkdir()
    _, kmax = decks.write_deck(name, str(de))
    decks.write_deck(name, str(dl))
    binary = os.path.join(os.path.dirname(ab.LIB_PATH), exe)
    r = subprocess.run([binary, "inputs.txt"], cwd=str(de), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = [ln for ln in r.stdout.splitlines() if not re.fullmatch(r"\d+ of \d+ time steps", ln)]
    assert len(out) == len(LINES), r.stdout
    for ln, pat in zip(out, LINES):
        assert re.fullmatch(pat, ln), (ln, pat)
    with ab.Simulation(str(dl / "inputs.txt"), kmax=kmax, outdir=str(dl)) as sim:
        sim.run_all()
        steps = sim.steps[1]
    fname = decks.DECKS[name].get("name", "data.dat")
    be, le = dat_blocks(str(de / fname))
    bl, ll = dat_blocks(str(dl / fname))
    assert len(le) == len(ll) and len(be) == len(bl)
    for (ta, a), (tb, b) in zip(be, bl):
        assert ta == tb
        assert np.array_equal(a, b), (name, ta)
    rec = json.load(open(str(de / "aem_run.json")))
    assert rec["solver"] == "FDTD-B200" and rec["mode"] == ("kmax" if kmax else "standard")
    assert rec["steps"] == steps and rec["loop_s"] > 0 and rec["mcells_per_s"] > 0
    assert rec["algorithmic_bytes_per_step"] > 0 and rec["kernel_launches"] >= steps
