"""Generate the post-processing fixtures under tests/golden/postproc/.

For small decks (tests/decks.py) covering the reference post-processors'
modes, the FP32 oracle writes the .dat files and the
reference's own example post-processors (run unchanged from the reference
checkout, matplotlib replaced by a no-op module because only the CSV output
is used) write the CSVs:

  pp_antenna  dipole_port                         radiating_dipole_antenna/post_processor.py
              (lumped port, far field)            -> S_parameters.csv, Realized_antenna_gain.csv
  pp_scatter  tfsf_sphere + clear run             metal_sphere_monostatic_scattering/post_processor.py
                                                  -> Scattering_Far_Field.csv
  pp_slab     pbc_sheets + clear + metal runs     trans_and_refl_infinite_multilayered_slab/post_processor.py
                                                  -> S_parameters.csv (wave ports, use_metal)
  pp_igp      igp + clear + full-clear runs       metal_half_sphere_IGP_monostatic_scattering/post_processor.py
                                                  -> Scattering_Far_Field.csv (use_IGP_full_clear)
  pp_kmax_te  kmax_te + clear + metal runs        oblique_angle_plane_waves_w_periodic_boundaries_kmax/
  pp_kmax_tm  kmax_tm + clear + metal runs          post_processor_kmax.py -> S_parameters_k.csv

The GPU post-processor (alpineem_b200.postprocess) must reproduce the CSVs
from the committed .dat files (tests/test_postprocess.py).  Run here,
where the reference checkout and the oracle build exist:

    python tests/golden/make_postproc_fixtures.py
"""
import copy
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
# the reference checkout whose example post-processors this script runs
REF = os.path.join(os.environ.get("ALPINEEM_REFERENCE", "/root/reference"), "examples")
ORACLE = os.path.join(ROOT, "oracle", "_build", "fdtd_oracle")
ORACLE_K = os.path.join(ROOT, "oracle", "_build", "fdtd_oracle_kmax")
KMAX_EX = "oblique_angle_plane_waves_w_periodic_boundaries_kmax"

import decks  # noqa: E402


def _variant(name, out, **change):
    d = copy.deepcopy(decks.DECKS[name])
    d.update(change)
    d["name"] = out
    return d


CASES = {
    "pp_antenna": ("radiating_dipole_antenna", [_variant("dipole_port", "data.dat")]),
    "pp_scatter": ("metal_sphere_monostatic_scattering",
                   [_variant("tfsf_sphere", "data.dat"), _variant("tfsf_sphere", "clear.dat", objects=[])]),
    "pp_slab": ("trans_and_refl_infinite_multilayered_slab",
                [_variant("pbc_sheets", "data.dat"), _variant("pbc_sheets", "clear.dat", objects=[], sheets=[]),
                 _variant("pbc_sheets", "metal.dat", sheets=[],
                          mats=[("simple", 9, (1, 1, 1), ("1E8", "1E8", "1E8"))],
                          objects=[("block", 9, (16, 1, 1), (10, 10, 12))])]),
    "pp_igp": ("metal_half_sphere_IGP_monostatic_scattering",
               [_variant("igp", "data.dat"),
                _variant("igp", "clear.dat", objects=[("block", 6, (1, 1, 1), (32, 32, 16))]),
                _variant("igp", "IGP_full_clear.dat", igp=None, objects=[])]),
}
for _m in ("te", "tm"):
    _n = "kmax_" + _m
    CASES["pp_" + _n] = (KMAX_EX, [_variant(_n, "data-k.dat"), _variant(_n, "clear-k.dat", objects=[], sheets=[]),
                                   _variant(_n, "metal-k.dat", sheets=[],
                                            mats=[("simple", 9, (1, 1, 1), ("1E8", "1E8", "1E8"))],
                                            objects=[("block", 9, (14, 1, 1), (8, 10, 10))])])


def main():
    if not os.path.exists(ORACLE):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    for case, (example, dks) in CASES.items():
        tmp = tempfile.mkdtemp(prefix="pp_")
        for q, d in enumerate(dks):
            if d.get("igp") is None:
                d.pop("igp", None)
            deck = "inputs%d.txt" % q
            with open(os.path.join(tmp, deck), "w") as f:
                f.write(decks.deck_text(d))
            binary = ORACLE_K if d.get("kmax") else ORACLE
            r = subprocess.run([binary, deck], cwd=tmp, capture_output=True, text=True, timeout=1200)
            if r.returncode != 0:
                raise SystemExit(r.stdout[-2000:] + r.stderr[-2000:])
        stub = os.path.join(tmp, "stub", "matplotlib")
        os.makedirs(stub)
        open(os.path.join(stub, "__init__.py"), "w").close()
        with open(os.path.join(stub, "pyplot.py"), "w") as f:
            f.write("def __getattr__(n):\n    return lambda *a, **k: None\n")
        env = dict(os.environ, PYTHONPATH=os.path.join(tmp, "stub"), MPLBACKEND="Agg")
        script = os.path.join(REF, example, "post_processor_kmax.py" if example == KMAX_EX else "post_processor.py")
        r = subprocess.run([sys.executable, script], cwd=tmp, env=env, capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise SystemExit(r.stderr[-2000:])
        dst = os.path.join(HERE, "postproc", case)
        os.makedirs(dst, exist_ok=True)
        for f in sorted(os.listdir(tmp)):
            if f.endswith(".dat") or f.endswith(".csv"):
                shutil.copy(os.path.join(tmp, f), dst)
        print(case, sorted(os.listdir(dst)))
        shutil.rmtree(tmp)


if __name__ == "__main__":
    main()
