"""Regenerate the committed golden fixtures from the reference checkout.

Run in a container that has the AlpineEM reference at ``--ref`` (default:
the ALPINEEM_REFERENCE environment variable, else ``/root/reference``):

    python tests/golden/make_fixtures.py

For each example below it executes the example's own deck writers
(``master.py``, ``master_clear.py``, ``master_metal.py`` ...) in a scratch
directory with ``os.system`` replaced by a no-op, so only the positional
``inputs*.txt`` files are produced (the solver is never launched).  The
decks, any binary side inputs they name, and the example's committed
post-processed CSV outputs are copied under ``tests/golden/<case>/``.

The CSVs are the reference's published results of full example runs
(examples/*/README.md); they pin the solver end to end through the
post-processor.  Large CSVs are thinned to every ``--stride``-th row (the
frequency column is kept, so rows stay self-describing).
"""
import argparse
import json
import os
import runpy
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))

# case name -> (example dir, deck scripts, extra inputs, golden csv files,
#               post-processor settings restated from that example's copy)
CASES = {
    "multilayer_slab": dict(
        src="trans_and_refl_infinite_multilayered_slab",
        decks=["master.py", "master_clear.py", "master_metal.py"],
        extra=[],
        csv=["S_parameters.csv"],
        post=dict(simulation_type="plane wave", use_metal=True),
    ),
    "drude_slab": dict(
        src="trans_and_refl_infinite_Drude(plasma)_slab",
        decks=["master.py", "master_clear.py", "master_metal.py"],
        extra=[],
        csv=["S_parameters.csv"],
        post=dict(simulation_type="plane wave", use_metal=True),
    ),
    "subpixel_slab": dict(
        src="sub_pixel_averaging_and_conforming_dielectric_slab",
        decks=["master.py", "master_clear.py", "master_metal.py"],
        extra=["optional_geom_bulk.bin", "materials_id_opfile.npy"],
        csv=["S_parameters.csv"],
        post=None,  # filled from the example's post_processor.py below
    ),
    "pec_sphere": dict(
        src="metal_sphere_monostatic_scattering",
        decks=["master.py", "master_clear.py"],
        extra=[],
        csv=["Scattering_Far_Field.csv", "Scattering_Far_Field-MP.csv", "Scattering_Far_Field-ACC.csv"],
        post=dict(simulation_type="plane wave", use_metal=False),
    ),
    "dipole_antenna": dict(
        src="radiating_dipole_antenna",
        decks=["master.py"],
        extra=[],
        csv=["S_parameters.csv", "Realized_antenna_gain.csv"],
        post=dict(simulation_type="antenna", use_metal=False),
    ),
    "igp_half_sphere": dict(
        src="metal_half_sphere_IGP_monostatic_scattering",
        decks=["master.py", "master_clear.py", "master_clear_no_IGP.py"],
        extra=[],
        csv=["Scattering_Far_Field.csv"],
        post=None,
    ),
}


def _post_settings(pp_path):
    """Read the settings block of an example's post_processor.py copy."""
    out = {}
    with open(pp_path) as f:
        for line in f:
            s = line.split("#")[0].strip()
            for key in ("simulation_type", "use_metal", "use_IGP_full_clear", "padding",
                        "data_filename", "clear_filename", "metal_filename", "IGP_full_clear_filename"):
                if s.startswith(key + "=") or s.startswith(key + " ="):
                    out[key] = eval(s.split("=", 1)[1])  # literal values only
    return out


def _run_decks(ex_dir, scripts, extra, dst):
    tmp = tempfile.mkdtemp()
    try:
        for e in extra:
            shutil.copy(os.path.join(ex_dir, e), tmp)
        cwd = os.getcwd()
        os.chdir(tmp)
        real_system = os.system
        os.system = lambda cmd: 0
        try:
            for s in scripts:
                runpy.run_path(os.path.join(ex_dir, s), run_name="__main__")
        finally:
            os.system = real_system
            os.chdir(cwd)
        for fn in sorted(os.listdir(tmp)):
            if fn.startswith("inputs") and fn.endswith(".txt"):
                shutil.copy(os.path.join(tmp, fn), dst)
    finally:
        shutil.rmtree(tmp)


def _thin_csv(src, dst, stride):
    with open(src) as f:
        lines = f.read().splitlines()
    keep = [lines[0]] + [l for n, l in enumerate(lines[1:]) if n % stride == 0]
    with open(dst, "w") as f:
        f.write("\n".join(keep) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ALPINEEM_REFERENCE", "/root/reference"))
    ap.add_argument("--stride", type=int, default=4)
    args = ap.parse_args()
    manifest = {}
    for case, spec in CASES.items():
        ex_dir = os.path.join(args.ref, "examples", spec["src"])
        dst = os.path.join(HERE, case)
        os.makedirs(dst, exist_ok=True)
        _run_decks(ex_dir, spec["decks"], spec["extra"], dst)
        for e in spec["extra"]:
            if e.endswith(".bin"):
                shutil.copy(os.path.join(ex_dir, e), dst)
        for c in spec["csv"]:
            _thin_csv(os.path.join(ex_dir, c), os.path.join(dst, c), args.stride)
        post = _post_settings(os.path.join(ex_dir, "post_processor.py"))
        manifest[case] = dict(source="examples/" + spec["src"], decks=spec["decks"], csv=spec["csv"],
                              csv_row_stride=args.stride, post_processor=post)
        print(case, "->", sorted(os.listdir(dst)))
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    sys.exit(main())
