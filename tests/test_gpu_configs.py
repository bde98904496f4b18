"""Parity at the full benchmark configurations, not only on small decks.

* PEC-sphere scattering (alpineem_b200.workloads.pec_sphere): 96^3 cells,
  10-cell CPML with the graded profile of the configuration (extension
  cpml_grading), TF/SF box inset 15 cells (tfsf_inset), x-polarised plane
  wave, PEC sphere of radius 20 cells, 37 far-field angles, 3 point probes
  (probe), all 2000 steps.  The FP32 GPU run against the FP32 oracle: every
  numeric .dat block and every probe series at relative L2 <= 1e-4, the
  far-field series on their common time axis at <= 1e-3 (the tolerance set
  for far-field outputs; both FP32 runs accumulate millions of terms per
  bin, in different orders).  Against the FP64 oracle: probe series
  <= 1e-4, far-field series <= 1e-3.
* Dispersive anisotropic layered slab (workloads.layered_slab): the full
  128 x 128 x 512 unit cell (eight anisotropic lossy layers, a 2-pole Drude
  layer, a 100 S sheet, 12-cell CPML on z), 600 of its 8000 steps (the
  oracle needs minutes for the whole run): reflected and transmitted plane
  sums against the FP64 oracle at <= 1e-4, and against the FP32 oracle at
  <= 1e-4 or twice that oracle's own FP64 error, whichever is larger,
  and the on-the-fly spectra at 256 frequencies against a float64 DFT of the
  run's own samples at <= 1e-12.

* Batched constant-k sweep (workloads.kmax_batch): four of its 64 unit
  cells (TE and TM, normal and oblique incidence, two depths), each with the
  sweep's 16x16-patch sheet, slab and 128-frequency spectra, advanced
  together by run_batch (graph replay, one stream each) for 320 steps;
  every instance's four plane sums (TE and TM, reflected and transmitted)
  against its own FP64 oracle run at <= 1e-4.

With AEM_PRECISION_REPORT set to a file name, the errors against FP64 are
appended to it as JSON lines, as in test_gpu_precision.py.
"""
import json
import os

import numpy as np
import pytest

from datfile import dat_blocks, rel_l2
from test_gpu_parity import _check_far_field, _run_oracle
from test_gpu_precision import _far_field_err

pytestmark = pytest.mark.gpu

TOL, TOL_FF64 = 1e-4, 1e-3


def _write(d, deck, ext):
    from alpineem_b200.deck import deck_text
    with open(os.path.join(d, "inputs.txt"), "w") as f:
        f.write(deck_text(deck))
    with open(os.path.join(d, "inputs.txt.b200"), "w") as f:
        f.write(ext)


def _report(entry):
    rep = os.environ.get("AEM_PRECISION_REPORT")
    if rep:
        with open(rep, "a") as f:
            f.write(json.dumps(entry) + "\n")


def _blocks_err(odat, gdat, skip_far_field=True):
    ob, _ = dat_blocks(odat)
    gb, _ = dat_blocks(gdat)
    assert len(ob) == len(gb)
    peak = max(np.linalg.norm(b) for _, b in ob)
    worst = {}
    for (ta, a), (tb, b) in zip(ob, gb):
        assert ta == tb and a.shape == b.shape, (ta, tb)
        if skip_far_field and (ta.startswith("far field rE") or ta.startswith("far field phase correction")):
            continue
        worst[ta] = rel_l2(a, b, floor=1e-3 * peak)
    return worst, peak


def test_pec_sphere_full(tmp_path, oracle_bin, gpu_lib):
    import alpineem_b200 as ab
    from alpineem_b200 import workloads
    deck, ext, probes = workloads.pec_sphere()
    o32, o64, gd = tmp_path / "o32", tmp_path / "o64", tmp_path / "gpu"
    for p in (o32, o64, gd):
        p.mkdir()
        _write(str(p), deck, ext)
    _run_oracle(oracle_bin["fdtd_oracle"], str(o32), dump_fields=False)
    _run_oracle(oracle_bin["fdtd_oracle_f64"], str(o64), dump_fields=False)
    with ab.Simulation(str(gd / "inputs.txt"), outdir=str(gd)) as sim:
        sim.run_all()
        raw = [sim.probe("point", q) for q in range(3 * len(probes))]

    # FP32 GPU against the FP32 oracle
    worst, peak = _blocks_err(str(o32 / "data.dat"), str(gd / "data.dat"))
    assert max(worst.values()) <= TOL, worst
    _check_far_field("pec_sphere", str(o32 / "data.dat"), str(gd / "data.dat"), peak, tol=TOL_FF64)
    pw, _ = _blocks_err(str(o32 / "data_probes.dat"), str(gd / "data_probes.dat"))
    assert len(pw) == 3 * len(probes) and max(pw.values()) <= TOL, pw
    # the file holds the raw samples aem_read_probe returns
    gb, _ = dat_blocks(str(gd / "data_probes.dat"))
    for (_, b), r in zip(gb, raw):
        np.testing.assert_allclose(b[:, 0], r, rtol=1e-8, atol=1e-30)

    # FP32 GPU against the FP64 oracle
    p64, _ = _blocks_err(str(o64 / "data_probes.dat"), str(gd / "data_probes.dat"))
    w64, peak64 = _blocks_err(str(o64 / "data.dat"), str(gd / "data.dat"))
    ff64 = _far_field_err(str(o64 / "data.dat"), str(gd / "data.dat"), peak64)
    _report({"deck": "pec_sphere_96_full", "probe_rel_l2": max(p64.values()),
             "dat_series_rel_l2": max(w64.values()), "far_field_rel_l2": ff64})
    assert max(p64.values()) <= TOL, p64
    assert max(w64.values()) <= TOL, w64
    assert ff64 <= TOL_FF64, ff64


def test_layered_slab_full_grid(tmp_path, oracle_bin, gpu_lib):
    import alpineem_b200 as ab
    from alpineem_b200 import workloads
    steps = 600
    deck, ext, layers = workloads.layered_slab()
    o32, o64, gd = tmp_path / "o32", tmp_path / "o64", tmp_path / "gpu"
    for p in (o32, o64, gd):
        p.mkdir()
        _write(str(p), deck, ext)
    _run_oracle(oracle_bin["fdtd_oracle"], str(o32), max_steps=steps, dump_fields=False, dump_series=True)
    _run_oracle(oracle_bin["fdtd_oracle_f64"], str(o64), max_steps=steps, dump_fields=False, dump_series=True)
    with ab.Simulation(str(gd / "inputs.txt"), outdir=str(gd)) as sim:
        sim.run(steps)
        g = {k: sim.probe(k) for k in ("reflected", "transmitted")}
        dt = sim.time_step
        spectra = {k: sim.spectrum(k) for k in ("reflected", "transmitted")}
    o = {k: np.loadtxt(str(o32 / ("series_%s.txt" % k))) for k in ("reflected", "transmitted")}
    o64s = {k: np.loadtxt(str(o64 / ("series_%s.txt" % k))) for k in ("reflected", "transmitted")}
    peak = max(np.linalg.norm(v) for v in o.values())
    errs32 = {k: rel_l2(o[k], g[k], floor=1e-3 * peak) for k in o}
    errs64 = {k: rel_l2(o64s[k], g[k], floor=1e-3 * peak) for k in o}
    oracle64 = {k: rel_l2(o64s[k], o[k], floor=1e-3 * peak) for k in o}
    _report({"deck": "layered_slab_128x128x512_%d_steps" % steps, "probe_rel_l2": max(errs64.values()),
             "fp32_oracle_rel_l2": max(oracle64.values())})
    assert max(errs64.values()) <= TOL, errs64
    # against the FP32 oracle: within the tolerance, or within twice the FP32
    # oracle's own error against FP64 (its 16384-term plane sums are
    # sequential FP32, the GPU's a tree)
    for k in o:
        assert errs32[k] <= max(TOL, 2 * oracle64[k]), (k, errs32[k], oracle64[k])
    m = np.arange(steps)
    for k, (f, X) in spectra.items():
        assert len(f) == 256 and f[0] == 1e9 and f[-1] == 3e10
        ref = np.exp(-2j * np.pi * np.outer(f, m) * dt) @ g[k]
        assert np.linalg.norm(X - ref) <= 1e-12 * np.linalg.norm(ref), k


def test_kmax_batch_instances(tmp_path, oracle_bin, gpu_lib):
    import alpineem_b200 as ab
    from alpineem_b200 import workloads
    from alpineem_b200.deck import deck_text
    steps, g = 320, 32
    picks = (1, 2, 3, 4)  # TM 128, TE 128, TM 192 oblique, TE 128 oblique
    # decks longer than the run: the oracle, cut short, dumps the raw sums
    decks = workloads.kmax_batch(steps=steps + 64)
    kinds = ("reflected", "transmitted", "reflected_tm", "transmitted_tm")
    sims = []
    try:
        for q in picks:
            d = tmp_path / ("gpu%d" % q)
            d.mkdir()
            sims.append(ab.Simulation(deck_text=deck_text(decks[q]), ext_text=workloads.KMAX_BATCH_EXT, kmax=True,
                                      outdir=str(d)))
        ab.run_batch(sims, steps, g)
        got = [{k: sim.probe(k) for k in kinds} for sim in sims]
    finally:
        for sim in sims:
            sim.close()
    worst = 0.0
    for q, gq in zip(picks, got):
        od = tmp_path / ("o64_%d" % q)
        od.mkdir()
        _write(str(od), decks[q], workloads.KMAX_BATCH_EXT)
        _run_oracle(oracle_bin["fdtd_oracle_kmax_f64"], str(od), max_steps=steps, dump_fields=False, dump_series=True)
        o = {}
        for k in kinds:
            a = np.loadtxt(str(od / ("series_%s.txt" % k)))
            o[k] = a[:, 0] + 1j * a[:, 1]
        peak = max(np.linalg.norm(v) for v in o.values())
        errs = {k: rel_l2(o[k], gq[k], floor=1e-3 * peak) for k in kinds}
        _report({"deck": "kmax_batch_instance_%d_%d_steps" % (q, steps), "probe_rel_l2": max(errs.values())})
        worst = max(worst, max(errs.values()))
        assert max(errs.values()) <= TOL, (q, errs)
