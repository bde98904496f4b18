"""The launch-shape autotuner of the general H/E update (aem_autotune,
extension `autotune N`): it times candidate shapes on the run's own steps,
and every shape computes each cell with the same statements, so a tuned run
must end with exactly the fields of an untuned one, through aem_run and
through the batched driver, and report a shape from the candidate list."""
import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
SHAPES = {(16, 8), (8, 8), (32, 8), (4, 8), (64, 8), (16, 4), (8, 4), (32, 4)}


def _sim(name, d, ext=""):
    import alpineem_b200 as ab
    _, kmax = decks.write_deck(name, str(d))
    if ext:
        p = d / "inputs.txt.b200"
        p.write_text((p.read_text() if p.exists() else "") + ext)
    return ab.Simulation(str(d / "inputs.txt"), kmax=kmax, outdir=str(d))


@pytest.mark.parametrize("name", ["tfsf_sphere", "kmax_te", "drude_pbc"])
def test_tuned_run_equals_untuned(name, tmp_path, gpu_lib):
    a, b, c = tmp_path / "plain", tmp_path / "api", tmp_path / "ext"
    for p in (a, b, c):
        p.mkdir()
    total = decks.DECKS[name]["steps"]
    with _sim(name, a) as s:
        s.run(total)
        want = [s.field(f) for f in FIELDS]
    with _sim(name, b) as s:
        shape = s.autotune(3)
        assert shape["update_h"] in SHAPES and shape["update_e"] in SHAPES
        assert s.steps[0] == 24  # eight candidates, three steps each
        s.run(total)
        got = [s.field(f) for f in FIELDS]
    for f, u, v in zip(FIELDS, want, got):
        assert np.array_equal(u, v), (name, f)
    with _sim(name, c, "autotune 2\n") as s:
        s.run(total)
        assert s.steps[0] == total
        got = [s.field(f) for f in FIELDS]
    for f, u, v in zip(FIELDS, want, got):
        assert np.array_equal(u, v), (name, f)


def test_tuned_batch_equals_untuned(tmp_path, gpu_lib):
    """Constant-k unit cells advanced together by the batched driver, each
    tuning its own shape first (their z extents differ)."""
    import alpineem_b200 as ab
    names = ["kmax_te", "kmax_tm"]
    plain = []
    for q, n in enumerate(names):
        d = tmp_path / ("p%d" % q)
        d.mkdir()
        with _sim(n, d) as s:
            s.run(128)
            plain.append([s.field(f) for f in FIELDS])
    sims = []
    try:
        for q, n in enumerate(names):
            d = tmp_path / ("b%d" % q)
            d.mkdir()
            sims.append(_sim(n, d, "autotune 2\n"))
        ab.run_batch(sims, 128, 32)
        for s, want in zip(sims, plain):
            assert s.steps[0] == 128
            for f, u in zip(FIELDS, want):
                assert np.array_equal(s.field(f), u), f
    finally:
        for s in sims:
            s.close()
