"""On-the-fly spectra of the per-step series (sidecar extension
`dft_freqs f_start f_stop count`, aem_read_spectrum): the tap kernel adds
x[m] exp(-2 pi i f m dt) to FP64 sums with Kahan compensation every step.
Each spectrum must equal a float64 numpy DFT of the same raw samples
(aem_read_probe) to 1e-12 relative (the reference post-processors take
numpy FFTs of these series: utility_scripts/post_processor.py,
post_processor_kmax.py), on a constant-k unit cell (TE and TM plane sums)
and on a lumped-port antenna (port voltage).  Graph replay accumulates in
the same order as eager steps, so its spectra are bit-identical; a deck
without per-step series rejects the extension."""
import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu

EXT = "dft_freqs 1e9 2e10 64\n"


def _numpy_dft(x, dt, freqs):
    m = np.arange(len(x))
    return np.exp(-2j * np.pi * np.outer(freqs, m * dt)) @ x


def _sim(name, tmp_path, ext=EXT):
    import alpineem_b200 as ab
    d = decks.DECKS[name]
    return ab.Simulation(deck_text=decks.deck_text(d), ext_text=ext, kmax=bool(d.get("kmax")), outdir=str(tmp_path))


@pytest.mark.parametrize("name,series", [("kmax_te", ("reflected", "transmitted", "reflected_tm", "transmitted_tm")),
                                         ("kmax_tm", ("reflected", "transmitted", "reflected_tm", "transmitted_tm")),
                                         ("dipole_port", ("port_voltage",))])
def test_spectrum_matches_fp64_dft(name, series, tmp_path, gpu_lib):
    with _sim(name, tmp_path) as sim:
        sim.run(sim.steps[1])
        dt = sim.time_step
        nonzero = 0
        for kind in series:
            f, X = sim.spectrum(kind)
            assert len(f) == 64 and f[0] == 1e9 and abs(f[-1] - 2e10) <= 1e-6
            x = sim.probe(kind)
            if not np.any(x):  # e.g. the TE sums of a TM unit cell are exactly zero
                assert not np.any(X), (name, kind)
                continue
            nonzero += 1
            ref = _numpy_dft(x, dt, f)
            err = np.linalg.norm(X - ref) / np.linalg.norm(ref)
            assert err <= 1e-12, (name, kind, err)
        assert nonzero >= 1, name


def test_spectrum_graph_replay_bit_identical(tmp_path, gpu_lib):
    out = []
    for mode in ("eager", "graph"):
        d = tmp_path / mode
        d.mkdir()
        with _sim("kmax_te", d) as sim:
            total = sim.steps[1]
            if mode == "graph":
                sim.run(1)
                sim.run_graph(total - 1, 32)
            else:
                sim.run(total)
            out.append([sim.spectrum(k)[1] for k in ("reflected", "transmitted", "reflected_tm", "transmitted_tm")])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_spectrum_needs_a_series(tmp_path, gpu_lib):
    import alpineem_b200 as ab
    with pytest.raises(ab.AemError, match="dft_freqs"):
        _sim("tfsf_sphere", tmp_path)
    with _sim("kmax_te", tmp_path, ext=None) as sim:
        sim.run(3)
        with pytest.raises(ab.AemError, match="dft_freqs"):
            sim.spectrum("reflected")
