"""TF/SF corrections in their own kernels (k_tfsf_h / k_tfsf_e) against the
same corrections inside the update kernels (AEM_TFSF_INLINE=1): when the
TF/SF faces stay clear of every CPML slab no CPML term reaches them, so
adding the corrections after the update is the reference's sequence of
operations and every field must agree bit for bit; plane waves at oblique
and normal incidence, an image ground plane, periodic y and z with a
Drude layer, and random materials across the faces."""
import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
CASES = ["tfsf_sphere", "smoke", "igp", "video", "raster_pbc_yz", "drude_pbc"]


def _fields(name, d, monkeypatch, inline):
    import alpineem_b200 as ab
    if inline:
        monkeypatch.setenv("AEM_TFSF_INLINE", "1")
    else:
        monkeypatch.delenv("AEM_TFSF_INLINE", raising=False)
    _, kmax = decks.write_deck(name, str(d))
    with ab.Simulation(str(d / "inputs.txt"), kmax=kmax, outdir=str(d)) as sim:
        sim.run(decks.DECKS[name]["steps"] // 2)
        return [sim.field(c) for c in FIELDS]


@pytest.mark.parametrize("name", CASES)
def test_tfsf_kernels_equal_inline(name, tmp_path, gpu_lib, monkeypatch):
    a, b = tmp_path / "sep", tmp_path / "inline"
    a.mkdir()
    b.mkdir()
    fa = _fields(name, a, monkeypatch, False)
    fb = _fields(name, b, monkeypatch, True)
    for c, u, v in zip(FIELDS, fa, fb):
        assert np.array_equal(u, v), "%s: %s differs (max %.3g)" % (name, c, np.abs(u - v).max())
