"""The fused H+E kernels (k_yee4 on grids without x/y periodicity, k_yee on
x- or y-periodic ones) against the general two-kernel update
(k_update_h / k_update_e, selected by AEM_TWO_KERNEL=1): both apply the
reference's statements in its order in FP32, so every field must agree bit
for bit, on every deck the fused kernels take (ports, CPML on six faces,
material interfaces across tile seams, bulk-file ellipsoids, x- and
z-periodic grids, chunk boundaries in z, CPML slabs up to 23 cells deep), at an odd step inside the run and
at its end."""
import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
FUSED = ["dipole_port", "fused_wide", "ellipsoids_small", "dipole_pbc_x", "fused_long_z", "fused_pml_edge", "fused_pml_deep"]


def _fields(name, d, monkeypatch, two_kernel, steps):
    import alpineem_b200 as ab
    if two_kernel:
        monkeypatch.setenv("AEM_TWO_KERNEL", "1")
    else:
        monkeypatch.delenv("AEM_TWO_KERNEL", raising=False)
    decks.write_deck(name, str(d))
    out = []
    with ab.Simulation(str(d / "inputs.txt"), outdir=str(d)) as sim:
        # the first step shows which update ran (the fused kernel's own phase)
        sim.profile(True)
        sim.run(1)
        assert (sim.profile_read()["yee"][1] > 0) != two_kernel
        sim.profile(False)
        for s in steps:
            sim.run(s - sim.steps[0])
            out.append([sim.field(c) for c in FIELDS])
    return out


@pytest.mark.parametrize("name", FUSED)
def test_fused_equals_two_kernel(name, tmp_path, gpu_lib, monkeypatch):
    a, b = tmp_path / "fused", tmp_path / "two"
    a.mkdir()
    b.mkdir()
    total = decks.DECKS[name]["steps"]
    steps = (total // 2 + 1, total)
    fa = _fields(name, a, monkeypatch, False, steps)
    fb = _fields(name, b, monkeypatch, True, steps)
    for s, x, y in zip(steps, fa, fb):
        for c, u, v in zip(FIELDS, x, y):
            assert np.array_equal(u, v), "%s step %d: %s differs (max %.3g)" % (name, s, c, np.abs(u - v).max())
