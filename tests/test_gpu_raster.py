"""The device rasteriser (aem_raster.cu) against the host model builder.

A run without sheets, Drude poles or <name>_geometry.bin draws its per-cell
material ids on the GPU; AEM_HOST_RASTER=1 keeps the host builder's ids
(aem_model.cpp, the restatement of fdtd_solver.f90:2051-2288).  Both must
give the same id in every cell and therefore bit-identical fields: bulk
files of random ids (unknown, negative and fractional values), objects of
every kind reaching the grid's faces and the periodic duplicate layer or
crossing out of the grid, periodic x and periodic y,z grids, and the
bulk-file ellipsoid workload.  Parity of the
same decks against the oracle is covered by the deck parity test."""
import numpy as np
import pytest

import decks

pytestmark = pytest.mark.gpu

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _ellipsoids_device():
    d = dict(decks.DECKS["ellipsoids_small"])
    d["_ext"] = d["_ext"] + "geometry_bin no\n"
    return d


def _clipped(base, extra):
    """`base` with objects that reach outside the grid (both builders clip
    them to cells 1..N-1; the reference writes them out of its arrays'
    bounds, so the oracle decks keep every object inside)."""
    d = dict(decks.DECKS[base])
    d["objects"] = list(d["objects"]) + extra
    return d


EXTRA = {
    "ellipsoids_device": _ellipsoids_device,
    "raster_clip_x": lambda: _clipped("raster_pbc_x", [
        ("block", 3, (35, 3, 5), (10, 6, 6)), ("sphere", 5, (2, 12, 20), 5), ("cylinder", 2, "z", (5, 5, 30), (10, 3))]),
    "raster_clip_yz": lambda: _clipped("raster_pbc_yz", [
        ("sphere", 3, (20, 1, 13), 4), ("cylinder", 5, "z", (26, 11, 1), (20, 3)), ("block", 3, (-2, 4, 4), (6, 3, 3))]),
}
CASES = ["raster_pbc_x", "raster_pbc_yz"] + sorted(EXTRA)


def _run(name, d, monkeypatch, host):
    import alpineem_b200 as ab
    if host:
        monkeypatch.setenv("AEM_HOST_RASTER", "1")
    else:
        monkeypatch.delenv("AEM_HOST_RASTER", raising=False)
    if name in EXTRA:
        decks.DECKS[name] = EXTRA[name]()
    decks.write_deck(name, str(d))
    with ab.Simulation(str(d / "inputs.txt"), outdir=str(d)) as sim:
        ids = sim.field("material")
        sim.run(decks.DECKS[name]["steps"] // 2)
        return ids, [sim.field(c) for c in FIELDS], sim.transfer_bytes[0]


@pytest.mark.parametrize("name", CASES)
def test_device_ids_equal_host_ids(name, tmp_path, gpu_lib, monkeypatch):
    a, b = tmp_path / "device", tmp_path / "host"
    a.mkdir()
    b.mkdir()
    ids_d, f_d, h2d_d = _run(name, a, monkeypatch, False)
    ids_h, f_h, h2d_h = _run(name, b, monkeypatch, True)
    assert ids_d.shape == ids_h.shape
    # the host path uploads one byte per cell, the device path the bulk
    # file's four (or nothing without a bulk file)
    assert h2d_d != h2d_h
    assert len(np.unique(ids_h)) > 2, "the deck should exercise several materials"
    bad = np.argwhere(ids_d != ids_h)
    assert bad.size == 0, "%s: %d cells differ, first (z, y, x) %s: device %d host %d" % (
        name, len(bad), tuple(bad[0]), ids_d[tuple(bad[0])], ids_h[tuple(bad[0])])
    for c, u, v in zip(FIELDS, f_d, f_h):
        assert np.array_equal(u, v), "%s: %s differs (max %.3g)" % (name, c, np.abs(u - v).max())


def test_material_field_matches_geometry_output(tmp_path, gpu_lib, monkeypatch):
    """The material indices read back (comp 6) against <name>_geometry.bin of
    the same deck: channel 0 holds each cell's material id as the reference
    writes it, which maps to the index through the deck's material list."""
    import alpineem_b200 as ab
    monkeypatch.delenv("AEM_HOST_RASTER", raising=False)
    name = "raster_pbc_x"
    d = dict(decks.DECKS[name])
    d["_ext"] = ""
    decks.DECKS["raster_geo"] = d
    decks.write_deck("raster_geo", str(tmp_path))
    with ab.Simulation(str(tmp_path / "inputs.txt"), outdir=str(tmp_path)) as sim:
        ids = sim.field("material")
    geo = np.fromfile(str(tmp_path / "data_geometry.bin"), np.float32).reshape(ids.shape + (4,))[..., 0]
    known = {float(m[1]): r + 1 for r, m in enumerate(d["mats"])}
    expect = np.vectorize(lambda v: known.get(float(int(v)), -1) if v >= 0 else 0)(geo)
    # cells whose geometry value names no material keep what was there
    # before (background or an earlier object), so compare the rest
    sel = expect >= 0
    assert sel.mean() > 0.5
    assert np.array_equal(ids[sel], expect[sel])
