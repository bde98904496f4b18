"""Small input decks in the reference's positional grammar
(main_fdtd/fdtd_solver.f90:726-1298; template main_fdtd/master.py:51-296),
one per solver feature, sized so the CPU oracle finishes each in seconds.
Used by the GPU parity tests and smoke()."""
import os

from alpineem_b200.deck import deck_text  # noqa: F401  (re-exported for the tests)


ANG = [(0, 0), (45, 30), (90, 180), (135, 270), (180, 0)]

DECKS = {
    # tiny all-round case (CPML, oblique TF/SF, dielectric sphere, far field)
    "smoke": dict(n=(32, 32, 32), steps=100, f="30E9", pulse=2, excitation=("plane wave", 1, 0, 50, 20, 10),
                  ff=[(90, 0), (30, 60)], ffc=(16, 16, 16), mats=[("simple", 3, (2.5, 2.5, 2.5), (0.005, 0.005, 0.005))],
                  objects=[("sphere", 3, (16, 16, 16), 3)]),
    # CPML on six faces, oblique TF/SF plane wave, dielectric + lossy sphere
    # (material interfaces), far field at 5 angles
    "tfsf_sphere": dict(n=(36, 34, 32), steps=220, f="20E9", pulse=2,
                        excitation=("plane wave", 1, 0, 30, 40, 20), ff=ANG, ffc=(18, 17, 16),
                        mats=[("simple", 5, (4, 3, 2.5), (0.01, 0.02, 0.0)), ("simple", 6, (1, 1, 1), ("1E8", "1E8", "1E8"))],
                        objects=[("sphere", 5, (18, 17, 16), 4), ("block", 6, (15, 15, 19), (3, 2, 2))]),
    # Gaussian-pulse lumped port driving a PEC dipole, far field at 3 angles
    "dipole_port": dict(n=(34, 34, 34), steps=300, f="15E9", pulse=1, excitation=("antenna", "0.001", 0, 1),
                        ff=[(90, 0), (90, 180), (45, 0)], ffc=(17, 17, 17),
                        mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8"))],
                        objects=[("block", 4, (17, 17, 12), (1, 1, 5)), ("block", 4, (17, 17, 18), (1, 1, 5))],
                        ports=[("basic", "z", 50, (17, 17, 17), (1, 1, 1))]),
    # unit cell periodic in y,z: dielectric slabs, Smith-Maloney sheets of
    # two normals, x-propagating plane wave, reflected/transmitted sums
    "pbc_sheets": dict(n=(40, 10, 12), dl=("0.5E-3", "0.5E-3", "0.5E-3"), steps=400, f="8E9", bc=(0, 0, 1, 1, 1, 1),
                       excitation=("plane wave", 1, 0, 90, 0, 90), name="data.dat",
                       mats=[("simple", 5, (2.1, 2.1, 2.1), (0, 0, 0)), ("simple", 6, (3.5, 3.0, 3.5), (0.01, 0, 0)),
                             ("sheet", 4, 25), ("sheet", 7, 50)],
                       objects=[("block", 5, (16, 1, 1), (5, 10, 12)), ("block", 6, (21, 1, 1), (4, 10, 12))],
                       sheets=[("x", 4, 16, (1, 1), (10, 12)), ("x", 7, 21, (1, 1), (10, 12)), ("z", 4, 5, (18, 1), (3, 10))]),
    # Drude ADE (2 poles) in a y,z-periodic unit cell
    "drude_pbc": dict(n=(40, 8, 8), dl=("0.5E-3", "0.5E-3", "0.5E-3"), steps=400, f="8E9", bc=(0, 0, 1, 1, 1, 1),
                      excitation=("plane wave", 1, 0, 90, 0, 0),
                      mats=[("plasma", 9, (3, 3, 3), (0.1, 0.1, 0.1), [("30E9", "10E9"), ("40E9", "5E9")])],
                      objects=[("block", 9, (16, 1, 1), (8, 8, 8))]),
    # x,y periodic, z propagating (z-marching with CPML on z only), Drude +
    # z-normal sheet
    "pbc_xy": dict(n=(8, 10, 36), dl=("0.5E-3", "0.5E-3", "0.5E-3"), steps=350, f="8E9", bc=(1, 1, 1, 1, 0, 0),
                   excitation=("plane wave", 1, 0, 0, 0, 90),
                   mats=[("plasma", 3, (2, 2, 2), (0.0, 0.0, 0.0), [("20E9", "8E9")]), ("sheet", 8, 40)],
                   objects=[("block", 3, (1, 1, 16), (8, 10, 5))], sheets=[("z", 8, 22, (1, 1), (8, 10))]),
    # image ground plane (-z) with a mirrored incident wave and far field
    "igp": dict(n=(32, 32, 32), steps=200, f="20E9", igp=("-z", 16), excitation=("plane wave", 1, 0, 180, 0, 90),
                ff=[(0, 0), (30, 45), (60, 90)], ffc=(16, 16, 16),
                mats=[("simple", 6, (1, 1, 1), ("1E8", "1E8", "1E8"))],
                objects=[("block", 6, (1, 1, 1), (32, 32, 16)), ("sphere", 6, (16, 16, 16), 4)]),
    # 2-D video slice and a cylinder
    "video": dict(n=(32, 31, 30), steps=100, f="25E9", excitation=("plane wave", 1, 0, 60, 120, 45),
                  video=("y", 15), mats=[("simple", 2, (3, 3, 3), (0, 0, 0))],
                  objects=[("cylinder", 2, "z", (16, 15, 12), (6, 3))]),
    # every step's cell-averaged fields exported (<name>_full_*.bin): a
    # dipole on the fused kernel and a constant-k unit cell (complex records)
    "full_dipole": dict(n=(26, 24, 22), steps=90, f="15E9", pulse=1, excitation=("antenna", 1, 0, 1), full="yes",
                        mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 5, (3, 3, 3), (0.01, 0, 0))],
                        objects=[("block", 4, (13, 12, 7), (1, 1, 5)), ("block", 4, (13, 12, 13), (1, 1, 5)),
                                 ("sphere", 5, (6, 7, 11), 3)],
                        ports=[("basic", "z", 50, (13, 12, 12), (1, 1, 1))]),
    "full_kmax": dict(kmax=True, n=(28, 6, 8), dl=("0.25E-3", "0.25E-3", "0.25E-3"), steps=150, f="8E9",
                      bc=(0, 0, 1, 1, 1, 1), excitation=("plane wave", 1, 0, "TE", "+"), k=("200.0", "100.0"), full="yes",
                      mats=[("simple", 5, (4, 4, 4), (0, 0, 0))], objects=[("block", 5, (10, 1, 1), (6, 6, 8))]),
    # constant-k periodic solver, TE and TM, oblique k in the y,z plane
    "kmax_te": dict(kmax=True, n=(36, 10, 10), dl=("0.25E-3", "0.25E-3", "0.25E-3"), steps=300, f="8E9", bc=(0, 0, 1, 1, 1, 1),
                    excitation=("plane wave", 1, 0, "TE", "+"), k=("300.0", "150.0"),
                    mats=[("simple", 5, (4, 4, 4), (0, 0, 0)), ("sheet", 7, 30)],
                    objects=[("block", 5, (14, 1, 1), (8, 10, 10))], sheets=[("x", 7, 14, (1, 1), (10, 10))]),
    "kmax_tm": dict(kmax=True, n=(36, 10, 10), dl=("0.25E-3", "0.25E-3", "0.25E-3"), steps=300, f="8E9", bc=(0, 0, 1, 1, 1, 1),
                    excitation=("plane wave", 1, 0, "TM", "-"), k=("0.0", "250.0"),
                    mats=[("simple", 5, (4, 4, 4), (0.02, 0.02, 0.02))],
                    objects=[("block", 5, (14, 1, 1), (8, 10, 10))]),
    # --- decks of the fused H+E kernel (no TF/SF, sheets, Drude or kmax) ---
    # x-periodic array of dipoles between lossy dielectric blocks; 2 CTAs in
    # x (wrap across them), several in y, far field on the y and z faces
    "dipole_pbc_x": dict(n=(40, 30, 34), steps=240, f="15E9", pulse=1, bc=(1, 1, 0, 0, 0, 0),
                         excitation=("antenna", 1, 0, 1), ff=[(90, 0), (60, 90), (30, 200)], ffc=(20, 15, 17),
                         mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 5, (3, 2, 4), (0.01, 0, 0.02))],
                         objects=[("block", 4, (20, 15, 12), (1, 1, 5)), ("block", 4, (20, 15, 18), (1, 1, 5)),
                                  ("sphere", 5, (9, 10, 20), 5), ("block", 5, (30, 4, 8), (12, 6, 6))],
                         ports=[("basic", "z", 50, (20, 15, 17), (1, 1, 1))]),
    # long z-periodic column whose port lies inside the y CPML slabs: the
    # bulk / port / CPML pass order of the reference
    "dipole_long_z": dict(n=(24, 20, 150), steps=200, f="15E9", pulse=1, bc=(0, 0, 0, 0, 1, 1),
                          excitation=("antenna", 1, 0, 1),
                          mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 6, (5, 5, 5), (0, 0, 0))],
                          objects=[("block", 4, (12, 10, 60), (1, 1, 6)), ("block", 4, (12, 10, 67), (1, 1, 6)),
                                   ("cylinder", 6, "z", (12, 10, 100), (40, 3))],
                          ports=[("basic", "z", 50, (12, 10, 66), (1, 1, 1))]),
    # z-periodic column wide enough to keep the port out of the CPML: three
    # z chunks of the fused kernel, the first recomputing the H plane across
    # the periodic wrap
    "fused_long_z": dict(n=(40, 36, 150), steps=200, f="15E9", pulse=1, bc=(0, 0, 0, 0, 1, 1),
                         excitation=("antenna", 1, 0, 1),
                         mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 6, (5, 5, 5), (0, 0, 0))],
                         objects=[("block", 4, (20, 18, 60), (1, 1, 6)), ("block", 4, (20, 18, 67), (1, 1, 6)),
                                  ("cylinder", 6, "z", (20, 18, 100), (40, 3))],
                         ports=[("basic", "z", 50, (20, 18, 66), (1, 1, 1))]),
    # long in x: three 128-cell tiles of the vectorised fused kernel, so the
    # -x halo column between CTAs is recomputed; materials across the tile
    # seams at x = 128 and 256, far field on all faces
    "fused_long_x": dict(n=(300, 22, 26), steps=220, f="15E9", pulse=1, excitation=("antenna", 1, 0, 1),
                         ff=[(90, 0), (45, 120)], ffc=(150, 11, 13),
                         mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 5, (4, 3, 2), (0.01, 0, 0))],
                         objects=[("block", 4, (150, 11, 8), (1, 1, 4)), ("block", 4, (150, 11, 14), (1, 1, 4)),
                                  ("block", 5, (120, 6, 6), (20, 8, 12)), ("sphere", 5, (256, 11, 13), 5)],
                         ports=[("basic", "z", 50, (150, 11, 13), (1, 1, 1))]),
    # long in x with the port clear of every CPML slab: three 128-cell x
    # tiles of the TMA-fed fused kernel (-x halo columns recomputed across
    # the seams at x = 128 and 256), materials across the seams, far field
    "fused_wide": dict(n=(300, 40, 34), steps=200, f="15E9", pulse=1, excitation=("antenna", 1, 0, 1),
                       ff=[(90, 0), (45, 120), (150, 250)], ffc=(150, 20, 17),
                       mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 5, (4, 3, 2), (0.01, 0, 0))],
                       objects=[("block", 4, (150, 20, 11), (1, 1, 5)), ("block", 4, (150, 20, 18), (1, 1, 5)),
                                ("block", 5, (120, 14, 12), (20, 10, 12)), ("sphere", 5, (256, 20, 17), 5)],
                       ports=[("basic", "z", 50, (150, 20, 17), (1, 1, 1))]),
    # x CPML 20 cells deep (sidecar pml_cells 19): the high x slab spans the
    # seam between the second and third 128-cell tiles of the fused kernel,
    # a lossy anisotropic block reaches into both x slabs and the y/z CPML
    # corner
    "fused_pml_edge": dict(n=(260, 52, 50), steps=120, f="15E9", pulse=1, excitation=("antenna", 1, 0, 1),
                           ff=[(90, 0), (45, 120)], ffc=(130, 26, 25),
                           mats=[("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 5, (4, 3, 2), (0.01, 0, 0))],
                           objects=[("block", 4, (130, 26, 20), (1, 1, 5)), ("block", 4, (130, 26, 30), (1, 1, 5)),
                                    ("block", 5, (5, 40, 12), (250, 6, 6))],
                           ports=[("basic", "z", 50, (130, 26, 25), (1, 1, 1))], _ext="pml_cells 19\n"),
    # CPML 23 cells deep (pml_cells 22) on every face
    "fused_pml_deep": dict(n=(260, 60, 60), steps=120, f="15E9", pulse=1, excitation=("antenna", 1, 0, 1),
                           ff=[(90, 0)], ffc=(130, 30, 30),
                           mats=[("simple", 5, (4, 3, 2), (0.01, 0, 0))],
                           objects=[("block", 5, (5, 44, 16), (250, 6, 6))],
                           ports=[("basic", "z", 50, (130, 30, 30), (1, 1, 1))], _ext="pml_cells 22\n"),
    # the throughput workload at 48^3: bulk-file ellipsoids, 6-cell CPML
    # (sidecar), a 1-cell port and 56 far-field angles
    "ellipsoids_small": "ellipsoids_small",
}


def _ellipsoids_small():
    from alpineem_b200 import workloads
    d, ext, bulk = workloads.dipole_ellipsoids(n=48, steps=260, n_ell=6, seed=2, pml_cells=6, dl="1E-3", f="20E9",
                                               theta_step=30, phi_step=45, arm=8, semi=(64, 256))
    d["_ext"] = ext.replace("geometry_bin no\n", "")
    d["_bulk"] = bulk
    return d


DECKS["ellipsoids_small"] = _ellipsoids_small()


def _gridded_port():
    """A gridded (one-way mode) port feeding a parallel-plate line: two PEC
    plates (sigma = 1e8) 6 cells apart in y, and on the port plane the TEM
    mode between them, written alongside as the reference's mode file
    ((4, n1+1, n2+1) float32, first index fastest: E1, E2, H1, H2 weights
    per point; fdtd_solver.f90:3723-3744): E along y uniform across the gap
    (1 / gap), H along x (1 / width)."""
    import numpy as np
    n1, n2, dl = 8, 6, 1e-3
    feed = np.zeros((n2 + 1, n1 + 1, 4), np.float32)
    feed[:n2, :, 1] = 1.0 / (n2 * dl)
    feed[:n2, :, 2] = 1.0 / (n1 * dl)
    return dict(n=(30, 28, 40), steps=250, f="10E9", pulse=1, excitation=("antenna", 1, 0, 1),
                ff=[(0, 0), (90, 45), (150, 300)], ffc=(15, 14, 20),
                mats=[("simple", 1, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 5, (2, 2, 2), (0.005, 0.005, 0.005))],
                objects=[("block", 1, (6, 9, 10), (20, 1, 24)), ("block", 1, (6, 16, 10), (20, 1, 24)),
                         ("sphere", 5, (15, 12, 30), 3)],
                ports=[("gridded", "+z", 50, (11, 10, 15), (n1, n2), "feed.bin")],
                _files={"feed.bin": feed.tobytes()})


# a gridded port: the mode projection of H, the H zeroing behind the feed
# plane and the E overwrite, with far field
DECKS["gridded_port"] = _gridded_port()
# constant-k unit cell with far-field angles: Bloch phase removed from the
# Huygens currents (ref :7202-7331) and binned every step (ref :7333-7507)
DECKS["kmax_ff"] = dict(kmax=True, n=(36, 10, 10), dl=("0.25E-3", "0.25E-3", "0.25E-3"), steps=300, f="8E9",
                        bc=(0, 0, 1, 1, 1, 1), excitation=("plane wave", 1, 0, "TE", "+"), k=("300.0", "150.0"),
                        ff=[(90, 0), (45, 0), (120, 180)], ffc=(18, 5, 5),
                        mats=[("simple", 5, (4, 4, 4), (0, 0, 0))], objects=[("block", 5, (14, 1, 1), (8, 10, 10))])


def _raster_bulk(shape, seed, ids):
    """Bulk ids (gz, gy, gx) drawn from `ids` (fractional values truncate,
    negative and unknown ones leave the background)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return rng.choice(np.array(ids, np.float32), size=shape)


# --- decks of the device rasteriser (no sheets, Drude poles or geometry
# output, so the ids are drawn on the GPU): a bulk file of random ids
# (unknown, negative and fractional values among them) under objects of
# every kind reaching the grid's faces and the periodic duplicate layer,
# overlapping one another, one with a material id the deck does not define
# (it keeps the previous object's material, ref :2101-2288).  Every object
# stays inside the grid: the reference writes cells outside it out of its
# arrays' bounds
DECKS["raster_pbc_x"] = dict(
    n=(40, 30, 34), steps=160, f="15E9", pulse=1, bc=(1, 1, 0, 0, 0, 0), excitation=("antenna", 1, 0, 1),
    ff=[(90, 0), (50, 100)], ffc=(20, 15, 17), bulk="ids.bin",
    mats=[("simple", 2, (2, 2, 2), (0.01, 0.01, 0.01)), ("simple", 3, (3, 2.5, 4), (0, 0, 0)),
          ("simple", 4, (1, 1, 1), ("1E8", "1E8", "1E8")), ("simple", 5, (1.5, 1.5, 1.5), (0.002, 0, 0))],
    objects=[("block", 3, (33, 3, 5), (9, 6, 6)), ("sphere", 5, (6, 12, 20), 5), ("sphere", 9, (30, 22, 10), 3),
             ("cylinder", 2, "x", (1, 8, 27), (41, 3)), ("cylinder", 3, "y", (28, 1, 6), (30, 2)),
             ("block", 4, (20, 15, 12), (1, 1, 5)), ("block", 4, (20, 15, 18), (1, 1, 5))],
    ports=[("basic", "z", 50, (20, 15, 17), (1, 1, 1))],
    _ext="geometry_bin no\n", _bulk=_raster_bulk((34, 30, 40), 11, [0, 0, 0, 2, 3, 3.7, 5, 9, -1]))
DECKS["raster_pbc_yz"] = dict(
    n=(40, 12, 14), dl=("0.5E-3", "0.5E-3", "0.5E-3"), steps=300, f="8E9", bc=(0, 0, 1, 1, 1, 1),
    excitation=("plane wave", 1, 0, 90, 0, 90), bulk="ids.bin",
    mats=[("simple", 2, (2, 2, 2), (0.01, 0.01, 0.01)), ("simple", 3, (3, 2.5, 4), (0, 0, 0)),
          ("simple", 5, (1.5, 1.5, 1.5), (0.002, 0, 0))],
    objects=[("sphere", 3, (20, 5, 8), 4), ("cylinder", 5, "z", (26, 10, 1), (15, 3)),
             ("block", 2, (30, 9, 10), (4, 5, 6)), ("cylinder", 3, "x", (6, 6, 7), (3, 0))],
    _ext="geometry_bin no\n", _bulk=_raster_bulk((14, 12, 40), 12, [0, 0, 2, 3, 5, 5.5, 7, -3]))


def write_deck(name, directory, fname="inputs.txt"):
    """Write deck `name` (and its sidecar / bulk geometry file, if any) into
    `directory`; returns (path, kmax)."""
    d = DECKS[name]
    path = os.path.join(directory, fname)
    with open(path, "w") as f:
        f.write(deck_text(d))
    if "_ext" in d:
        with open(path + ".b200", "w") as f:
            f.write(d["_ext"])
    if "_bulk" in d:
        d["_bulk"].tofile(os.path.join(directory, d["bulk"]))
    for fn, data in d.get("_files", {}).items():
        with open(os.path.join(directory, fn), "wb") as f:
            f.write(data)
    return path, bool(d.get("kmax"))
