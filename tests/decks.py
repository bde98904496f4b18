"""Small input decks in the reference's positional grammar
(main_fdtd/fdtd_solver.f90:726-1298; template main_fdtd/master.py:51-296),
one per solver feature, sized so the CPU oracle finishes each in seconds.
Used by the GPU parity tests and smoke()."""
import os


def deck_text(d):
    L = []
    w = L.append
    w("%d,%d,%d" % tuple(d["n"]))
    w("%s,%s,%s" % tuple(d.get("dl", ("1E-3", "1E-3", "1E-3"))))
    w(str(d["steps"]))
    w(str(d.get("factor", 1)))
    w(str(d.get("f", "10E9")))
    w(str(d.get("pulse", 2)))
    w(",".join(str(b) for b in d.get("bc", (0, 0, 0, 0, 0, 0))))
    if "igp" in d:
        w("IGP")
        w(d["igp"][0])
        w(str(d["igp"][1]))
    else:
        w("none")
    ex = d["excitation"]
    if ex[0] == "plane wave":
        w("plane wave")
        w("%s,%s" % (ex[1], ex[2]))
        if d.get("kmax"):
            w(ex[3])  # TE / TM
            w(ex[4])  # + / -
        else:
            w("%s,%s,%s" % tuple(ex[3:6]))
    else:
        w("antenna")
        w("%s,%s" % (ex[1], ex[2]))
        w(str(ex[3]))
    if d.get("kmax"):
        w("%s,%s" % tuple(d["k"]))
    ff = d.get("ff", [])
    w(str(len(ff)))
    if ff:
        w("%d,%d,%d" % tuple(d["ffc"]))
        for t, p in ff:
            w("%s,%s" % (t, p))
    if "video" in d:
        w("yes")
        w(d["video"][0])
        w(str(d["video"][1]))
    else:
        w("no")
    w(d.get("full", "no"))
    w(d.get("name", "data.dat"))
    mats = d.get("mats", [])
    w(str(len(mats)))
    for m in mats:
        if m[0] == "sheet":
            w("sheet")
            w(str(m[1]))
            w(str(m[2]))
        else:
            w("volume")
            w(m[0])  # simple / plasma
            w(str(m[1]))
            w("%s,%s,%s" % tuple(m[2]))
            w("%s,%s,%s" % tuple(m[3]))
            if m[0] == "plasma":
                w(str(len(m[4])))
                for wp, gm in m[4]:
                    w("%s,%s,%s" % (wp, wp, wp))
                    w("%s,%s,%s" % (gm, gm, gm))
    if "bulk" in d:
        w("yes")
        w(d["bulk"])
    else:
        w("no")
    objs = d.get("objects", [])
    w(str(len(objs)))
    for o in objs:
        w(o[0])
        w(str(o[1]))
        if o[0] == "block":
            w("%d,%d,%d" % tuple(o[2]))
            w("%d,%d,%d" % tuple(o[3]))
        elif o[0] == "sphere":
            w("%d,%d,%d" % tuple(o[2]))
            w(str(o[3]))
        else:
            w(o[2])
            w("%d,%d,%d" % tuple(o[3]))
            w("%d,%d" % tuple(o[4]))
    sheets = d.get("sheets", [])
    w(str(len(sheets)))
    for s in sheets:
        w(s[0])
        w(str(s[1]))
        w(str(s[2]))
        w("%d,%d" % tuple(s[3]))
        w("%d,%d" % tuple(s[4]))
    ports = d.get("ports", [])
    w(str(len(ports)))
    for p in ports:
        w(p[0])
        w(p[1])
        w(str(p[2]))
        w("%d,%d,%d" % tuple(p[3]))
        if p[0] == "basic":
            w("%d,%d,%d" % tuple(p[4]))
        else:
            w("%d,%d" % tuple(p[4]))
            w(p[5])
    w("0")
    return "\n".join(L) + "\n"


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
    # constant-k periodic solver, TE and TM, oblique k in the y,z plane
    "kmax_te": dict(kmax=True, n=(36, 10, 10), dl=("0.25E-3", "0.25E-3", "0.25E-3"), steps=300, f="8E9", bc=(0, 0, 1, 1, 1, 1),
                    excitation=("plane wave", 1, 0, "TE", "+"), k=("300.0", "150.0"),
                    mats=[("simple", 5, (4, 4, 4), (0, 0, 0)), ("sheet", 7, 30)],
                    objects=[("block", 5, (14, 1, 1), (8, 10, 10))], sheets=[("x", 7, 14, (1, 1), (10, 10))]),
    "kmax_tm": dict(kmax=True, n=(36, 10, 10), dl=("0.25E-3", "0.25E-3", "0.25E-3"), steps=300, f="8E9", bc=(0, 0, 1, 1, 1, 1),
                    excitation=("plane wave", 1, 0, "TM", "-"), k=("0.0", "250.0"),
                    mats=[("simple", 5, (4, 4, 4), (0.02, 0.02, 0.02))],
                    objects=[("block", 5, (14, 1, 1), (8, 10, 10))]),
}


def write_deck(name, directory, fname="inputs.txt"):
    d = DECKS[name]
    path = os.path.join(directory, fname)
    with open(path, "w") as f:
        f.write(deck_text(d))
    return path, bool(d.get("kmax"))
