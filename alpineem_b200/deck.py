"""Input decks in the reference's positional grammar
(main_fdtd/fdtd_solver.f90:726-1298; the annotated template that master.py
fills is main_fdtd/master.py:51-296), written from a plain dict so callers
and tests can build decks without string templates.

Keys of the dict (all lists/tuples in the reference's order):
  n (nx,ny,nz), dl (dx,dy,dz), steps, factor, f, pulse, bc (6 flags),
  igp (wall, index), excitation ("plane wave", amp, delay, theta, phi, pol)
  or ("antenna", amp, delay, port#) [kmax: ("plane wave", amp, delay,
  "TE"/"TM", "+"/"-")], kmax (bool), k (k1, k2), ff [(theta, phi)...],
  ffc (ic,jc,kc), video (axis, index), full, name, mats, bulk (file name),
  objects, sheets, ports.
"""


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
