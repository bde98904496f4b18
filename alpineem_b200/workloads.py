"""Synthetic workloads in the reference's input grammar.

The reference ships no benchmark decks; these builders generate the
throughput workloads from seeded random draws, as decks for
alpineem_b200.deck plus a bulk-geometry array (the contents of the
reference's optional_geom_bulk.bin, main_fdtd/fdtd_solver.f90:2051-2095:
float32 material ids, x fastest).
"""
import numpy as np


def _ellipsoids(bulk, n_ell, rng, semi, eps_range, lo, hi, first_id):
    """Rasterise axis-aligned ellipsoids into `bulk` (shape (nz, ny, nx)).
    Cell (i, j, k) (1-based) is inside when its centre (i-0.5, ...) lies in
    the ellipsoid.  Returns the material list entries."""
    nz, ny, nx = bulk.shape
    mats = []
    for e in range(n_ell):
        mid = first_id + e
        eps = float(rng.uniform(*eps_range))
        ax = rng.uniform(semi[0], semi[1], size=3)  # semi-axes x, y, z in cells
        c = np.array([rng.uniform(lo[a], hi[a]) for a in range(3)])
        mats.append(("simple", mid, (eps, eps, eps), (0, 0, 0)))
        b0 = [max(1, int(np.floor(c[a] - ax[a]))) for a in range(3)]
        b1 = [min((nx, ny, nz)[a], int(np.ceil(c[a] + ax[a])) + 1) for a in range(3)]
        i = np.arange(b0[0], b1[0] + 1) - 0.5
        j = np.arange(b0[1], b1[1] + 1) - 0.5
        k = np.arange(b0[2], b1[2] + 1) - 0.5
        r = (((k[:, None, None] - c[2]) / ax[2]) ** 2 + ((j[None, :, None] - c[1]) / ax[1]) ** 2 +
             ((i[None, None, :] - c[0]) / ax[0]) ** 2)
        sl = bulk[b0[2] - 1:b1[2], b0[1] - 1:b1[1], b0[0] - 1:b1[0]]
        sl[r <= 1.0] = mid
    return mats


def dipole_ellipsoids(n=1024, steps=4000, n_ell=64, seed=2, pml_cells=16, dl="2E-3", f="5E9",
                      theta_step=10, phi_step=10, arm=30, semi=(5, 40)):
    """Large single-GPU throughput run: an n^3 grid (spacing dl) with
    `pml_cells` of CPML on every face, a z-directed dipole of two 1x1x`arm`
    PEC arms around a 1-cell 50-ohm basic lumped port driven by a Gaussian
    pulse, `n_ell` dielectric ellipsoids (eps_r ~ U[2,12], semi-axes ~
    U[semi] cells scaled by n/1024, centres ~ U over the interior, numpy
    default_rng(seed)), and time-domain far fields on a theta_step x
    phi_step degree grid (theta 0..180, phi 0..360-phi_step).

    Returns (deck, ext_text, bulk): the deck as a dict for
    alpineem_b200.deck.deck_text, the extension lines, and bulk of shape
    (n, n, n) float32.
    """
    rng = np.random.default_rng(seed)
    scale = n / 1024.0
    bulk = np.zeros((n, n, n), np.float32)
    lo = [pml_cells + 4] * 3
    hi = [n - pml_cells - 4] * 3
    mats = [("simple", 1, (1, 1, 1), ("1E8", "1E8", "1E8"))]
    mats += _ellipsoids(bulk, n_ell, rng, (semi[0] * scale, semi[1] * scale), (2.0, 12.0), lo, hi, first_id=2)
    c = n // 2
    arm = max(1, min(arm, c - pml_cells - 3))
    ff = [(t, p) for t in range(0, 181, theta_step) for p in range(0, 360, phi_step)]
    d = dict(n=(n, n, n), dl=(dl, dl, dl), steps=steps, factor=1, f=f, pulse=1, bc=(0, 0, 0, 0, 0, 0),
             excitation=("antenna", 1, 0, 1), ff=ff, ffc=(c, c, c), name="data.dat", mats=mats,
             bulk="optional_geom_bulk.bin",
             objects=[("block", 1, (c, c, c - arm), (1, 1, arm)), ("block", 1, (c, c, c + 1), (1, 1, arm))],
             ports=[("basic", "z", 50, (c, c, c), (1, 1, 1))])
    # port S11 spectra on the fly at 512 frequencies over the Gaussian
    # pulse's band (post-processor bounds 0 .. 2.146 f)
    ext = "pml_cells %d\ngeometry_bin no\ndft_freqs 1e8 %.6g 512\n" % (pml_cells, 2.146 * float(f))
    return d, ext, bulk


# CPML profile of the scattering and layered-slab configurations: cubic
# grading, sigma_max = 0.8 (m+1) / (eta0 d), kappa_max = 1, alpha from 0.05
# at the inner edge to 0 at the outer wall (the reference's direction)
BASELINE_CPML = "cpml_grading 3 0.8 1 0.05\n"


def pec_sphere(n=96, steps=2000, radius=20, inset=15, seed=0, n_probes=3, dl="5E-3", f="1E9",
               theta_step=5, factor=0.98 / 0.99):
    """PEC-sphere scattering: an n^3 grid of `dl` cells with 10 cells of
    CPML on every face (BASELINE_CPML profile), the TF/SF box `inset` cells
    in from every edge, an x-polarised differentiated-Gaussian plane wave
    travelling +z (theta = 0, pol = 270 deg), a PEC sphere (sigma = 1e8, the
    reference's encoding of a metal volume) of `radius` cells at the grid
    centre, time-domain far fields at theta = 0..180 in `theta_step` degree
    steps at phi = 0, and `n_probes` point probes drawn with numpy
    default_rng(seed) in the scattered-field region (between the CPML and
    the TF/SF box).  factor = 0.98/0.99 turns the reference's Courant number
    0.98/sqrt(3) into 0.99/sqrt(3).  With f = 1 GHz the post-processor's
    band of a differentiated Gaussian (0.183 f .. 3.087 f) is
    0.18 .. 3.09 GHz.

    Returns (deck, ext_text, probes) with probes a list of (i, j, k)."""
    rng = np.random.default_rng(seed)
    npml = 11  # 10 cells of CPML: the reference's npml = cells + 1
    N = n + 1
    lo, hi = inset, N - inset
    probes = []
    while len(probes) < n_probes:
        p = tuple(int(v) for v in rng.integers(npml + 1, N - npml - 1, size=3))
        if all(lo <= v <= hi for v in p):
            continue  # inside the total-field box
        probes.append(p)
    c = n // 2
    ff = [(t, 0) for t in range(0, 181, theta_step)]
    d = dict(n=(n, n, n), dl=(dl, dl, dl), steps=steps, factor=repr(factor), f=f, pulse=2, bc=(0, 0, 0, 0, 0, 0),
             excitation=("plane wave", 1, 0, 0, 0, 270), ff=ff, ffc=(c, c, c), name="data.dat",
             mats=[("simple", 1, (1, 1, 1), ("1E8", "1E8", "1E8"))],
             objects=[("sphere", 1, (c, c, c), radius)])
    ext = BASELINE_CPML + "tfsf_inset %d\n" % inset + "".join("probe %d %d %d\n" % p for p in probes)
    return d, ext, probes


def layered_slab(nxy=128, nz=512, steps=8000, seed=1, n_layers=8, pml_cells=12, dl="1E-3", f="10E9", n_freqs=256,
                 z0=60):
    """Dispersive, anisotropic layered slab with a thin sheet: an nxy x nxy
    x nz unit cell of `dl` cells, periodic in x and y, `pml_cells` of CPML
    on both z faces (BASELINE_CPML profile), a normally incident
    x-polarised differentiated-Gaussian plane wave travelling +z.  From
    z = z0 up: `n_layers` dielectric layers (thickness ~ U{8..40} cells,
    diagonal eps_r with every axis ~ U[1, 10], sigma ~ U[0, 0.05] S/m,
    numpy default_rng(seed)), then one 2-pole Drude layer (omega_p ~
    U[1e10, 5e10] rad/s, gamma ~ U[1e8, 1e10] 1/s, same generator), and a
    Smith-Maloney sheet of 100 S (0.01 ohm/sq) on the top face of the
    first layer.  The reflected and transmitted plane sums are recorded
    every step and their spectra accumulated on the fly at `n_freqs`
    frequencies from 1 to 30 GHz.  With f = 10 GHz the post-processor's
    band of the pulse is 1.83 .. 30.9 GHz.

    Returns (deck, ext_text, layers) with layers a list of
    (z_start, thickness, material id)."""
    rng = np.random.default_rng(seed)
    mats, objects, layers = [], [], []
    z = z0
    for q in range(n_layers):
        t = int(rng.integers(8, 41))
        eps = tuple(float(v) for v in rng.uniform(1.0, 10.0, size=3))
        sig = float(rng.uniform(0.0, 0.05))
        mid = 2 + q
        mats.append(("simple", mid, tuple("%.6f" % v for v in eps), ("%.6f" % sig,) * 3))
        objects.append(("block", mid, (1, 1, z), (nxy, nxy, t)))
        layers.append((z, t, mid))
        z += t
    t = int(rng.integers(8, 41))
    poles = [("%.6E" % rng.uniform(1e10, 5e10), "%.6E" % rng.uniform(1e8, 1e10)) for _ in range(2)]
    mid = 2 + n_layers
    mats.append(("plasma", mid, (1, 1, 1), (0, 0, 0), poles))
    objects.append(("block", mid, (1, 1, z), (nxy, nxy, t)))
    layers.append((z, t, mid))
    z += t
    if z >= nz - pml_cells - 6:
        raise ValueError("the layer stack reaches the CPML; enlarge nz")
    sheet_z = layers[0][0] + layers[0][1]
    mats.append(("sheet", 1, "0.01"))
    d = dict(n=(nxy, nxy, nz), dl=(dl, dl, dl), steps=steps, factor=1, f=f, pulse=2, bc=(1, 1, 1, 1, 0, 0),
             excitation=("plane wave", 1, 0, 0, 0, 270), name="data.dat", mats=mats, objects=objects,
             sheets=[("z", 1, sheet_z, (1, 1), (nxy, nxy))])
    ext = BASELINE_CPML + "pml_cells %d\ndft_freqs 1e9 3e10 %d\n" % (pml_cells, n_freqs)
    return d, ext, layers


# sidecar extension of every kmax_batch instance: on-the-fly spectra of the
# TE/TM reflected and transmitted plane sums at 128 frequencies
KMAX_BATCH_EXT = "dft_freqs 2e9 1.8e10 128\n"


def kmax_batch(n_inst=64, steps=6000, seed=3, dl="1E-3", f="10E9", nxy=64, depth=10, patch=16):
    """Batched constant-k unit cells (the fan-out that
    utility_scripts/parallel_kmax.py runs as separate processes): n_inst decks
    of nxy x nxy x Z cells, periodic in x and y with CPML on z, Z drawn from
    {128, 192, 256, 384, 512} (numpy default_rng(seed)).  Instance q has
    incidence theta = 2.5 * (q // 2) degrees in the x-z plane, TE for even q
    and TM for odd q, k1 = 2 pi f sin(theta) / c, k2 = 0.  Every cell holds a
    `depth`-cell eps_r = 3, sigma = 0.002 slab under a 0-ohm (PEC) sheet
    drawn from a patch x patch binary pattern (fill 0.5, the same seed), runs
    of set pixels merged into sheet rectangles.  Returns a list of deck
    dicts for alpineem_b200.deck.deck_text (kmax)."""
    rng = np.random.default_rng(seed)
    zs = rng.choice([128, 192, 256, 384, 512], size=n_inst)
    bits = rng.random((patch, patch)) < 0.5
    cell = nxy // patch
    sheets = []
    for r in range(patch):
        c = 0
        while c < patch:
            if not bits[r, c]:
                c += 1
                continue
            c1 = c
            while c1 < patch and bits[r, c1]:
                c1 += 1
            sheets.append((c * cell + 1, r * cell + 1, (c1 - c) * cell, cell))
            c = c1
    fval = float(f)
    decks_ = []
    for q in range(n_inst):
        Z = int(zs[q])
        theta = np.deg2rad(2.5 * (q // 2))
        k1 = 2.0 * np.pi * fval * np.sin(theta) / 299792458.0
        z0 = Z // 2 - depth // 2
        d = dict(kmax=True, n=(nxy, nxy, Z), dl=(dl, dl, dl), steps=steps, f=f, pulse=2, bc=(1, 1, 1, 1, 0, 0),
                 excitation=("plane wave", 1, 0, "TE" if q % 2 == 0 else "TM", "+"), k=("%.6f" % k1, "0.0"),
                 name="data.dat",
                 mats=[("simple", 2, (3, 3, 3), (0.002, 0.002, 0.002)), ("sheet", 3, 0)],
                 objects=[("block", 2, (1, 1, z0), (nxy, nxy, depth))],
                 sheets=[("z", 3, z0 + depth, (a, b), (sa, sb)) for a, b, sa, sb in sheets])
        decks_.append(d)
    return decks_


def adjoint_probe(n=192, steps=3000, design=(64, 64, 32), seed=4, pml_cells=12, dl="1E-3", f="20E9",
                  freq=10e9, gap=40, arm=10, port_z=None):
    """Design-gradient workload: an n^3 grid (spacing dl, `pml_cells` of
    CPML on every face) driven by a z-directed 1-cell 50-ohm lumped port
    (Gaussian pulse) between two 1x1x`arm` PEC arms near the -z side, a
    design box of `design` cells (x, y, z) centred in x and y above it whose
    eps_r is drawn from U[1, 4] (numpy default_rng(seed)), and an Ez probe
    `gap` cells beyond the box's +z face on the axis.  The figure of merit is
    |DFT of the probe at `freq`|^2.

    Returns (deck, ext_text, lo, n, probe, freq, eps) with eps of shape
    (nz, ny, nx) float32 and probe = (comp, i, j, k)."""
    rng = np.random.default_rng(seed)
    c = n // 2
    nx, ny, nz = design
    lo = (c - nx // 2 + 1, c - ny // 2 + 1, 0)
    pz = port_z if port_z is not None else pml_cells + arm + 8
    z0 = pz + arm + 1 + max(4, (n - 2 * pml_cells - nz - gap) // 4 - arm)
    lo = (lo[0], lo[1], z0)
    probe = (2, c, c, z0 + nz - 1 + gap)
    if probe[3] >= n + 1 - pml_cells - 1:
        raise ValueError("the probe falls into the CPML; enlarge n or shrink the gap")
    eps = rng.uniform(1.0, 4.0, size=(nz, ny, nx)).astype(np.float32)
    d = dict(n=(n, n, n), dl=(dl, dl, dl), steps=steps, factor=1, f=f, pulse=1, bc=(0, 0, 0, 0, 0, 0),
             excitation=("antenna", 1, 0, 1), name="data.dat",
             mats=[("simple", 1, (1, 1, 1), ("1E8", "1E8", "1E8"))],
             objects=[("block", 1, (c, c, pz - arm), (1, 1, arm)), ("block", 1, (c, c, pz + 1), (1, 1, arm))],
             ports=[("basic", "z", 50, (c, c, pz), (1, 1, 1))])
    ext = "pml_cells %d\ngeometry_bin no\n" % pml_cells
    return d, ext, lo, design, probe, float(freq), eps
