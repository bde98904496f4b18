"""Design gradients (aem_design_*): the forward pass against the solver, the
adjoint gradient against central finite differences, checkpoint segments,
the torch.autograd wrapper, and the frequency-domain overlap estimate of
the reference's workflow as a consistency check.

The workload is alpineem_b200.workloads.adjoint_probe at 48^3 (6-cell CPML,
300 steps, a 10x10x6 design box of eps_r ~ U[1, 4], an Ez probe 8 cells
beyond it, figure of merit |DFT_10GHz(Ez)|^2).  Finite differences use the
FP64 build of the same kernels with delta = 1e-3, as the gradient check
asks; one FP64 forward pass per perturbed cell and sign.

Tolerances: the FP64 adjoint is the exact derivative of the FP64 loop, so
it meets central differences to the difference's own truncation (measured
~1e-7; bound 1e-5).  The FP32 adjoint of the FP32 loop (the reference's
arithmetic) meets them to 1e-3 relative, the north-star tolerance, on every
cell whose derivative is above 1 % of the largest checked one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FD_DELTA = 1e-3


def _setup(tmp_path, **kw):
    from alpineem_b200 import workloads
    from alpineem_b200.deck import deck_text
    args = dict(n=48, steps=300, design=(10, 10, 6), pml_cells=6, gap=8, arm=4)
    args.update(kw)
    d, ext, lo, n, probe, freq, eps = workloads.adjoint_probe(**args)
    path = tmp_path / "inputs.txt"
    path.write_text(deck_text(d))
    (tmp_path / "inputs.txt.b200").write_text(ext)
    return str(path), lo, n, probe, freq, eps


def _design(path, lo, n, probe, freq, precision):
    from alpineem_b200.adjoint import Design
    return Design(path, lo, n, probe, freq, precision=precision)


def test_forward_equals_solver(tmp_path, gpu_lib, monkeypatch):
    """With the deck's own material (vacuum) in the design box, the FP32
    forward pass reproduces the two-kernel solver's fields bit for bit."""
    import alpineem_b200 as ab
    path, lo, n, probe, freq, eps = _setup(tmp_path)
    monkeypatch.setenv("AEM_TWO_KERNEL", "1")
    with ab.Simulation(path, outdir=str(tmp_path)) as sim:
        sim.run(sim.steps[1])
        sim.synchronize()
        ref = {c: sim.field(c) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    with _design(path, lo, n, probe, freq, 32) as d:
        d.set_design(np.ones_like(eps))
        d.forward(0)
        for c, r in ref.items():
            g = d.field(c)
            assert g.shape == r.shape
            assert np.array_equal(g, r), "%s differs (max %.3g)" % (c, np.abs(g - r).max())


def _fd(d64, eps, cells, sigma=None, which="eps"):
    """Central differences; the step is the one the float32 design values
    actually take (x +- 1e-3 rounds to a whole number of float32 ulps)."""
    out = []
    for (z, y, x) in cells:
        vals, pts = [], []
        for sgn in (1, -1):
            e = eps.copy()
            s = None if sigma is None else sigma.copy()
            a = e if which == "eps" else s
            a[z, y, x] = np.float32(float(a[z, y, x]) + sgn * FD_DELTA)
            pts.append(float(a[z, y, x]))
            d64.set_design(e, s)
            vals.append(d64.forward(0)[0])
        out.append((vals[0] - vals[1]) / (pts[0] - pts[1]))
    return np.array(out)


def _cells(n, count, seed):
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(0, n[2])), int(rng.integers(0, n[1])), int(rng.integers(0, n[0]))) for _ in range(count)]


def test_gradient_matches_finite_differences(tmp_path, gpu_lib):
    path, lo, n, probe, freq, eps = _setup(tmp_path)
    cells = _cells(n, 8, 11)
    with _design(path, lo, n, probe, freq, 64) as d64, _design(path, lo, n, probe, freq, 32) as d32:
        fd = _fd(d64, eps, cells)
        d64.set_design(eps)
        f64, _ = d64.forward(50)
        g64 = d64.gradient()
        d32.set_design(eps)
        f32, _ = d32.forward(50)
        g32 = d32.gradient()
    assert abs(f32 - f64) <= 1e-3 * abs(f64)
    a64 = np.array([g64[c] for c in cells])
    a32 = np.array([g32[c] for c in cells])
    scale = np.abs(fd).max()
    assert scale > 0
    err64 = np.abs(a64 - fd) / np.maximum(np.abs(fd), 1e-2 * scale)
    err32 = np.abs(a32 - fd) / np.maximum(np.abs(fd), 1e-2 * scale)
    assert err64.max() <= 1e-5, (err64, fd, a64)
    assert err32.max() <= 1e-3, (err32, fd, a32)


def test_sigma_gradient_matches_finite_differences(tmp_path, gpu_lib):
    path, lo, n, probe, freq, eps = _setup(tmp_path)
    sigma = np.random.default_rng(5).uniform(0.0, 0.5, size=eps.shape).astype(np.float32)
    cells = _cells(n, 4, 12)
    with _design(path, lo, n, probe, freq, 64) as d64:
        fde = _fd(d64, eps, cells, sigma, "eps")
        fds = _fd(d64, eps, cells, sigma, "sig")
        d64.set_design(eps, sigma)
        d64.forward(64)
        ge, gs = d64.gradient(sigma=True)
    for fd, g in ((fde, ge), (fds, gs)):
        a = np.array([g[c] for c in cells])
        scale = np.abs(fd).max()
        err = np.abs(a - fd) / np.maximum(np.abs(fd), 1e-2 * scale)
        assert err.max() <= 1e-5, (err, fd, a)


def test_checkpoint_segments_do_not_change_the_gradient(tmp_path, gpu_lib):
    """Store-everything (one segment), even and uneven segments: the
    recomputed segments replay the forward pass bit for bit, so the
    gradients are identical."""
    path, lo, n, probe, freq, eps = _setup(tmp_path)
    with _design(path, lo, n, probe, freq, 32) as d:
        d.set_design(eps)
        grads = []
        for k in (300, 50, 7):
            d.forward(k)
            grads.append(d.gradient())
        # a second gradient from the same forward pass recomputes the last
        # segment too
        grads.append(d.gradient())
    for g in grads[1:]:
        assert np.array_equal(g, grads[0])


# The reference's gradient (adjoint_optimization.py:121-134) is the overlap
# at one frequency of the spectra of a forward and an adjoint run.  Restated
# for this engine it estimates the gradient from the DFTs at the probe
# frequency of the forward E and of the adjoint field alone, assuming the
# adjoint field is a tone there.  Measured on a B200 against the exact
# gradient (rel. L2 over the design cells, eps / sigma): 300 steps 4.1e-2 /
# 5.6e-2, 1000 steps 1.5e-2 / 0.14, 2000 steps 5.3e-3 / 0.12, 3000 steps
# 5.1e-3 / 2.8e-2 (correlation 0.99999); the estimate approaches the exact
# gradient as the window grows and the forward pulse has decayed.
OVERLAP_TOL_EPS = 1e-2
OVERLAP_TOL_SIGMA = 5e-2


def test_overlap_estimate_agrees_with_gradient(tmp_path, gpu_lib):
    path, lo, n, probe, freq, eps = _setup(tmp_path, steps=3000)
    with _design(path, lo, n, probe, freq, 32) as d:
        d.set_design(eps)
        d.set_overlap(True)
        d.forward(200)
        ge, gs = d.gradient(sigma=True)
        oe, os_ = d.gradient_overlap()
    rel_e = np.linalg.norm(oe - ge) / np.linalg.norm(ge)
    rel_s = np.linalg.norm(os_ - gs) / np.linalg.norm(gs)
    assert rel_e <= OVERLAP_TOL_EPS, rel_e
    assert rel_s <= OVERLAP_TOL_SIGMA, rel_s
    assert np.corrcoef(oe.ravel(), ge.ravel())[0, 1] > 0.9999


def test_overlap_needs_enabling(tmp_path, gpu_lib):
    import alpineem_b200 as ab
    path, lo, n, probe, freq, eps = _setup(tmp_path)
    with _design(path, lo, n, probe, freq, 32) as d:
        d.set_design(eps)
        d.forward(100)
        g = d.gradient()
        with pytest.raises(ab.AemError, match="overlap"):
            d.gradient_overlap()
        # the check leaves the gradient itself unchanged
        d.set_overlap(True)
        d.forward(100)
        assert np.array_equal(d.gradient(), g)


def test_autograd_function(tmp_path, gpu_lib):
    import torch
    from alpineem_b200.adjoint import fom
    path, lo, n, probe, freq, eps = _setup(tmp_path)
    with _design(path, lo, n, probe, freq, 32) as d:
        x = torch.tensor(eps, device="cuda", requires_grad=True)
        f = fom(d, x, checkpoint_every=100)
        (2.0 * f).backward()
        d.set_design(eps)
        d.forward(100)
        g = d.gradient(scale=2.0)
    assert np.array_equal(x.grad.cpu().numpy(), g)


def test_rejected_layouts(tmp_path, gpu_lib):
    import alpineem_b200 as ab
    from alpineem_b200.adjoint import Design
    path, lo, n, probe, freq, eps = _setup(tmp_path)
    with pytest.raises(ab.AemError, match="CPML"):
        Design(path, (3, 20, 20), n, probe, freq)
    with pytest.raises(ab.AemError, match="design box"):
        Design(path, lo, n, (2, lo[0] + 2, lo[1] + 2, lo[2] + 2), freq)
