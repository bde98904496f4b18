"""Design gradients: dF/d(eps_r, sigma) for every cell of a design box, with
F = |D|^2 and D = sum_n c^n exp(-i 2 pi f n dt) the single-frequency DFT of
one probe E component over the run.

The reference's optimisation workflow
(optimization_scripts/adjoint_optimization/adjoint_optimization.py:55-134)
runs the solver once forward and once with a rescaled, delayed source, and
forms per-material gradients from the overlap of the two runs' field
spectra.  Here the library computes the exact derivative of the discrete
time loop: a forward run with checkpoints, then the transposed update run
backwards in time, recomputing each checkpoint segment (aem_design_* in
include/alpineem_b200.h).  `DesignFoM` wraps the pair as a
torch.autograd.Function, so a design tensor's .grad is dF/d eps_r per cell.

Arrays are (nz, ny, nx) over the design box, x fastest, like the
reference's Fortran (x, y, z) order read in C.
"""
import ctypes

import numpy as np

from . import AemError, load_library

PRECISION = {32: 4, 64: 8}


def _ptr(a):
    """(pointer, keep-alive) for a float32 numpy array or CUDA tensor."""
    if a is None:
        return None, None
    try:
        import torch
        if isinstance(a, torch.Tensor):
            if a.dtype != torch.float32:
                raise ValueError("design arrays must be float32")
            a = a.contiguous()
            if a.is_cuda:
                torch.cuda.current_stream(a.device).synchronize()
            return a.data_ptr(), a
    except ImportError:
        pass
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.ctypes.data, a


class Design:
    """A design-gradient run over the deck at `inputs_path`.

    lo, n     : design box, cells lo..lo+n-1 (reference indices, x, y, z)
    probe     : (comp, i, j, k), comp 0/1/2 = Ex/Ey/Ez at reference edge i, j, k
    freq      : DFT frequency (Hz)
    precision : 32 (the reference's FP32 arithmetic) or 64 (FP64 state, for
                finite-difference checks)
    """

    def __init__(self, inputs_path, lo, n, probe, freq, precision=32, outdir=None):
        self._lib = load_library()
        self._h = ctypes.c_void_p()
        i3 = ctypes.c_int * 3
        rc = self._lib.aem_design_create(str(inputs_path).encode(), outdir.encode() if outdir else None,
                                         i3(*lo), i3(*n), PRECISION[precision], ctypes.byref(self._h))
        if rc != 0:
            raise AemError(self._lib.aem_design_last_error(None).decode())
        self.lo, self.n = tuple(lo), tuple(n)
        self.shape = (n[2], n[1], n[0])
        self.precision = precision
        comp, i, j, k = probe
        self._check(self._lib.aem_design_set_probe(self._h, int(comp), int(i), int(j), int(k), float(freq)))

    def _check(self, rc):
        if rc != 0:
            raise AemError(self._lib.aem_design_last_error(self._h).decode())

    def set_design(self, eps, sigma=None):
        """Per-cell eps_r (and sigma in S/m, None: the deck's materials):
        float32 arrays or CUDA tensors of shape (nz, ny, nx)."""
        if tuple(eps.shape) != self.shape or (sigma is not None and tuple(sigma.shape) != self.shape):
            raise ValueError("design arrays must have shape %s" % (self.shape,))
        pe, ke = _ptr(eps)
        ps, ks = _ptr(sigma)
        self._check(self._lib.aem_design_set_eps(self._h, pe, ps))
        del ke, ks

    def forward(self, checkpoint_every=200):
        """Run all steps; returns (F, D).  checkpoint_every < 1: plain run
        (no gradient afterwards)."""
        f = ctypes.c_double()
        d = (ctypes.c_double * 2)()
        self._check(self._lib.aem_design_forward(self._h, int(checkpoint_every), ctypes.byref(f), d))
        return f.value, complex(d[0], d[1])

    def gradient(self, scale=1.0, sigma=False, out=None):
        """scale * dF/d eps_r per design cell (and dF/d sigma when `sigma`),
        as float32 numpy arrays, or into `out` (CUDA tensor, or a pair of
        them with sigma) without a host copy."""
        if out is not None:
            outs = out if isinstance(out, (tuple, list)) else (out, None)
            for t in outs:
                if t is not None and (tuple(t.shape) != self.shape or not t.is_contiguous()):
                    raise ValueError("gradient outputs must be contiguous with shape %s" % (self.shape,))
            self._check(self._lib.aem_design_gradient(self._h, outs[0].data_ptr() if outs[0] is not None else None,
                                                      outs[1].data_ptr() if outs[1] is not None else None,
                                                      float(scale)))
            return out
        ge = np.empty(self.shape, np.float32)
        gs = np.empty(self.shape, np.float32) if sigma else None
        self._check(self._lib.aem_design_gradient(self._h, ge.ctypes.data, gs.ctypes.data if sigma else None,
                                                  float(scale)))
        return (ge, gs) if sigma else ge

    def set_overlap(self, enable=True):
        """Keep the spectra at the probe frequency of the forward E and of
        the adjoint field on the design edges during gradient(), for
        gradient_overlap()."""
        self._check(self._lib.aem_design_set_overlap(self._h, 1 if enable else 0))

    def gradient_overlap(self, scale=1.0):
        """(dF/d eps_r, dF/d sigma) per design cell estimated from the two
        spectra of the last gradient() alone: the frequency-domain overlap
        of the reference's adjoint_optimization.py:121-134, restated for
        this engine's adjoint field (a tone at the probe frequency assumed).
        A consistency check on gradient(), not a replacement for it."""
        ge = np.empty(self.shape, np.float32)
        gs = np.empty(self.shape, np.float32)
        self._check(self._lib.aem_design_gradient_overlap(self._h, ge.ctypes.data, gs.ctypes.data, float(scale)))
        return ge, gs

    def timing(self):
        """(forward ms, gradient ms, forward launches, gradient launches) of
        the last calls, from CUDA events on the run's stream."""
        ms = (ctypes.c_double * 2)()
        n = (ctypes.c_longlong * 2)()
        self._check(self._lib.aem_design_timing(self._h, ms, n))
        return ms[0], ms[1], n[0], n[1]

    def field(self, name):
        """A field component (Ex..Hz) of the current forward state, reference
        layout, as a float64 array (nz, ny, nx)."""
        comp = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"].index(name)
        dims = (ctypes.c_int * 3)()
        self._check(self._lib.aem_design_get_field(self._h, comp, dims, None))
        out = np.empty(dims[0] * dims[1] * dims[2], np.float64)
        self._check(self._lib.aem_design_get_field(self._h, comp, dims, out.ctypes.data))
        return out.reshape(dims[2], dims[1], dims[0])

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.aem_design_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _function():
    import torch

    class DesignFoM(torch.autograd.Function):
        """F(eps) of a Design as an autograd node: forward runs the
        checkpointed forward pass, backward the adjoint sweep; the gradient
        is written straight into a CUDA tensor.  A Design holds one forward
        state: call backward before the next forward on the same Design."""

        @staticmethod
        def forward(ctx, eps, design, checkpoint_every):
            design.set_design(eps.detach())
            f, _ = design.forward(checkpoint_every)
            ctx.design = design
            ctx.like = eps
            return torch.tensor(f, dtype=torch.float64, device=eps.device)

        @staticmethod
        def backward(ctx, g):
            eps = ctx.like
            grad = torch.empty(eps.shape, dtype=torch.float32, device=eps.device)
            scale = float(g.item())
            if eps.is_cuda:
                ctx.design.gradient(scale=scale, out=grad)
            else:
                grad.copy_(torch.from_numpy(ctx.design.gradient(scale=scale)))
            return grad.to(eps.dtype), None, None

    return DesignFoM


def fom(design, eps, checkpoint_every=200):
    """F as a differentiable function of the design tensor `eps`."""
    return _function().apply(eps, design, checkpoint_every)
