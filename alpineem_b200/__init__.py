"""alpineem_b200 -- B200 (sm_100a) implementation of AlpineEM's FDTD core.

The reference drives its solver as an executable: ``master.py`` writes a
positional ``inputs.txt`` and runs ``./<solver> inputs.txt``
(main_fdtd/master.py:438-441); ``post_processor.py`` then reads the
``<name>.dat`` it leaves behind.  This package offers the same solver as

* ``_lib/FDTD-B200`` -- drop-in executable (set ``solver='<path>/FDTD-B200'``
  in master.py; ``FDTD-B200-kmax`` or ``--kmax`` for the constant-k build);
* :class:`Simulation` -- the C ABI of ``libalpineem_b200.so`` through ctypes,
  for stepping a run and reading its series and fields from Python;
* :func:`run_deck` -- one call equivalent to the executable.

There is no CPU fallback: importing works without a GPU, but creating a
simulation needs the CUDA library and a device, and fails loudly otherwise.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libalpineem_b200.so")
EXE_PATH = os.path.join(_HERE, "_lib", "FDTD-B200")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "alpineem_b200.h")

STANDARD, KMAX = 0, 1
SERIES = {"incident": 0, "reflected": 1, "transmitted": 2, "reflected_tm": 3, "transmitted_tm": 4,
          "port_voltage": 5, "e_theta": 6, "e_phi": 7}
FIELDS = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5, "material": 6}
# per-step samples that aem_read_probe returns; "point" is the extension
# `probe i j k` (index 3 p + c: probe p, component c = Ex, Ey, Ez)
PROBE_KINDS = {"reflected": 1, "transmitted": 2, "reflected_tm": 3, "transmitted_tm": 4, "port_voltage": 5,
               "point": 6}

_lib = None


class AemError(RuntimeError):
    """A failing call of the solver library (message from aem_last_error)."""


class AemDiverged(AemError):
    """A run stopped by the watchdog (extension `watchdog K`): E or H holds a
    NaN or Inf."""


def load_library():
    """Load libalpineem_b200.so (built in-tree by alpineem_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libalpineem_b200.so is not built (%s); run `python alpineem_b200/build.py`" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    h = ctypes.c_void_p
    lib.aem_version.restype = ctypes.c_int
    lib.aem_create_from_file.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(h)]
    lib.aem_run.argtypes = [h, ctypes.c_int]
    lib.aem_run_graph.argtypes = [h, ctypes.c_int, ctypes.c_int]
    lib.aem_autotune.argtypes = [h, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.aem_run_batch.argtypes = [ctypes.POINTER(h), ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.aem_steps.argtypes = [h, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.aem_synchronize.argtypes = [h]
    lib.aem_write_outputs.argtypes = [h]
    lib.aem_get_series.argtypes = [h, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    lib.aem_get_field.argtypes = [h, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
    lib.aem_grid.argtypes = [h, ctypes.POINTER(ctypes.c_int)]
    lib.aem_device_bytes.argtypes = [h, ctypes.POINTER(ctypes.c_size_t)]
    lib.aem_last_error.argtypes = [h]
    lib.aem_last_error.restype = ctypes.c_char_p
    lib.aem_destroy.argtypes = [h]
    lib.aem_create_from_memory.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_size_t,
                                           ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(h)]
    lib.aem_check_deck.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.aem_read_probe.argtypes = [h, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.aem_time_step.argtypes = [h, ctypes.POINTER(ctypes.c_double)]
    lib.aem_checkpoint_save.argtypes = [h, ctypes.c_char_p]
    lib.aem_checkpoint_load.argtypes = [h, ctypes.c_char_p]
    lib.aem_read_spectrum.argtypes = [h, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.aem_profile.argtypes = [h, ctypes.c_int]
    lib.aem_profile_read.argtypes = [h, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
    lib.aem_launch_count.argtypes = [h, ctypes.POINTER(ctypes.c_longlong)]
    lib.aem_workload.argtypes = [h, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double)]
    lib.aem_far_field_size.argtypes = [h, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
    lib.aem_flush.argtypes = [h]
    lib.aem_dft.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                            ctypes.c_void_p, ctypes.c_void_p]
    lib.aem_stream.argtypes = [h, ctypes.POINTER(ctypes.c_void_p)]
    lib.aem_dft_batch.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_longlong, ctypes.c_double,
                                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lib.aem_transfer_bytes.argtypes = [h, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    i3 = ctypes.c_int * 3
    lib.aem_design_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i3, i3, ctypes.c_int, ctypes.POINTER(h)]
    lib.aem_design_set_probe.argtypes = [h, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
    lib.aem_design_set_eps.argtypes = [h, ctypes.c_void_p, ctypes.c_void_p]
    lib.aem_design_forward.argtypes = [h, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.aem_design_gradient.argtypes = [h, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    lib.aem_design_set_overlap.argtypes = [h, ctypes.c_int]
    lib.aem_design_gradient_overlap.argtypes = [h, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    lib.aem_design_timing.argtypes = [h, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
    lib.aem_design_get_field.argtypes = [h, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
    lib.aem_design_stream.argtypes = [h, ctypes.POINTER(ctypes.c_void_p)]
    lib.aem_design_last_error.argtypes = [h]
    lib.aem_design_last_error.restype = ctypes.c_char_p
    lib.aem_design_destroy.argtypes = [h]
    _lib = lib
    return lib


PHASES = ["update_h", "update_e", "ports", "ff_currents", "ff_bin", "taps", "yee", "other"]


def dft(x, dt, freqs, stream=0):
    """Spectrum of a device time series at the given frequencies:
    sum_m x[m] exp(-i 2 pi f m dt).  `x` is a CUDA float32 tensor, `freqs`
    a CUDA float64 tensor (Hz); returns a complex128 CUDA tensor.  Runs the
    library's kernels (aem_dft) on `stream` (default: the current stream)."""
    import torch
    lib = load_library()
    if x.dtype != torch.float32 or not x.is_cuda or freqs.dtype != torch.float64 or not freqs.is_cuda:
        raise ValueError("x must be a CUDA float32 tensor and freqs a CUDA float64 tensor")
    x, freqs = x.contiguous(), freqs.contiguous()
    out = torch.empty(2 * freqs.numel(), dtype=torch.float64, device=x.device)
    st = stream or torch.cuda.current_stream(x.device).cuda_stream
    rc = lib.aem_dft(x.data_ptr(), x.numel(), float(dt), freqs.data_ptr(), freqs.numel(), out.data_ptr(), st)
    if rc != 0:
        raise AemError(lib.aem_last_error(None).decode())
    return torch.view_as_complex(out.view(-1, 2))


def dft_batch(x, dt, freqs, stream=0):
    """Spectra of the rows of `x` (CUDA float64, shape (nseries, n)) at
    `freqs` (CUDA float64, Hz): sum_m x[s, m] exp(-i 2 pi f m dt), as a
    complex128 CUDA tensor (nseries, nf).  Runs aem_dft_batch on `stream`
    (default: the current stream)."""
    import torch
    lib = load_library()
    if x.dtype != torch.float64 or not x.is_cuda or x.dim() != 2 or freqs.dtype != torch.float64 or not freqs.is_cuda:
        raise ValueError("x must be a 2-D CUDA float64 tensor and freqs a CUDA float64 tensor")
    x, freqs = x.contiguous(), freqs.contiguous()
    ns, n = x.shape
    out = torch.empty((ns, 2 * freqs.numel()), dtype=torch.float64, device=x.device)
    st = stream or torch.cuda.current_stream(x.device).cuda_stream
    rc = lib.aem_dft_batch(x.data_ptr(), n, ns, n, float(dt), freqs.data_ptr(), freqs.numel(), out.data_ptr(), st)
    if rc != 0:
        raise AemError(lib.aem_last_error(None).decode())
    return torch.view_as_complex(out.view(ns, -1, 2))


def check_deck(deck_text, ext_text=None, kmax=False):
    """Validate a deck without a GPU; returns the reference grid sizes
    (X, Y, Z) or raises AemError with the reference's "ERROR: ..." text."""
    lib = load_library()
    g = (ctypes.c_int * 3)()
    rc = lib.aem_check_deck(deck_text.encode(), ext_text.encode() if ext_text else None, KMAX if kmax else STANDARD, g)
    if rc != 0:
        raise AemError(lib.aem_last_error(None).decode())
    return tuple(g)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


class Simulation:
    """One solver run on the current CUDA device.

    ``Simulation("inputs.txt").run_all()`` reproduces ``./FDTD inputs.txt``
    of the reference: it writes ``<name>_geometry.bin`` at creation and
    ``<name>.dat`` (and video files when the deck asks) on
    :meth:`write_outputs`.  Output files go to ``outdir`` (default: current
    directory, like the reference executable).
    """

    def __init__(self, inputs_path=None, kmax=False, outdir=None, deck_text=None, ext_text=None, bulk=None):
        self._lib = load_library()
        self._h = ctypes.c_void_p()
        mode = KMAX if kmax else STANDARD
        od = os.fsencode(outdir) if outdir else None
        if deck_text is None:
            rc = self._lib.aem_create_from_file(os.fsencode(inputs_path), mode, od, ctypes.byref(self._h))
        else:
            ptr, n = None, 0
            if bulk is not None:
                if bulk.dtype != np.float32 or not bulk.flags.c_contiguous:
                    raise ValueError("bulk must be a contiguous float32 array (x fastest)")
                ptr, n = bulk.ctypes.data, bulk.size
            rc = self._lib.aem_create_from_memory(deck_text.encode(), ext_text.encode() if ext_text else None, ptr, n,
                                                  mode, od, ctypes.byref(self._h))
        if rc != 0:
            raise AemError(self._lib.aem_last_error(None).decode())
        self.kmax = kmax

    def _check(self, rc):
        if rc == -5:
            raise AemDiverged(self._lib.aem_last_error(self._h).decode())
        if rc < 0:
            raise AemError(self._lib.aem_last_error(self._h).decode())
        return rc

    @property
    def steps(self):
        d, t = ctypes.c_int(), ctypes.c_int()
        self._lib.aem_steps(self._h, ctypes.byref(d), ctypes.byref(t))
        return d.value, t.value

    @property
    def time_step(self):
        """del_t in seconds."""
        dt = ctypes.c_double()
        self._check(self._lib.aem_time_step(self._h, ctypes.byref(dt)))
        return dt.value

    @property
    def grid(self):
        g = (ctypes.c_int * 3)()
        self._lib.aem_grid(self._h, g)
        return tuple(g)

    @property
    def device_bytes(self):
        b = ctypes.c_size_t()
        self._lib.aem_device_bytes(self._h, ctypes.byref(b))
        return b.value

    def run(self, nsteps):
        self._check(self._lib.aem_run(self._h, int(nsteps)))

    def run_graph(self, nsteps, steps_per_graph=64):
        """run() replaying one captured CUDA graph of `steps_per_graph`
        steps for every whole chunk (same results as run())."""
        self._check(self._lib.aem_run_graph(self._h, int(nsteps), int(steps_per_graph)))

    def synchronize(self):
        self._check(self._lib.aem_synchronize(self._h))

    def run_all(self, write=True):
        done, total = self.steps
        self.run(total - done)
        self.synchronize()
        if write:
            self.write_outputs()
        return self

    def write_outputs(self):
        self._check(self._lib.aem_write_outputs(self._h))

    def series(self, kind, index=0):
        """A time series of the finished run (complex for kmax)."""
        k = SERIES[kind] if isinstance(kind, str) else int(kind)
        n = self.steps[1]
        re, im = np.zeros(n), np.zeros(n)
        m = self._check(self._lib.aem_get_series(self._h, k, int(index), _dptr(re), _dptr(im), n))
        return (re[:m] + 1j * im[:m]) if self.kmax else re[:m]

    def field(self, comp):
        """Final field component in the reference's layout, shape (nz, ny, nx) of F-order (x fastest);
        "material" gives the cells' material indices (0 = background, r = r-th volume material)."""
        c = FIELDS[comp] if isinstance(comp, str) else int(comp)
        dims = (ctypes.c_int * 3)()
        self._check(self._lib.aem_get_field(self._h, c, dims, None, None))
        n = dims[0] * dims[1] * dims[2]
        re, im = np.zeros(n), np.zeros(n)
        self._check(self._lib.aem_get_field(self._h, c, dims, _dptr(re), _dptr(im)))
        shape = (dims[2], dims[1], dims[0])
        out = re.reshape(shape)
        if c == 6:
            return out.astype(np.uint8)
        return out + 1j * im.reshape(shape) if self.kmax else out

    def probe(self, kind, index=0, first=1, n=None):
        """Raw per-step samples of the steps run so far (port voltage,
        unnormalised plane sums, or a point-probe component: kind "point",
        index 3 p + c); synchronises."""
        k = PROBE_KINDS[kind] if isinstance(kind, str) else int(kind)
        if n is None:
            n = self.steps[0] - first + 1
        re, im = np.zeros(n), np.zeros(n)
        self._check(self._lib.aem_read_probe(self._h, k, int(index), int(first), int(n), _dptr(re), _dptr(im)))
        return (re + 1j * im) if self.kmax else re

    def autotune(self, steps_per_candidate=2):
        """Tune the general update's launch shape on the run's next steps
        (up to 8 x steps_per_candidate of them; the fields are unchanged).
        Returns {"update_h": (z planes, rows), "update_e": (z planes, rows)}."""
        out = (ctypes.c_int * 4)()
        self._check(self._lib.aem_autotune(self._h, int(steps_per_candidate), out))
        return {"update_h": (out[0], out[1]), "update_e": (out[2], out[3])}

    def checkpoint_save(self, path):
        """Write the whole run state after the steps done so far to `path`."""
        self._check(self._lib.aem_checkpoint_save(self._h, os.fsencode(path)))

    def checkpoint_load(self, path):
        """Restore a state written by checkpoint_save of a run of the same
        deck; the run continues from that step."""
        self._check(self._lib.aem_checkpoint_load(self._h, os.fsencode(path)))

    def spectrum(self, kind, index=0, n=4096):
        """On-the-fly spectrum of a per-step series over the steps run so
        far (sidecar extension `dft_freqs f_start f_stop count`):
        X(f) = sum_m x[m] exp(-2 pi i f m dt) of the raw samples that
        probe() returns.  Returns (freqs in Hz, complex128 array)."""
        k = SERIES[kind] if isinstance(kind, str) else int(kind)
        f, re, im = np.zeros(n), np.zeros(n), np.zeros(n)
        m = self._check(self._lib.aem_read_spectrum(self._h, k, int(index), int(n), _dptr(f), _dptr(re), _dptr(im)))
        return f[:m], re[:m] + 1j * im[:m]

    def profile(self, enable=True):
        """Turn per-phase event timing on (clearing the record) or off."""
        self._check(self._lib.aem_profile(self._h, 1 if enable else 0))

    def profile_read(self):
        """{phase: (milliseconds, launches)} since profiling was turned on."""
        ms = (ctypes.c_double * len(PHASES))()
        nl = (ctypes.c_longlong * len(PHASES))()
        self._check(self._lib.aem_profile_read(self._h, ms, nl))
        return {PHASES[p]: (ms[p], nl[p]) for p in range(len(PHASES))}

    def flush(self):
        """Bin the far-field contributions still held in the 32-step batch buffer."""
        self._check(self._lib.aem_flush(self._h))

    @property
    def stream(self):
        """The cudaStream_t the solver launches on (an integer handle)."""
        s = ctypes.c_void_p()
        self._check(self._lib.aem_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    @property
    def transfer_bytes(self):
        """(host->device, device->host) bytes copied so far."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self._lib.aem_transfer_bytes(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    @property
    def launches(self):
        n = ctypes.c_longlong()
        self._check(self._lib.aem_launch_count(self._h, ctypes.byref(n)))
        return n.value

    @property
    def workload(self):
        """(cells per step as the reference counts them, algorithmic bytes per step)."""
        c, b = ctypes.c_longlong(), ctypes.c_double()
        self._check(self._lib.aem_workload(self._h, ctypes.byref(c), ctypes.byref(b)))
        return c.value, b.value

    @property
    def far_field_size(self):
        """(Huygens-surface cells, far-field angles): each step bins their
        product of contributions."""
        c, a = ctypes.c_longlong(), ctypes.c_int()
        self._check(self._lib.aem_far_field_size(self._h, ctypes.byref(c), ctypes.byref(a)))
        return c.value, a.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.aem_destroy(self._h)
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


def run_batch(sims, nsteps, steps_per_graph=64):
    """Advance independent runs together: each Simulation (same device, its
    own stream) replays its CUDA graph of `steps_per_graph` steps, the runs
    round-robin, so that small grids overlap on the GPU.  Each run's results
    equal Simulation.run()'s."""
    sims = list(sims)
    if not sims:
        return
    lib = load_library()
    arr = (ctypes.c_void_p * len(sims))(*[s._h for s in sims])
    rc = lib.aem_run_batch(arr, len(sims), int(nsteps), int(steps_per_graph))
    if rc != 0:
        msg = lib.aem_last_error(None)
        raise RuntimeError("aem_run_batch failed (%d): %s" % (rc, msg.decode() if msg else ""))


def run_deck(inputs_path, kmax=False, outdir=None):
    """Run a whole deck and write the reference's output files."""
    with Simulation(inputs_path, kmax=kmax, outdir=outdir) as sim:
        sim.run_all()


def exported_symbols():
    """Function names declared in include/alpineem_b200.h."""
    import re
    with open(HEADER_PATH) as f:
        txt = f.read()
    return sorted(set(re.findall(r"\b(aem_[a-z_]+)\s*\(", txt)))
