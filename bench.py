"""bench.py -- FDTD time-step throughput of the B200 solver.

Workload "dipole_ellipsoids": a 1024^3 grid (2 mm cells, 16-cell CPML on
every face) with a 60-cell z dipole fed by a 1-cell 50-ohm lumped port
(Gaussian pulse), 64 random dielectric ellipsoids (eps_r ~ U[2,12],
semi-axes ~ U[5,40] cells, numpy default_rng(2)) given as a bulk geometry
array, and time-domain far fields at 684 angles (10 x 10 degree theta/phi
grid); deck length 4000 steps (alpineem_b200/workloads.py).  One bench step
is one full FDTD time step of that deck: H and E updates with CPML, the
port half-steps, the Huygens-surface currents and the retarded-time binning
of all 684 angles (binned once per 32 steps over the buffered currents).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is Mcell-updates/s, cells counted as the reference does
((X-1)(Y-1)(Z-1) per step): K steps timed with CUDA events on the solver's
stream, inputs resident on the device (28 GB of fields and tables, far above
the 126 MB L2, so no L2 flush is needed).  With N > 1 (torchrun) every rank
runs an independent replica (a single grid is not split across GPUs) and
the value is the sum of the ranks' cell-updates over the slowest rank's
time.  `e2e` times a complete K-step job through the C ABI from host
buffers: model upload, K steps each followed by a device->host read of that
step's port voltage, and the output files (phases_s splits it into model
set-up, steps and writes).  `--impl reference` times the CPU oracle (a
C/OpenMP restatement of the reference's Fortran loop) on the same workload
on all host threads: the GPU grid when host memory allows it, else the
largest power-of-two fraction of it that fits (reference_grid).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FDTD Mcell-updates/s"
UNIT = "Mcell-updates/s"
WORKLOAD = "dipole_ellipsoids"
FALLBACK_HBM_GBS = 6650.0
ORACLE = os.path.join(ROOT, "oracle", "_build", "fdtd_oracle")


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=96)
    ap.add_argument("--warmup", type=int, default=32)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=1024, help="grid cells per axis of the GPU workload")
    ap.add_argument("--cpu-n", type=int, default=0,
                    help="grid cells per axis of the reference arm (0: the GPU grid if host memory allows)")
    ap.add_argument("--cpu-baseline-n", type=int, default=512, help="grid cells per axis of the cpu_baseline sample")
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed steps of the cpu_baseline sample")
    ap.add_argument("--no-configs", action="store_true", help="skip the scattering and layered-slab measurements")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched kmax-instance measurement")
    ap.add_argument("--batch-steps", type=int, default=192, help="timed steps of every batched instance")
    ap.add_argument("--batch-graph", type=int, default=32, help="steps per captured CUDA graph")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the design-gradient measurement")
    ap.add_argument("--adjoint-n", type=int, default=192, help="grid cells per axis of the design-gradient workload")
    ap.add_argument("--adjoint-steps", type=int, default=3000)
    ap.add_argument("--adjoint-checkpoint", type=int, default=200, help="steps between forward checkpoints")
    ap.add_argument("--adjoint-fd", type=int, default=20,
                    help="design cells checked against FP64 central differences (2 FP64 runs each)")
    return ap.parse_args()


def ranks():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def dram_traffic_ratio():
    """Measured DRAM bytes of one fused Yee launch over its algorithmic bytes,
    from the committed ncu record profiles/yee_update_dipole_ellipsoids.json
    (field dram_traffic_over_algorithmic), or None.  The capture runs a
    smaller instance of the workload; the ratio (halo re-reads of the tiles)
    carries over to the full grid, the per-cell bytes do not (the CPML share
    of the cells shrinks as the grid grows)."""
    p = os.path.join(ROOT, "profiles", "yee_update_dipole_ellipsoids.json")
    try:
        with open(p) as f:
            return float(json.load(f)["dram_traffic_over_algorithmic"])
    except (OSError, KeyError, ValueError):
        return None


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def host_mem_available():
    """Bytes of host memory available (MemAvailable), or None."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def reference_grid(n):
    """Grid of the CPU runs: the GPU workload's own n^3 when the oracle's
    working set (about 52 B per cell plus the bulk file) fits in the host's
    available memory with a margin, else the largest power-of-two fraction
    of n that does."""
    avail = host_mem_available() or 0
    m = n
    while m > 128 and 64 * m ** 3 > 0.8 * avail:
        m //= 2
    return m


def workload_config(n):
    """The `config` object of both arms' JSON lines for an n^3 grid."""
    return {"workload": WORKLOAD, "grid": [n, n, n], "cells": n ** 3, "cpml_cells": 16, "ellipsoids": 64,
            "far_field_angles": 684, "s11_frequencies": 512, "deck_steps": 4000,
            "l2": "no flush: the fields and tables (about 28 GB at 1024^3) are far above the 126 MB L2"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) != len(self.FIELDS):
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def write_case(directory, deck, ext, bulk):
    """A deck directory the oracle (or the FDTD-B200 launcher) can run."""
    from alpineem_b200.deck import deck_text
    with open(os.path.join(directory, "inputs.txt"), "w") as f:
        f.write(deck_text(deck))
    with open(os.path.join(directory, "inputs.txt.b200"), "w") as f:
        f.write(ext)
    bulk.tofile(os.path.join(directory, deck["bulk"]))


def oracle_sample(n, warm, steps, threads=None):
    """Time `steps` oracle steps (after `warm` untimed ones) on an n^3
    instance of the workload; returns (Mcell-updates/s, threads, cells)."""
    from alpineem_b200 import workloads
    if not os.path.exists(ORACLE):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    deck, ext, bulk = workloads.dipole_ellipsoids(n=n)
    with tempfile.TemporaryDirectory() as d:
        write_case(d, deck, ext, bulk)
        del bulk
        threads = threads or os.cpu_count() or 1
        env = dict(os.environ, ORACLE_MAX_STEPS=str(warm + steps), ORACLE_WARMUP_STEPS=str(warm),
                   ORACLE_TIMING_FILE=os.path.join(d, "timing.json"), OMP_NUM_THREADS=str(threads),
                   OMP_PROC_BIND="close", OMP_PLACES="cores")
        r = subprocess.run([ORACLE, "inputs.txt"], cwd=d, env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle failed: " + r.stdout[-1000:] + r.stderr[-1000:])
        with open(os.path.join(d, "timing.json")) as f:
            t = json.load(f)
    return t["cells"] * t["steps"] / t["seconds"] / 1e6, t["threads"], t["cells"]


def reference_arm(args):
    """The reference's CPU path on this box's host cores: the oracle on the
    GPU arm's own grid when host memory allows (else a power-of-two fraction
    of it, reference_grid), 1 untimed warm-up step, then min(--steps, 3)
    timed steps at 1024^3 (a step there is seconds of work on all host
    threads) or --steps after --warmup on smaller grids."""
    rank, _, world = ranks()
    if rank != 0:
        return
    n = args.cpu_n or reference_grid(args.n)
    warm, steps = (1, min(args.steps, 3)) if n >= 1024 else (args.warmup, args.steps)
    v, threads, cells = oracle_sample(n, warm, steps)
    sample = ("%d^3 instance of the workload (%d cells, 64 ellipsoids, 684 far-field angles, 16-cell CPML, "
              "port spectra at 512 frequencies), %d timed steps after %d warm-up; grid %s"
              % (n, cells, steps, warm, "= the GPU arm's" if n == args.n else
                 "reduced from %d^3: host memory" % args.n))
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": round(cells / (v * 1e6) * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(n),
            "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "cpu_model": cpu_model()},
            "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_kmax(rank, world, steps, g, barrier, max_over_ranks):
    """The batched constant-k sweep (64 unit cells, workloads.kmax_batch,
    each with on-the-fly spectra of its four plane sums at 128 frequencies,
    workloads.KMAX_BATCH_EXT): wall time of the instances run one after
    another with plain launches, against the same instances advanced
    together by aem_run_batch (one stream per instance, one CUDA graph of g
    steps per instance).  Ranks take every world-th instance.  Setup, a
    warm-up of each run (4 steps and the launch-shape autotuning, 16 steps)
    and the graph capture (one untimed chunk) are outside both timings."""
    import numpy as np

    import alpineem_b200 as ab
    from alpineem_b200.parallel import shard
    from alpineem_b200 import workloads
    from alpineem_b200.deck import deck_text

    # every instance tunes the launch shape of its update kernels during its
    # warm-up (8 candidate shapes x 2 steps, extension `autotune 2`)
    tune = 2
    warm = 4 + 8 * tune
    ext = workloads.KMAX_BATCH_EXT + "autotune %d\n" % tune
    kinds = ("reflected", "transmitted", "reflected_tm", "transmitted_tm")
    decks = shard(workloads.kmax_batch(steps=warm + 2 * g + steps), rank, world)
    tmp = tempfile.mkdtemp(prefix="aem_batch_")
    seq = 0.0
    cells = 0
    spectra = []
    for d in decks:
        sim = ab.Simulation(deck_text=deck_text(d), ext_text=ext, kmax=True, outdir=tmp)
        cells += sim.workload[0]
        sim.run(warm + g)
        sim.synchronize()
        t0 = time.perf_counter()
        sim.run(steps)
        sim.synchronize()
        seq += time.perf_counter() - t0
        spectra.append([sim.spectrum(k)[1] for k in kinds])
        sim.close()
    sims = [ab.Simulation(deck_text=deck_text(d), ext_text=ext, kmax=True, outdir=tmp) for d in decks]
    try:
        for s in sims:
            s.run(warm)
        ab.run_batch(sims, g, g)  # captures every instance's graph
        for s in sims:
            s.synchronize()
        barrier()
        t0 = time.perf_counter()
        ab.run_batch(sims, steps, g)
        for s in sims:
            s.synchronize()
        bat = time.perf_counter() - t0
        # the same steps in the same order: the spectra must agree bit for bit
        same = all(np.array_equal(a, b) for s, ref in zip(sims, spectra) for a, b in zip([s.spectrum(k)[1] for k in kinds], ref))
    finally:
        for s in sims:
            s.close()
    seq, bat = max_over_ranks(seq), max_over_ranks(bat)
    return {"workload": "kmax_batch", "instances": 64, "grid": "64 x 64 x Z, Z in {128..512}, complex64",
            "steps_timed": steps, "steps_per_graph": g, "sequential_s": round(seq, 4), "batched_s": round(bat, 4),
            "speedup": round(seq / bat, 2),
            "batched_mcell_updates_per_s": round(world * cells * steps / bat / 1e6, 1),
            "spectra": "128 frequencies x 4 plane sums per instance, FP64 Kahan, accumulated every step",
            "spectra_equal_sequential_batched": bool(same)}


def adjoint_gradient(args, max_over_ranks):
    """Design gradient (workloads.adjoint_probe: 192^3, 12-cell CPML, 3000
    steps, 64x64x32 design cells of eps_r ~ U[1,4], |DFT_10GHz(Ez)|^2 at a
    probe 40 cells beyond the box): device time of a plain FP32 forward run
    against the checkpointed forward run plus the adjoint sweep (which
    recomputes every checkpoint segment but the last), and the same with
    the whole design-box history kept (one segment).  With --adjoint-fd C,
    C random design cells are checked against FP64 central differences
    (delta = 1e-3).  Every rank runs its own replica."""
    import numpy as np
    from alpineem_b200 import workloads
    from alpineem_b200.adjoint import Design
    from alpineem_b200.deck import deck_text

    n, steps, K = args.adjoint_n, args.adjoint_steps, args.adjoint_checkpoint
    d, ext, lo, box, probe, freq, eps = workloads.adjoint_probe(n=n, steps=steps)
    tmp = tempfile.mkdtemp(prefix="aem_adj_")
    path = os.path.join(tmp, "inputs.txt")
    with open(path, "w") as f:
        f.write(deck_text(d))
    with open(path + ".b200", "w") as f:
        f.write(ext)
    out = {"workload": "adjoint_probe", "grid": [n] * 3, "cpml_cells": 12, "steps": steps,
           "design_box": list(box), "design_cells": int(np.prod(box)), "probe": list(probe), "freq_hz": freq,
           "figure_of_merit": "|DFT of Ez at the probe|^2", "dtype": "f32", "checkpoint_every": K}
    with Design(path, lo, box, probe, freq, precision=32) as dsn:
        dsn.set_design(eps)
        dsn.forward(0)  # warm-up
        f_plain, _ = dsn.forward(0)
        t_plain = dsn.timing()[0]
        f_ck, _ = dsn.forward(K)
        g = dsn.gradient()
        t_fwd, t_grad, l_fwd, l_grad = dsn.timing()
        dsn.forward(steps)
        g_all = dsn.gradient()
        t_fwd_all, t_grad_all, _, _ = dsn.timing()
        sweep = {}
        for k in (100, 50):
            if k < steps and k != K:
                dsn.forward(k)
                dsn.gradient()
                tf, tg, _, _ = dsn.timing()
                sweep[str(k)] = round((max_over_ranks(tf) + max_over_ranks(tg)) / max_over_ranks(t_plain), 3)
        cells = n ** 3
        t_plain, t_fwd, t_grad = max_over_ranks(t_plain), max_over_ranks(t_fwd), max_over_ranks(t_grad)
        t_fwd_all, t_grad_all = max_over_ranks(t_fwd_all), max_over_ranks(t_grad_all)
        out.update({"fom": f_plain, "plain_forward_ms": round(t_plain, 2),
                    "forward_mcell_updates_per_s": round(cells * steps / (t_plain / 1e3) / 1e6, 1),
                    "checkpointed_forward_ms": round(t_fwd, 2), "gradient_ms": round(t_grad, 2),
                    "ratio": round((t_fwd + t_grad) / t_plain, 3),
                    "store_all_forward_ms": round(t_fwd_all, 2), "store_all_gradient_ms": round(t_grad_all, 2),
                    "store_all_ratio": round((t_fwd_all + t_grad_all) / t_plain, 3),
                    "ratio_by_checkpoint_interval": sweep,
                    "gradient_launches": l_grad, "forward_launches": l_fwd,
                    "segments_equal": bool(np.array_equal(g, g_all)), "fom_equal": f_plain == f_ck,
                    "grad_abs_max": float(np.abs(g).max())})
    if args.adjoint_fd > 0:
        rng = np.random.default_rng(7)
        pick = [tuple(int(rng.integers(0, s)) for s in eps.shape) for _ in range(args.adjoint_fd)]
        errs = []
        with Design(path, lo, box, probe, freq, precision=64) as d64:
            for c in pick:
                vals, pts = [], []
                for sgn in (1, -1):
                    e = eps.copy()
                    e[c] = np.float32(float(e[c]) + sgn * 1e-3)
                    pts.append(float(e[c]))
                    d64.set_design(e)
                    vals.append(d64.forward(0)[0])
                fd = (vals[0] - vals[1]) / (pts[0] - pts[1])
                errs.append({"cell": list(c), "fd": fd, "adjoint_f32": float(g[c]),
                             "rel_err": abs(float(g[c]) - fd) / abs(fd) if fd else None})
        out["fd_check"] = {"delta": 1e-3, "fd_precision": "f64", "cells": errs,
                           "max_rel_err": max(e["rel_err"] for e in errs if e["rel_err"] is not None)}
    return out


def config_runs(max_over_ranks, world):
    """The scattering (workloads.pec_sphere: 96^3, 2000 steps) and layered
    unit-cell (workloads.layered_slab: 128 x 128 x 512, 8000 steps)
    configurations, each run whole on the device: Mcell-updates/s of all
    its steps (CUDA events on the solver's stream, every rank a replica),
    the per-phase split, and the update kernels' HBM roofline (the
    algorithmic bytes of the Yee/CPML update over their summed event time);
    then the same run again through CUDA-graph replay, timed by events
    around the whole run (no per-phase events)."""
    import torch
    import alpineem_b200 as ab
    from alpineem_b200 import workloads
    from alpineem_b200.deck import deck_text
    peak, _ = hbm_peak()
    out = {}
    for name, (deck, ext, _) in (("pec_sphere", workloads.pec_sphere()), ("layered_slab", workloads.layered_slab())):
        tmp = tempfile.mkdtemp(prefix="aem_cfg_")
        # the first 16 steps tune the update kernels' launch shape (inside the timing)
        sim = ab.Simulation(deck_text=deck_text(deck), ext_text=ext + "autotune 2\n", outdir=tmp)
        cells, bytes_step = sim.workload
        steps = sim.steps[1]
        sim.synchronize()
        sim.profile(True)
        t0 = time.perf_counter()
        sim.run(steps)
        sim.synchronize()
        wall = max_over_ranks(time.perf_counter() - t0)
        prof = sim.profile_read()
        sim.profile(False)
        shape = sim.autotune(0)  # the shapes the run tuned (no further steps)
        sim.close()
        # the same run through CUDA-graph replay (aem_run_graph, 64-step
        # graphs after the tuning steps), unprofiled: CUDA events on the
        # solver's stream around the whole run, and the host clock
        sim = ab.Simulation(deck_text=deck_text(deck), ext_text=ext + "autotune 2\n", outdir=tmp)
        sim.synchronize()
        stream = torch.cuda.ExternalStream(sim.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        ev0.record(stream)
        sim.run_graph(steps, 64)
        ev1.record(stream)
        sim.synchronize()
        gwall = max_over_ranks(time.perf_counter() - t0)
        gdev = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
        sim.close()
        dev_ms = max_over_ranks(sum(v[0] for v in prof.values()))
        t_upd = (prof["update_h"][0] + prof["update_e"][0] + prof["yee"][0]) / steps / 1e3
        out[name] = {"grid": list(deck["n"]), "steps": steps, "cells": cells,
                     "device_mcell_updates_per_s": round(world * cells * steps / (dev_ms / 1e3) / 1e6, 1),
                     "wall_mcell_updates_per_s": round(world * cells * steps / wall / 1e6, 1),
                     "graph_device_mcell_updates_per_s": round(world * cells * steps / gdev / 1e6, 1),
                     "graph_wall_mcell_updates_per_s": round(world * cells * steps / gwall / 1e6, 1),
                     "phases_ms_per_step": {k: round(v[0] / steps, 5) for k, v in prof.items() if v[1]},
                     "update_roofline_frac": round(bytes_step / t_upd / 1e9 / peak, 4),
                     "update_path": "fused k_yee4" if prof["yee"][1] else "k_update_h + k_update_e",
                     "launch_shape": {k: {"z_planes": v[0], "rows": v[1]} for k, v in shape.items()}}
    return out


def ours(args):
    import torch
    import alpineem_b200 as ab
    from alpineem_b200 import workloads
    from alpineem_b200.deck import deck_text

    rank, local, world = ranks()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    K, W = args.steps, args.warmup
    t0 = time.time()
    deck, ext, bulk = workloads.dipole_ellipsoids(n=args.n)
    t_gen = time.time() - t0
    tmp = tempfile.mkdtemp(prefix="aem_bench_")
    t0 = time.time()
    sim = ab.Simulation(deck_text=deck_text(deck), ext_text=ext, bulk=bulk, outdir=tmp)
    t_setup = time.time() - t0
    cells, bytes_step = sim.workload

    # warm-up (its far-field contributions binned before the timed region),
    # then K timed steps whose own contributions are binned inside it;
    # per-phase events bracket every launch
    sim.run(W)
    sim.flush()
    sim.synchronize()
    sim.profile(True)
    stream = torch.cuda.ExternalStream(sim.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = sim.launches
    barrier()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        sim.run(K)
        sim.flush()
        ev1.record(stream)
        sim.synchronize()
        barrier()
    ms = ev0.elapsed_time(ev1)
    launches = sim.launches - launches0
    prof = sim.profile_read()
    ff_cells, ff_angles = sim.far_field_size
    # steady state of the far-field binning: one whole 32-step batch
    sim.profile(True)
    sim.run(32)
    steady = sim.profile_read()
    sim.profile(False)
    ms_max = max_over_ranks(ms)
    value = world * cells * K / (ms_max / 1e3) / 1e6

    # roofline of the Yee update (the fused kernel, or the H and E kernels)
    t_yee = (prof["update_h"][0] + prof["update_e"][0] + prof["yee"][0]) / K / 1e3
    peak, peak_kind = hbm_peak()
    achieved = bytes_step / t_yee / 1e9
    ratio = dram_traffic_ratio()
    kname = "k_yee4 (fused H+E step, TMA-fed)" if prof["yee"][1] else "k_update_h + k_update_e (one Yee step)"
    roofline = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1),
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": round(ratio * bytes_step) if ratio else None,
                "traffic_source": "profiles/yee_update_dipole_ellipsoids.json (ncu DRAM bytes / algorithmic bytes "
                                  "of a 384^3 capture, times this launch's algorithmic bytes)",
                "algorithmic_bytes": round(bytes_step), "bytes_per_cell_update": round(bytes_step / cells, 2)}
    phases = {k: round(v[0] / K, 4) for k, v in prof.items() if v[1]}
    far_field = None
    if prof["ff_bin"][1] and prof["ff_bin"][0] > 0:
        contrib = ff_cells * ff_angles
        far_field = {"metric": "binned far-field contributions/s", "face_cells": ff_cells, "angles": ff_angles,
                     "contributions_per_step": contrib, "batch_steps": 32,
                     "timed_ms_per_step": round(prof["ff_bin"][0] / K, 4),
                     "timed_note": "the K timed steps are binned in ceil(K/32) batches inside the timed region",
                     "steady_ms_per_step": round(steady["ff_bin"][0] / 32, 4),
                     "value": round(world * contrib / (steady["ff_bin"][0] / 32 / 1e3), 1)}
    n_s11 = len(sim.spectrum("port_voltage", 0, n=4096)[0])  # on-the-fly S11 spectra, accumulated every step
    sim.close()
    del sim

    e2e = None
    if not args.no_e2e:
        # a complete K-step job through the C ABI from host buffers
        deck_k = dict(deck, steps=K)
        pinned = torch.empty(bulk.size, dtype=torch.float32, pin_memory=True)
        pinned.numpy()[:] = bulk.reshape(-1)
        host_bulk = pinned.numpy()
        etmp = tempfile.mkdtemp(prefix="aem_e2e_")
        barrier()
        t0 = time.perf_counter()
        job = ab.Simulation(deck_text=deck_text(deck_k), ext_text=ext, bulk=host_bulk, outdir=etmp)
        job.synchronize()
        tc = time.perf_counter()
        for s in range(1, K + 1):
            job.run(1)
            job.probe("port_voltage", 0, first=s, n=1)
        ts = time.perf_counter()
        job.write_outputs()
        t1 = time.perf_counter()
        h2d, d2h = job.transfer_bytes
        job.close()
        wall = max_over_ranks(t1 - t0)
        e2e = {"value": round(world * cells * K / wall / 1e6, 3), "unit": UNIT,
               "h2d_bytes_per_step": round(h2d / K), "d2h_bytes_per_step": round(d2h / K),
               "seconds": round(wall, 3), "steps": K,
               "phases_s": {"create": round(tc - t0, 3), "steps": round(ts - tc, 3), "write": round(t1 - ts, 3)}}

    batched = None
    if not args.no_batch:
        batched = batched_kmax(rank, world, args.batch_steps, args.batch_graph, barrier, max_over_ranks)

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_gradient(args, max_over_ranks)

    configs = None
    if not args.no_configs:
        configs = config_runs(max_over_ranks, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cn = min(args.cpu_baseline_n, reference_grid(args.n))
        v, threads, ccells = oracle_sample(cn, 1, args.cpu_steps)
        cpu = {"value": round(v, 3), "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
               "sample": "oracle (C/OpenMP restatement of the reference loop) on a %d^3 instance of the workload "
                         "(%d cells, same CPML, ellipsoids, port and 684 far-field angles), %d timed steps after 1 warm-up"
                         % (cn, ccells, args.cpu_steps)}

    if rank == 0:
        config = dict(workload_config(args.n), parallelism="replicas" if world > 1 else "single")
        line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": round(ms_max / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": config,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
                "gpu_launches": launches, "phases_ms_per_step": phases, "far_field": far_field,
                "s11_frequencies": n_s11, "configs": configs, "batched_kmax": batched, "adjoint": adjoint,
                "setup_s": round(t_setup, 2), "workload_gen_s": round(t_gen, 2)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.steps < 1 or args.warmup < 3:
        sys.exit("--steps must be >= 1 and --warmup >= 3")
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
