#!/usr/bin/env python
"""Benchmark of the stochastic-KPM hot path (KPM moment recurrence).

Workload (one "step"): the Jackson-KPM moments mu_0..mu_{M-1} of R random-phase
vectors on the honeycomb lattice of 2048 x 1024 cells x 2 = 4,194,304 sites
(t = -2.7 eV, Anderson disorder in [-1, 1] eV), R = 64 vectors in one block,
M = 4096 moments, spectral window (-9.2, 9.2) eV.  B200 arm: the mixed form
(complex64 vectors and SpMM, FP64 moment accumulation) with the product
identity for the moments; the plain FP64 path is measured beside it.  Work is
counted as N * M * R orbital*moment*vec per step.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One process per GPU (torchrun for N > 1): every rank owns R independent
vectors (its statistics block; replicated H), no collective in the timed
region (weak scaling); the step time is the max over ranks.
`--impl reference` times KuboMSD's own compiled CPU engine (cpp/native.cpp,
built into oracle/_ref/) on this host's cores for the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "orbital·moment·vec/s mixed vs FP64 @MSD relerr≤1e-4; HBM GB/s; p50/p99 latency"
UNIT = "orbital·moment·vec/s"
BOUNDS = (-9.2, 9.2)
FALLBACK_HBM_GBS = 6650.0
# dram bytes (read + write) per launch of the dominant kernel for the default
# workload: an ncu capture of one step-kernel launch on 524,288 sites x 64
# complex64 columns read 553.9 MB and wrote 234.0 MB; traffic grows with the
# rows, so a 4,194,304-site launch moves (553.9 + 234.0) MB x 8.
NCU_TRAFFIC_PER_LAUNCH = (553.9e6 + 234.0e6) * 8


def parse():
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--lx", type=int, default=2048)
    p.add_argument("--ly", type=int, default=1024)
    p.add_argument("--vectors", type=int, default=64)
    p.add_argument("--moments", type=int, default=4096)
    p.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--method", choices=["doubling", "direct"], default="doubling")
    p.add_argument("--workload", choices=["honeycomb", "diamond", "batch", "serving", "series"],
                   default="honeycomb",
                   help="honeycomb: the headline KPM-moment workload; diamond: the nonorthogonal sp3 model "
                        "(8000 atoms x 4 orbitals, kappa(S)=50, block-Jacobi PCG to 1e-10, R=32, M=1024); "
                        "batch: a ragged batch of 32 nonorthogonal sp3 instances (4,000-32,000 orbitals), R=16; "
                        "serving: a Poisson request stream through the continuous-batching service; "
                        "series: the augmented series step of the stepwise MSD alone (honeycomb lx x ly, "
                        "[psi | phi] = 2 x vectors columns)")
    p.add_argument("--metric-storage", choices=["fp64", "mixed"], default="fp64",
                   help="diamond / batch workloads: storage of the CG work vectors (mixed: complex64, FP64 "
                        "arithmetic, solution, inner products and tests)")
    p.add_argument("--no-compare", action="store_true", help="skip the FP64 / direct comparison lines")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the per-configuration blocks (config 1 in full, config 2 at full size, the "
                        "config-3 stepwise MSD with the series step, a config-4 batch sample, a config-5 serving "
                        "window)")
    return p.parse_args()


def config(args, n):
    return {"workload": f"KPM moments, honeycomb {args.lx}x{args.ly}x2 = {n:,} sites, R={args.vectors}, "
                        f"M={args.moments}", "sites": n, "vectors_per_gpu": args.vectors, "moments": args.moments,
            "spectral_bounds_eV": list(BOUNDS), "disorder_eV": [-1., 1.], "hopping_eV": -2.7,
            "precision": args.precision, "moment_method": args.method,
            "l2_policy": "inputs larger than L2 (vector blocks of 2.1-4.3 GB per buffer)",
            "parallelism": f"dp{args.gpus} (statistics blocks per GPU, replicated H)"}


def peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        d = json.loads(path.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


M_FULL = 4096


def _ref_engine(H, S, threads, **kw):
    """KuboMSD's compiled CPU engine (oracle/_ref), or None when it is absent."""
    from oracle import ref_native
    if ref_native.load() is None:
        return None
    return ref_native.RefEngine(H, S, threads=threads, **kw)


def time_applications(run, steps=1):
    """Seconds of the set-up part (M=1: S B and mu_0) and of one operator
    application (an M=2 call minus the set-up) of a moments call `run(M)`."""
    t0 = time.perf_counter()
    run(1)
    t1 = time.perf_counter() - t0
    t2 = []
    for _ in range(steps):
        t0 = time.perf_counter()
        run(2)
        t2.append(time.perf_counter() - t0)
    t2 = min(t2)
    return t1, max(t2 - t1, 1e-9), t2


def cpu_baseline(H, n, threads, R=64, M=M_FULL, setup=None):
    """KuboMSD's compiled CPU engine (oracle/_ref) on a bounded sample of the
    moments workload: one M=1 call (S B and mu_0) and one M=2 call (one
    operator application) on the full lattice with all R vectors; the M-moment
    call is extrapolated as set-up + (M - 1) applications, which is exactly
    the work Engine::moments does (cpp/native.cpp:590-609)."""
    import scipy.sparse as sp
    B = np.exp(2j * np.pi * np.random.default_rng(9).random((n, R)))
    c, a = (BOUNDS[0] + BOUNDS[1]) / 2, (BOUNDS[1] - BOUNDS[0]) / 2
    eng = _ref_engine(H, sp.identity(n, format="csr"), threads)
    kind = "reference"
    if eng is not None:
        run = lambda m: eng.core.moments(B, m, c, a)  # noqa: E731
    else:  # the oracle restatement when the reference binary is absent
        from oracle import kpm_oracle as O
        oe = O.engine_from_model(H, sp.identity(n, format="csr"))
        run = lambda m: oe.moments(B, m, c, a)  # noqa: E731
        kind, threads = "port", 1
    t_setup, t_app, t_call = time_applications(run)
    full = t_setup + (M - 1) * t_app
    return {"value": n * M * R / full, "unit": UNIT, "cores": threads, "kind": kind, "seconds": t_setup + t_call,
            "applications_per_s": n * R / t_app, "seconds_per_application": t_app, "setup_seconds": t_setup,
            "sample": f"Engine::moments on the full {n:,}-site lattice with R={R} vectors: one M=1 call "
                      f"(set-up {t_setup:.2f} s) and one M=2 call (one operator application, {t_app:.2f} s), "
                      f"{threads} OpenMP threads; the M={M} call extrapolated as set-up + {M - 1} applications"}


def reference_sample_ly(lx, ly, steps, warmup, budget_s=180., s_per_site=7e-6):
    """Rows of the honeycomb the reference arm samples.  The engine's set-up
    and application times grow in proportion to the sites (every pass streams
    vector blocks far larger than the host caches), so when the full lattice
    would take more than `budget_s` over the steps asked for (about 7 us per
    site for an M=2 call at R=64 on 16 cores; an M=1 warm-up call is about a
    sixth of that) each step samples a lattice of the same structure with
    ly / 4 rows."""
    n_full = 2 * lx * ly
    if n_full * s_per_site * (steps + warmup / 6) <= budget_s or ly < 8:
        return ly
    return ly // 4


def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return
    from kubomsd_b200 import lattices
    import scipy.sparse as sp
    n_full = 2 * args.lx * args.ly
    ly = reference_sample_ly(args.lx, args.ly, args.steps, args.warmup)
    m = lattices.honeycomb(args.lx, ly, with_velocity=False)
    threads = len(os.sched_getaffinity(0))
    R, M = args.vectors, args.moments
    B = np.exp(2j * np.pi * np.random.default_rng(9).random((m.n, R)))
    c, a = (BOUNDS[0] + BOUNDS[1]) / 2, (BOUNDS[1] - BOUNDS[0]) / 2
    eng = _ref_engine(m.H, sp.identity(m.n, format="csr"), threads)
    kind = "reference"
    if eng is not None:
        run = lambda k: eng.core.moments(B, k, c, a)  # noqa: E731
    else:
        from oracle import kpm_oracle as O
        oe = O.engine_from_model(m.H, sp.identity(m.n, format="csr"))
        run = lambda k: oe.moments(B, k, c, a)  # noqa: E731
        kind, threads = "port", 1
    # warm-up steps are set-up calls (M=1); each timed step is one M=2 call
    # (set-up + one operator application on all R vectors)
    setups = []
    for _ in range(max(args.warmup, 1)):
        t0 = time.perf_counter()
        run(1)
        setups.append(time.perf_counter() - t0)
    t_setup = min(setups)
    apps = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run(2)
        apps.append(time.perf_counter() - t0 - t_setup)
    t_app = max(statistics.median(apps), 1e-9)
    full = t_setup + (M - 1) * t_app
    value = m.n * M * R / full
    where = (f"the full {m.n:,}-site lattice" if m.n == n_full else
             f"a {args.lx}x{ly}x2 = {m.n:,}-site honeycomb of the same structure (the {n_full:,}-site step time "
             f"extrapolated by the site count)")
    cb = {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
          "applications_per_s": m.n * R / t_app, "seconds_per_application": t_app, "setup_seconds": t_setup,
          "sample": f"Engine::moments on {where}, R={R}: warm-up steps are M=1 calls "
                    f"(set-up, min {t_setup:.2f} s), each timed step one M=2 call; the application time is its "
                    f"median minus the set-up ({t_app:.2f} s), and the M={M} call is extrapolated as set-up + "
                    f"{M - 1} applications ({threads} OpenMP threads)"}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": full * 1e3 * n_full / m.n,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded lattice and phases)",
            "applications_per_s": m.n * R / t_app,
            "config": {**config(args, n_full), "reference_sample": cb["sample"]}, "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


class _RefOps:
    """The compiled reference engine (oracle/_ref) behind the method names the
    oracle's stepwise orchestration calls, counting operator applications
    (moment steps of Engine::moments are direct: M - 1 per call)."""

    def __init__(self, ref, S):
        self.core, self.applications = ref.core, 0
        self.metric = type("M", (), {"mul": staticmethod(lambda B: S @ B)})()

    def moments(self, B, length, c, a):
        self.applications += (length - 1) * B.shape[1]
        return self.core.moments(B, length, c, a)

    def series(self, B, coeff, c, a, directions=()):
        self.applications += (len(coeff) - 1) * B.shape[1]
        return self.core.series(B, coeff, c, a, directions)


def _bench_call(fn, sync):
    sync()
    t0 = time.perf_counter()
    out = fn()
    sync()
    return out, time.perf_counter() - t0


def config_c1(threads):
    """Config 1 in full: 64 x 64 square lattice, R=8, M=512, 201 energies,
    stepwise MSD along x over 0-50 fs at dt = 1 fs, no VAC; FP64 and mixed,
    moment doubling.  Work counted as N per application of the scaled
    operator to one vector (moment and propagation steps)."""
    import torch
    import scipy.sparse as sp
    from kubomsd_b200 import kpm, lattices, stochastic
    from kubomsd_b200.config import RunConfig
    from kubomsd_b200.operators import build_operators
    m = lattices.square_lattice(64)
    B = kpm.random_phases(m.n, 20261019, range(8))
    grid = dict(energy_eV=np.linspace(-11, 11, 201), spectral_bounds=(-11.2, 11.2), n_moments=512, axes=("x",),
                include_vac=False, stochastic_method="stepwise")
    out = {"workload": "config 1 in full: stepwise MSD, square 64x64 = 4,096 sites, R=8, M=512, 201 energies, "
                       "0-50 fs at dt = 1 fs, x axis, no VAC", "unit": "orbital·moment·vec/s (N per operator "
                                                                        "application to one vector)"}
    res = {}
    for prec in ("fp64", "mixed"):
        cfg = RunConfig(time_fs=np.arange(51.), precision=prec, moment_doubling=True, **grid)
        ops = build_operators(m, cfg)
        stochastic.stepwise_samples(ops, cfg, B)
        a0, l0 = ops.native.vector_applications, _launches()
        (dos, nums, diag), dt = _bench_call(lambda: stochastic.stepwise_samples(ops, cfg, B), torch.cuda.synchronize)
        apps = ops.native.vector_applications - a0
        res[prec] = (dos, nums["msd_A2/commutator"])
        out[prec] = {"seconds": dt, "value": m.n * apps / dt, "vector_applications": apps,
                     "gpu_launches": _launches() - l0}
    from kubomsd_b200 import accuracy
    out["mixed_vs_fp64"] = accuracy.stepwise_errors(res["mixed"][0], res["mixed"][1], res["fp64"][0],
                                                    res["fp64"][1], np.arange(51.))
    out["value"] = out["mixed"]["value"]
    # each launch is a few microseconds over a 512 KiB vector block: launch- and latency-bound
    out["roofline"] = {"bound": "launch/latency (working set of 0.5-1 MiB per vector block, L2-resident)",
                       "achieved": None, "peak": None, "frac": None}
    ref = _ref_engine(m.H, m.S, threads, velocity=m.velocity)
    if ref is not None:
        from oracle import kpm_oracle as O
        eng = _RefOps(ref, sp.identity(m.n, format="csr"))
        t_end = 5.
        _, dt = _bench_call(lambda: O.stepwise_samples(eng, B, grid["energy_eV"], np.arange(t_end + 1.),
                                                        grid["spectral_bounds"], 512, [[1., 0., 0.]]), lambda: None)
        out["cpu_baseline"] = {"value": m.n * eng.applications / dt, "unit": out["unit"], "cores": threads,
                               "kind": "reference",
                               "sample": f"the same stepwise run over 0-{t_end:g} fs (the reference's compiled "
                                         f"Engine::moments / Engine::series driven by the oracle's restatement of "
                                         f"stepwise.py), {eng.applications} vector applications in {dt:.2f} s"}
    return out


def config_c3_msd(threads, R=64, M=4096, t_end=5.):
    """Config 3 stepwise MSD (the precision form's MSD(E, t)): honeycomb
    4,194,304 sites with its explicit velocity, R=64 vectors, M=4096, x axis,
    mixed form with moment doubling, over 0-t_end fs at dt = 1 fs (config 1's
    grid, truncated to keep the bench short; the cost is linear in the number
    of time points).  The augmented series step (MODE_SERIES: H, V and the
    Bessel accumulation fused, [psi | phi] = 2R columns) is timed on its own
    for its roofline."""
    import torch
    import scipy.sparse as sp
    from kubomsd_b200 import kpm, lattices, stochastic
    from kubomsd_b200.config import RunConfig
    from kubomsd_b200.operators import build_operators
    m = lattices.honeycomb(2048, 1024)
    n = m.n
    B = devstats_phases(n, 20261019, range(R))
    cfg = RunConfig(energy_eV=np.linspace(-9, 9, 201), time_fs=np.arange(t_end + 1.), spectral_bounds=BOUNDS,
                    n_moments=M, axes=("x",), include_vac=False, stochastic_method="stepwise", precision="mixed",
                    moment_doubling=True)
    ops = build_operators(m, cfg)
    c, a = kpm.scaling(cfg)
    out = {"workload": f"config 3 stepwise MSD: honeycomb {n:,} sites, R={R}, M={M}, 201 energies, 0-{t_end:g} fs "
                       f"at dt = 1 fs, x axis, mixed, moment doubling", "unit": "orbital·moment·vec/s (N per operator "
                                                                                  "application to one vector)"}
    # the augmented series step alone: one 1 fs Bessel propagation of [psi | phi]
    coeff, _ = kpm.bessel_coefficients(1., cfg, weighted_tail=True)
    aug = torch.cat([B, torch.zeros_like(B)], dim=1).contiguous()
    ops.native.series(aug, coeff, c, a, [[1., 0., 0.]])
    l0 = _launches()
    res, dt = _bench_call(lambda: ops.native.series(aug, coeff, c, a, [[1., 0., 0.]]), torch.cuda.synchronize)
    steps = len(coeff) - 1
    cols = 2 * R
    row_bytes = series_row_bytes(cols, 4, 4)  # complex64 vectors, 4-wide ELL rows of H and V
    peak, src = peaks()
    ach = n * row_bytes / (dt / steps) / 1e9
    out["series_step"] = {"seconds_per_1fs_propagation": dt, "steps": steps, "ms_per_step": dt / steps * 1e3,
                          "gpu_launches": _launches() - l0,
                          "roofline": {"bound": "hbm", "kernel": "cheb_step_kernel MODE_SERIES (inline velocity)",
                                       "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                       "peak_source": peak_src_note(src),
                                       "algorithmic_bytes_per_row": row_bytes,
                                       "timing": "propagation call time / Bessel steps (includes the set-up copies)"}}
    del res, aug
    a0 = ops.native.vector_applications
    (dos, nums, diag), dt = _bench_call(lambda: stochastic.stepwise_samples(ops, cfg, B, device=True),
                                        torch.cuda.synchronize)
    apps = ops.native.vector_applications - a0
    out.update(seconds=dt, value=n * apps / dt, vector_applications=apps)
    del ops, dos, nums
    torch.cuda.empty_cache()
    ref = _ref_engine(m.H, m.S, threads, velocity=m.velocity)
    if ref is not None:
        Rc = 8
        Bh = B[:, :Rc].cpu().numpy()
        augh = np.concatenate([Bh, np.zeros_like(Bh)], axis=1)
        cf = np.asarray(coeff[:2])
        _, t2 = _bench_call(lambda: ref.core.series(augh, cf, c, a, [[1., 0., 0.]]), lambda: None)
        _, t1 = _bench_call(lambda: ref.core.moments(Bh, 2, c, a), lambda: None)
        out["cpu_baseline"] = {"value": n * 2 * Rc / t2, "unit": out["unit"], "cores": threads, "kind": "reference",
                               "moments_application_per_s": n * Rc / t1,
                               "sample": f"Engine::series of [psi | phi] ({2 * Rc} columns) with one Chebyshev term "
                                         f"(one augmented application, {t2:.2f} s) and an M=2 Engine::moments call "
                                         f"on R={Rc} ({t1:.2f} s), full lattice, {threads} OpenMP threads"}
    return out


def config_c2(threads, storage=("fp64", "mixed"), M=1024):
    """Config 2 at full size: diamond sp3, 32,000 orbitals, kappa(S) = 50,
    block-Jacobi batched PCG to rtol 1e-10 in every operator application,
    R=32, M=1024 moments (direct: the general metric has no product identity)."""
    import torch
    import scipy.linalg as la
    import scipy.sparse as sp
    from types import SimpleNamespace
    from kubomsd_b200 import kpm, lattices
    from kubomsd_b200.native import B200Metric, B200Operators
    m = lattices.diamond_sp3(cells=10)
    S = sp.csr_matrix(m.S)
    blocks = [(a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)) for a, b in m.atom_slices]
    cfg = SimpleNamespace(metric_rtol=1e-10, metric_atol=0., metric_maxiter=1000, metric_residual_policy="fixed",
                          metric_check_interval=32, metric_gap_ratio=.1, metric_solver="pcg", precision="fp64",
                          moment_doubling=False)
    R, c, a = 32, 0., 40.
    B = torch.from_numpy(kpm.random_phases(m.n, 20261019, range(R))).cuda()
    out = {"workload": f"config 2: KPM moments, diamond sp3 {m.n:,} orbitals, kappa(S)=50, block-Jacobi PCG "
                       f"rtol 1e-10, R={R}, M={M}", "unit": UNIT}
    for st in storage:
        metric = B200Metric(S, S.diagonal().real.copy(), blocks, cfg)
        metric.set_storage(st)
        eng = B200Operators(SimpleNamespace(host_H=m.H, metric=SimpleNamespace(native=metric), velocity={},
                                            position={}, composite={}), cfg)
        eng.moments(B, 8, c, a)
        s0, l0 = metric.stats(), _launches()
        _, dt = _bench_call(lambda: eng.moments(B, M, c, a), torch.cuda.synchronize)
        s1 = metric.stats()
        iters = s1.max_iterations_sum - s0.max_iterations_sum
        solves = s1.calls - s0.calls
        vec = m.n * R * (16 if st == "fp64" else 8)
        # per PCG iteration: S p (read p, write Sp), update (read p, Sp, y, r; write y, r, z; y is complex128),
        # direction (read z, p; write p), and the 4x4-block S values and indices once
        s_bytes = S.nnz * 8 + S.nnz // 16 * 4
        it_bytes = 11 * vec + 2 * m.n * R * 16 + s_bytes
        out[f"storage_{st}"] = {"seconds": dt, "value": m.n * M * R / dt, "applications_per_s": m.n * R * (M - 1) / dt,
                                "metric_solves": solves, "pcg_iterations_per_solve": iters / max(solves, 1),
                                "us_per_pcg_iteration": dt / max(iters, 1) * 1e6, "gpu_launches": _launches() - l0,
                                "bytes_per_pcg_iteration": it_bytes}
        del eng, metric
        torch.cuda.empty_cache()
    best = min((k for k in out if k.startswith("storage_")), key=lambda k: out[k]["seconds"])
    out["value"] = out[best]["value"]
    peak, src = peaks()
    ach = out[best]["bytes_per_pcg_iteration"] / (out[best]["us_per_pcg_iteration"] * 1e-6) / 1e9
    out["roofline"] = {"bound": "L2/latency: the PCG working set (seven 16 MB vector blocks, 17 MB of S) is "
                                "L2-resident, so the HBM figure below is for information",
                       "kernel": "PCG iteration (pcg_spmv + pcg_update + pcg_direction)", "achieved": ach,
                       "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_source": peak_src_note(src),
                       "algorithmic_bytes_per_iteration": out[best]["bytes_per_pcg_iteration"]}
    ref = _ref_engine(m.H, S, threads, blocks=[(a0, b0, L) for a0, b0, L in blocks])
    if ref is not None:
        Bh = B.cpu().numpy()
        t_setup, t_app, _ = time_applications(lambda k: ref.core.moments(Bh, k, c, a))
        full = t_setup + (M - 1) * t_app
        out["cpu_baseline"] = {"value": m.n * M * R / full, "unit": UNIT, "cores": threads, "kind": "reference",
                               "applications_per_s": m.n * R / t_app,
                               "sample": f"Engine::moments on the full model, R={R}: one M=1 call (S B, "
                                         f"{t_setup:.2f} s) and one M=2 call (one H product + one PCG solve, "
                                         f"{t_app:.2f} s); M={M} extrapolated as set-up + {M - 1} applications"}
    return out


def config_c4(threads, ninst=32, R=16, M=64):
    """Config 4 (a sample of the batching form): a ragged batch of `ninst`
    nonorthogonal sp3 instances, cell counts log-uniform in 5..10 (4,000 to
    32,000 orbitals), on-site disorder W_i ~ U[0.1, 2] eV, kappa(S) = 50 per
    instance, block-Jacobi segmented PCG to rtol 1e-10 with complex64 CG work vectors,
    R=16, M=64, one batch call; the stated form's 256 instances of up to
    400,000 orbitals are not built (host model generation)."""
    import torch
    import scipy.linalg as la
    import scipy.sparse as sp
    from kubomsd_b200 import kpm, lattices
    from kubomsd_b200.batch import B200Batch
    rng = np.random.default_rng(4)
    cells = np.round(np.exp(rng.uniform(np.log(5), np.log(10), ninst))).astype(int)
    W = rng.uniform(.1, 2., ninst)
    ms = [lattices.diamond_sp3(cells=int(c), W=float(w), seed=100 + i) for i, (c, w) in enumerate(zip(cells, W))]
    Ss = [sp.csr_matrix(m.S) for m in ms]
    blocks = [[(a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)) for a, b in m.atom_slices]
              for m, S in zip(ms, Ss)]
    c, a = 0., 40.
    phases = [kpm.random_phases(m.n, 20261019 + i, range(R)) for i, m in enumerate(ms)]
    bt = B200Batch([m.H for m in ms], precision="mixed", overlaps=Ss, blocks=blocks, rtol=1e-10)
    B = bt.concat(phases)
    bt.moments(B, 8, c, a)
    s0, l0 = bt.metric.stats(), _launches()
    _, dt = _bench_call(lambda: bt.moments(B, M, c, a), torch.cuda.synchronize)
    s1 = bt.metric.stats()
    out = {"workload": f"config 4 sample: ragged batch of {ninst} nonorthogonal diamond sp3 instances, "
                       f"{min(m.n for m in ms):,}-{max(m.n for m in ms):,} orbitals ({bt.n:,} in total), kappa(S) "
                       f"= 50, block-Jacobi segmented PCG rtol 1e-10 (complex64 CG vectors), R={R}, M={M}",
           "unit": UNIT, "seconds": dt, "value": bt.n * M * R / dt, "gpu_launches": _launches() - l0,
           "segmented_solves": s1.calls - s0.calls,
           "pcg_iterations_per_solve": (s1.max_iterations_sum - s0.max_iterations_sum) / max(s1.calls - s0.calls, 1),
           "roofline": {"bound": "L2/latency: each instance's PCG working set is a few MB; the segmented PCG and "
                                 "step kernels cover all instances per launch", "achieved": None, "peak": None,
                        "frac": None}}
    ref_ids = [int(np.argmin(cells)), int(np.argmax(cells))]
    tot_app, tot_n = 0., 0
    for i in ref_ids:
        ref = _ref_engine(ms[i].H, Ss[i], threads, blocks=blocks[i])
        if ref is None:
            return out
        ph = phases[i]
        t_setup, t_app, _ = time_applications(lambda k: ref.core.moments(ph, k, c, a))
        tot_app += t_app
        tot_n += ms[i].n
    out["cpu_baseline"] = {"value": tot_n * R / tot_app * M / (M - 1), "unit": UNIT, "cores": threads,
                           "kind": "reference",
                           "sample": f"Engine::moments on the smallest and largest instances ({tot_n:,} orbitals), "
                                     f"R={R}: one operator application (H product + PCG solve) each, from an M=2 "
                                     f"minus an M=1 call; rate per orbital-vector application, times M/(M-1) moments "
                                     f"per application ({threads} OpenMP threads)"}
    return out


def config_c5(duration=3., rate=20., msd_fraction=.25):
    """Config 5 (a sampled window): Poisson arrivals at 20 req/s of DOS and
    stepwise-MSD jobs over resident orthogonal lattices (16k-4M sites) and
    nonorthogonal sp3 cells, M in {512, 1024, 2048}, R in {8, 32}, admitted by
    an HBM budget of 150 GB into 8 slots; p50/p99 latency and throughput."""
    from kubomsd_b200 import lattices
    from kubomsd_b200.serving import ResidentModel, Server, latency_summary, poisson_stream
    models = {
        "sq128": ResidentModel("sq128", lattices.square_lattice(128, seed=1), (-11.5, 11.5), replicas=8),
        "hc1024": ResidentModel("hc1024", lattices.honeycomb(1024, 512, seed=2), (-9.2, 9.2), replicas=8),
        "hc2048": ResidentModel("hc2048", lattices.honeycomb(2048, 1024, seed=3), (-9.2, 9.2), replicas=8),
        "sp3_8k": ResidentModel("sp3_8k", lattices.diamond_sp3(cells=4), (-40., 40.), precision="fp64",
                                replicas=8),
    }
    reqs = poisson_stream(rate, duration, models, seed=5, msd_fraction=msd_fraction, times_fs=(0., 1., 2.))
    srv = Server(models, slots=8, hbm_budget_bytes=150 * 10 ** 9)
    t0 = time.perf_counter()
    res = srv.serve(reqs)
    wall = time.perf_counter() - t0
    busy = sum(r.end - r.start for r in res)
    return {"workload": f"serving: Poisson {rate:g} req/s for a {duration:g} s window, {msd_fraction:.0%} stepwise "
                        "MSD jobs (x axis, 0/1/2 fs) and DOS jobs, M in {512,1024,2048}, R in {8,32}, models "
                        + ", ".join(f"{k} ({mm.n:,} orbitals)" for k, mm in models.items())
                        + ", 8 slots, HBM budget 150 GB",
            "latency": latency_summary(res), "requests": len(res), "errors": len(srv.errors),
            "error_messages": sorted({msg for _, msg in srv.errors})[:5],
            "jobs": {"dos": sum(r.kind == "dos" for r in res), "msd": sum(r.kind == "msd" for r in res)},
            "wall_s": wall, "requests_per_s": len(res) / wall, "offered_rate": rate,
            "slot_occupancy": busy / (8 * wall)}


def devstats_phases(n, seed, ids):
    from kubomsd_b200 import devstats
    return devstats.random_phases(n, seed, ids)


def _launches():
    from kubomsd_b200 import _abi
    return int(_abi.require_library().kmsd_kernel_launches())


def peak_src_note(src):
    return f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else src


def run_diamond(args):
    """Config 2: nonorthogonal sp3 diamond (10^3 cells x 8 atoms x 4 orbitals),
    block-Jacobi batched PCG at rtol 1e-10 in every operator application, FP64,
    R=32 vectors, M=1024 moments; work N*M*R per step."""
    import scipy.linalg as la
    import scipy.sparse as sp
    import torch
    from types import SimpleNamespace
    from kubomsd_b200 import _abi, kpm, lattices
    from kubomsd_b200.native import B200Metric, B200Operators
    lib = _abi.require_library()
    m = lattices.diamond_sp3(cells=10)
    S = sp.csr_matrix(m.S)
    blocks = [(a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)) for a, b in m.atom_slices]
    cfg = SimpleNamespace(metric_rtol=1e-10, metric_atol=0., metric_maxiter=1000, metric_residual_policy="fixed",
                          metric_check_interval=32, metric_gap_ratio=.1, metric_solver="pcg", precision="fp64",
                          moment_doubling=False)
    metric = B200Metric(S, S.diagonal().real.copy(), blocks, cfg)
    metric.set_storage(args.metric_storage)
    eng = B200Operators(SimpleNamespace(host_H=m.H, metric=SimpleNamespace(native=metric), velocity={},
                                        position={}, composite=m.composite), cfg)
    R, M = 32, args.moments if args.moments != 4096 else 1024
    bounds = (-40., 40.)
    c, a = 0., 40.
    B = torch.from_numpy(kpm.random_phases(m.n, 20261019, range(R))).cuda()
    for _ in range(args.warmup):
        eng.moments(B, min(M, 64), c, a)
    st0 = metric.stats()
    torch.cuda.synchronize()
    l0 = lib.kmsd_kernel_launches()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.steps):
        mu = eng.moments(B, M, c, a)
    e.record()
    torch.cuda.synchronize()
    st1 = metric.stats()
    ms = s.elapsed_time(e) / args.steps
    calls = st1.calls - st0.calls
    iters = st1.max_iterations_sum - st0.max_iterations_sum
    print(json.dumps({"metric": METRIC, "value": m.n * M * R / (ms / 1e3), "unit": UNIT, "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "c128",
                      "data": "synthetic (seeded diamond sp3 model, NumPy PCG64 phases)",
                      "config": {"workload": f"KPM moments, nonorthogonal diamond sp3 {m.n} orbitals, kappa(S)=50, "
                                             f"block-Jacobi PCG rtol 1e-10, R={R}, M={M}",
                                 "metric_storage": args.metric_storage,
                                 "spectral_bounds_eV": list(bounds), "metric_solves_per_step": calls / args.steps,
                                 "pcg_iterations_per_solve": iters / max(calls, 1)},
                      "gpu_launches": int(lib.kmsd_kernel_launches() - l0),
                      "mu0_over_n": float(mu[0].mean().item()) / m.n}))


def series_row_bytes(cols, real_bytes, ell_w):
    """Algorithmic bytes per row of one augmented series step (MODE_SERIES with
    the velocity applied from H's ELL row): T_k-1 read once (neighbours from
    cache), T_k-2 read, T_k written, the Bessel accumulator read and written;
    H's ELL row (column indices and values) and the velocity values aligned
    with it (real and imaginary planes)."""
    return 5 * cols * 2 * real_bytes + ell_w * (4 + real_bytes) + 2 * ell_w * real_bytes


def run_series(args):
    """The augmented series step alone: one 1 fs Bessel propagation of
    [psi | phi] (2R columns) on the honeycomb lx x ly x 2 with its explicit
    velocity along x, per step; CUDA events around the K timed propagations."""
    import torch
    from kubomsd_b200 import _abi, kpm, lattices
    from kubomsd_b200.config import RunConfig
    from kubomsd_b200.operators import build_operators
    lib = _abi.require_library()
    m = lattices.honeycomb(args.lx, args.ly)
    n, R = m.n, args.vectors
    cfg = RunConfig(energy_eV=[0.], time_fs=[0., 1.], spectral_bounds=BOUNDS, axes=("x",), include_vac=False,
                    precision=args.precision)
    ops = build_operators(m, cfg)
    B = devstats_phases(n, 20261019, range(R))
    aug = torch.cat([B, torch.zeros_like(B)], dim=1).contiguous()
    coeff, _ = kpm.bessel_coefficients(1., cfg, weighted_tail=True)
    c, a = kpm.scaling(cfg)
    for _ in range(max(args.warmup, 1)):
        res = ops.native.series(aug, coeff, c, a, [[1., 0., 0.]])
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device())
    l0 = lib.kmsd_kernel_launches()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(args.steps):
        res = ops.native.series(aug, coeff, c, a, [[1., 0., 0.]])
    e.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = s.elapsed_time(e) / args.steps
    bessel = len(coeff) - 1
    nnz = int(np.diff(m.H.tocsr().indptr).max())
    rb = series_row_bytes(2 * R, 4 if args.precision == "mixed" else 8, 4 if nnz <= 4 else 8 if nnz <= 8 else nnz)
    peak, src = peaks()
    ach = n * rb / (ms / bessel / 1e3) / 1e9
    print(json.dumps({"metric": "augmented series step (1 fs Bessel propagation of [psi | phi])",
                      "value": n * 2 * R * bessel / (ms / 1e3), "unit": "orbital·vec·step/s", "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                      "dtype": "c64" if args.precision == "mixed" else "c128", "data": "synthetic (seeded lattice)",
                      "config": {"workload": f"series step, honeycomb {args.lx}x{args.ly}x2 = {n:,} sites, "
                                             f"[psi | phi] = 2 x {R} columns, explicit velocity along x",
                                 "precision": args.precision, "bessel_steps": bessel},
                      "ms_per_bessel_step": ms / bessel, "gpu_launches": int(lib.kmsd_kernel_launches() - l0),
                      "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                   "peak_source": peak_src_note(src), "algorithmic_bytes_per_row": rb},
                      "clocks": clk, "checksum": float(res.abs().square().sum().item())}))


def run_batch(args):
    """Ragged batch of nonorthogonal instances (a sample of the 256-instance,
    4k-400k-orbital batching config): 32 diamond sp3 instances with
    log-uniform cell counts 5..10 (4,000-32,000 orbitals), disorder
    W_i ~ U[0.1, 2] eV, kappa(S)=50, block-Jacobi PCG to 1e-10, FP64, R=16,
    M=64 by default.  One batch call (one segmented PCG over all instances per
    step) is timed against separate per-instance engine calls."""
    import scipy.linalg as la
    import scipy.sparse as sp
    import torch
    from types import SimpleNamespace
    from kubomsd_b200 import _abi, kpm, lattices
    from kubomsd_b200.batch import B200Batch
    from kubomsd_b200.native import B200Metric, B200Operators
    lib = _abi.require_library()
    rng = np.random.default_rng(4)
    cells = np.round(np.exp(rng.uniform(np.log(5), np.log(10), 32))).astype(int)
    W = rng.uniform(.1, 2., 32)
    ms = [lattices.diamond_sp3(cells=int(c), W=float(w), seed=100 + i) for i, (c, w) in enumerate(zip(cells, W))]
    Hs, Ss = [m.H for m in ms], [sp.csr_matrix(m.S) for m in ms]
    blocks = [[(a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)) for a, b in m.atom_slices]
              for m, S in zip(ms, Ss)]
    R, M = 16, args.moments if args.moments != 4096 else 64
    c, a = 0., 40.
    phases = [torch.from_numpy(kpm.random_phases(m.n, 20261019 + i, range(R))).cuda() for i, m in enumerate(ms)]
    bt = B200Batch(Hs, precision=args.metric_storage, overlaps=Ss, blocks=blocks, rtol=1e-10)
    B = bt.concat(phases)
    N = bt.n
    for _ in range(args.warmup):
        bt.moments(B, min(M, 16), c, a)
    st0 = bt.metric.stats()
    torch.cuda.synchronize()
    l0 = lib.kmsd_kernel_launches()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.steps):
        mu = bt.moments(B, M, c, a)
    e.record()
    torch.cuda.synchronize()
    ms_batch = s.elapsed_time(e) / args.steps
    st1 = bt.metric.stats()
    launches = int(lib.kmsd_kernel_launches() - l0)
    solves = (st1.calls - st0.calls) / args.steps
    iters = (st1.max_iterations_sum - st0.max_iterations_sum) / max(st1.calls - st0.calls, 1)
    # the same instances through separate engine calls, one after another
    cfg = SimpleNamespace(metric_rtol=1e-10, metric_atol=0., metric_maxiter=1000, metric_residual_policy="fixed",
                          metric_check_interval=32, metric_gap_ratio=.1, metric_solver="pcg", precision="fp64",
                          moment_doubling=False)
    engines = []
    for H, S, bl in zip(Hs, Ss, blocks):
        met = B200Metric(S, S.diagonal().real.copy(), bl, cfg)
        engines.append(B200Operators(SimpleNamespace(host_H=H, metric=SimpleNamespace(native=met), velocity={},
                                                     position={}, composite={}), cfg))
    for eng, ph in zip(engines, phases):
        eng.moments(ph, 2, c, a)
    torch.cuda.synchronize()
    s.record()
    sep = [eng.moments(ph, M, c, a) for eng, ph in zip(engines, phases)]
    e.record()
    torch.cuda.synchronize()
    ms_sep = s.elapsed_time(e)
    host = lambda x: x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)  # noqa: E731
    err = max(float(np.max(np.abs(host(mu[i]) - host(sep[i]))) / float(np.max(np.abs(host(sep[i])))))
              for i in range(len(ms)))
    print(json.dumps({"metric": METRIC, "value": N * M * R / (ms_batch / 1e3), "unit": UNIT, "n_gpus": 1,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batch, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "c128",
                      "data": "synthetic (seeded diamond sp3 instances, NumPy PCG64 phases)",
                      "config": {"workload": f"ragged batch of {len(ms)} nonorthogonal diamond sp3 instances, "
                                             f"{int(min(m.n for m in ms)):,}-{int(max(m.n for m in ms)):,} orbitals "
                                             f"({N:,} in total), kappa(S)=50, block-Jacobi PCG rtol 1e-10, R={R}, "
                                             f"M={M}, FP64",
                                 "spectral_bounds_eV": [c - a, c + a], "segmented_solves_per_step": solves,
                                 "metric_storage": args.metric_storage,
                                 "pcg_iterations_per_solve": iters},
                      "gpu_launches": launches,
                      "separate_calls": {"ms": ms_sep, "value": N * M * R / (ms_sep / 1e3),
                                         "speedup_of_batch": ms_sep / ms_batch,
                                         "max_rel_diff_vs_batch": err}}))


def run_serving(args):
    """Config 5 (shortened): Poisson stream of KPM DOS jobs and stepwise MSD
    jobs (a fraction KMSD_SERVING_MSD, 0.25 by default) over resident
    orthogonal 2D lattices and nonorthogonal sp3 cells, admitted by an HBM
    budget of 150 GB into 8 concurrent slots; p50/p99 latency and the DOS
    jobs' moment throughput."""
    from kubomsd_b200 import lattices
    from kubomsd_b200.serving import ResidentModel, Server, latency_summary, poisson_stream
    models = {
        "sq128": ResidentModel("sq128", lattices.square_lattice(128, seed=1), (-11.5, 11.5), precision="mixed",
                               replicas=8),
        "hc1024": ResidentModel("hc1024", lattices.honeycomb(1024, 512, seed=2), (-9.2, 9.2),
                                precision="mixed", replicas=8),
        "hc2048": ResidentModel("hc2048", lattices.honeycomb(2048, 1024, seed=3),
                                (-9.2, 9.2), precision="mixed", replicas=8),
        "sp3_2k": ResidentModel("sp3_2k", lattices.diamond_sp3(cells=4), (-40., 40.), precision="fp64",
                                replicas=8),
    }
    duration = float(os.environ.get("KMSD_SERVING_SECONDS", "30"))
    rate = float(os.environ.get("KMSD_SERVING_RATE", "20"))
    msd = float(os.environ.get("KMSD_SERVING_MSD", "0.25"))  # fraction of stepwise MSD jobs (x axis, 0/1/2 fs)
    reqs = poisson_stream(rate, duration, models, seed=5, msd_fraction=msd, times_fs=(0., 1., 2.))
    srv = Server(models, slots=8, hbm_budget_bytes=150 * 10 ** 9)
    t0 = time.perf_counter()
    res = srv.serve(reqs)
    wall = time.perf_counter() - t0
    summ = latency_summary(res)
    omv = sum(models[r.model].n * (len(r.value) if hasattr(r.value, "__len__") else 0) * r.value.shape[1]
              for r in res if r.kind == "dos")
    print(json.dumps({"metric": METRIC, "value": omv / wall, "unit": UNIT, "n_gpus": 1, "steps": len(res),
                      "warmup": 0, "ms_per_step": wall / max(len(res), 1) * 1e3, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "c64 vectors / f64 accumulation (lattices), "
                      "c128 (sp3)", "data": "synthetic Poisson stream (seed 5)",
                      "config": {"workload": f"serving: Poisson {rate:g} req/s for {duration:g} s, {msd:.0%} "
                                             "stepwise MSD jobs, M in {512,1024,2048}, R in {8,32}, models "
                                             + ", ".join(f"{k} ({m.n:,} orbitals)" for k, m in models.items())
                                             + ", 8 slots, HBM budget 150 GB"},
                      "latency": summ, "errors": len(srv.errors), "offered_requests": len(reqs),
                      "wall_s": wall}))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "diamond":
        run_diamond(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "batch":
        run_batch(args)
        return
    if args.workload == "series":
        run_series(args)
        return
    import torch
    import torch.distributed as dist
    from types import SimpleNamespace
    from kubomsd_b200 import _abi, kpm, lattices
    from kubomsd_b200.native import B200Metric, B200Operators
    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    lib = _abi.require_library()
    m = lattices.honeycomb(args.lx, args.ly, with_velocity=False)
    n, R, M = m.n, args.vectors, args.moments
    # this rank's statistics block: sample ids rank*R .. rank*R+R-1
    from kubomsd_b200 import devstats
    B = devstats.random_phases(n, 20261019, range(rank * R, rank * R + R))  # NumPy's PCG64 stream, on the device
    host = torch.empty((n, R), dtype=torch.complex128, pin_memory=True)
    host.copy_(B)
    c, a = (BOUNDS[0] + BOUNDS[1]) / 2, (BOUNDS[1] - BOUNDS[0]) / 2

    def engine(precision, method):
        cfg = SimpleNamespace(metric_rtol=1e-10, metric_atol=0., metric_maxiter=1000,
                              metric_residual_policy="fixed", metric_check_interval=32, metric_gap_ratio=.1,
                              metric_solver="pcg", precision=precision, moment_doubling=method == "doubling")
        metric = B200Metric(m.S, np.ones(n), [], cfg)
        ops = SimpleNamespace(host_H=m.H, metric=SimpleNamespace(native=metric), velocity={}, position={},
                              composite={})
        return B200Operators(ops, cfg)

    eng = engine(args.precision, args.method)
    for _ in range(args.warmup):
        eng.moments(B, M, c, a)
    stream = torch.cuda.current_stream()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device()) if rank == 0 else None
    l0 = lib.kmsd_kernel_launches()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        mu = eng.moments(B, M, c, a)
    end.record(stream)
    torch.cuda.synchronize()
    launches = lib.kmsd_kernel_launches() - l0
    clk = clocks.stop() if clocks else None
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_step = ms / args.steps
    value = world * n * M * R / (ms_step / 1e3)
    mu_host = mu.cpu().numpy()
    assert np.allclose(mu_host[0], n, rtol=1e-6), "mu_0 must equal the vector norm N"

    # dominant kernel: one fused Chebyshev step per operator application
    C = 2 if args.precision == "mixed" else 1
    unit_bytes = 16
    row_bytes_vec = (R // C) * unit_bytes if R % C == 0 else ((R + 1) // 2) * unit_bytes
    nnz_row = m.H.nnz / n
    mat_bytes = 4 + nnz_row * (4 + (4 if args.precision == "mixed" else 8))
    passes = 3 if args.method == "doubling" else 4
    launches_per_step = (M + 1) // 2 if args.method == "doubling" else M - 1
    bytes_per_launch = n * (passes * row_bytes_vec + mat_bytes)
    avg_launch_s = (ms_step / 1e3) / launches_per_step
    achieved = bytes_per_launch / avg_launch_s / 1e9
    peak, peak_src = peaks()
    default_shape = (args.lx, args.ly, R, args.precision, args.method) == (2048, 1024, 64, "mixed", "doubling")
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": NCU_TRAFFIC_PER_LAUNCH if default_shape else None, "peak_source": peak_src,
            "kernel": "cheb_step_kernel",
            "algorithmic_bytes_per_launch": bytes_per_launch, "launches_per_step": launches_per_step,
            "bytes_per_omv": bytes_per_launch / (n * R * (2 if args.method == "doubling" else 1)),
            "timing": "moments-call time / step launches per call (includes the 3 small set-up kernels of each "
                      "call)"}

    apps_per_step = launches_per_step * R  # one operator application per step launch and column
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "applications_per_s": world * n * apps_per_step / (ms_step / 1e3),
            "value_counts": "moments: N*M*R per moments call; under the product identity each operator "
                            "application yields two moments, so applications_per_s (one application of the scaled "
                            "operator to one length-N vector = N) is value/2",
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 vectors / f64 accumulation" if args.precision == "mixed" else "c128",
            "data": "synthetic (seeded honeycomb lattice, NumPy PCG64 random phases)",
            "config": config(args, n), "roofline": roof, "gpu_launches": int(launches), "clocks": clk}

    if rank == 0:
        print(json.dumps({"partial": True, "value": value, "ms_per_step": ms_step, "roofline": roof}),
              file=sys.stderr, flush=True)
    # end to end through the reference-facing plugin call with host buffers
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    hostB = host.numpy()
    t0 = time.perf_counter()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        out = eng.moments(hostB, M, c, a)   # numpy in -> numpy out (H2D + D2H inside)
    e_end.record(stream)
    torch.cuda.synchronize()
    e_ms = e_start.elapsed_time(e_end)
    wall = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())
    assert isinstance(out, np.ndarray) and out.shape == (M, R)
    line["e2e"] = {"value": world * n * M * R / (e_ms / args.steps / 1e3), "unit": UNIT,
                   "h2d_bytes_per_step": int(n * R * 16), "d2h_bytes_per_step": int(M * R * 8),
                   "ms_per_step": e_ms / args.steps, "host_wall_ms_per_step": wall / args.steps * 1e3,
                   "call": "B200Operators.moments(numpy complex128 (N,R) from pinned memory) -> numpy (M,R)"}

    if world == 1 and not args.no_compare:
        compare = {}
        for prec, meth in (("fp64", "direct"), ("fp64", "doubling"), ("mixed", "direct")):
            if (prec, meth) == (args.precision, args.method):
                continue
            e2 = engine(prec, meth)
            e2.moments(B, M, c, a)
            torch.cuda.synchronize()
            s2, t2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s2.record(stream)
            mu2 = e2.moments(B, M, c, a)
            t2.record(stream)
            torch.cuda.synchronize()
            v2 = n * M * R / (s2.elapsed_time(t2) / 1e3)
            err = float(np.max(np.abs(mu_host - mu2.cpu().numpy())) / np.max(np.abs(mu2.cpu().numpy())))
            compare[f"{prec}_{meth}"] = {"value": v2, "ms_per_step": s2.elapsed_time(t2),
                                         "moments_relerr_vs_headline": err}
            del e2
            torch.cuda.empty_cache()
        line["compare"] = compare
        if "fp64_direct" in compare:
            line["speedup_vs_fp64_direct"] = value / compare["fp64_direct"]["value"]
        try:
            line["msd_check"] = msd_check()
        except Exception as exc:  # noqa: BLE001 - reported, not fatal to the timing line
            line["msd_check"] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(m.H, n, len(os.sched_getaffinity(0)), R, M)
    if rank == 0 and world == 1 and not args.no_configs:
        threads = len(os.sched_getaffinity(0))
        configs = {}
        for name, fn in (("c1", lambda: config_c1(threads)), ("c2", lambda: config_c2(threads)),
                         ("c3_msd", lambda: config_c3_msd(threads)), ("c4", lambda: config_c4(threads)),
                         ("c5", config_c5)):
            try:
                configs[name] = fn()
            except Exception as exc:  # noqa: BLE001 - reported, not fatal to the headline line
                configs[name] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.empty_cache()
        line["configs"] = configs
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def msd_check():
    """Mixed vs FP64 stepwise MSD on the 64x64 square lattice (R=8, M=512,
    0-10 fs): the tolerance the mixed form is held to (untimed)."""
    import torch
    from kubomsd_b200 import kpm, lattices, stochastic
    from kubomsd_b200.config import RunConfig
    from kubomsd_b200.operators import build_operators
    m = lattices.square_lattice(64)
    B = kpm.random_phases(m.n, 20261019, range(8))
    out = {}
    for prec in ("fp64", "mixed"):
        cfg = RunConfig(energy_eV=np.linspace(-11, 11, 201), time_fs=np.arange(11.), spectral_bounds=(-11.2, 11.2),
                        n_moments=512, axes=("x",), include_vac=False, stochastic_method="stepwise", precision=prec)
        ops = build_operators(m, cfg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dos, nums, _ = stochastic.stepwise_samples(ops, cfg, B)
        out[prec] = (dos, nums["msd_A2/commutator"], time.perf_counter() - t0)
    d64, m64, t64 = out["fp64"]
    d32, m32, t32 = out["mixed"]
    return {"case": "64x64 square, R=8, M=512, 0-10 fs dt=1 fs, 201 energies",
            "msd_relerr": float(np.max(np.abs(m32 - m64)) / np.max(np.abs(m64))),
            "dos_relerr": float(np.max(np.abs(d32 - d64)) / np.max(np.abs(d64))),
            "fp64_seconds": t64, "mixed_seconds": t32}


if __name__ == "__main__":
    main()
