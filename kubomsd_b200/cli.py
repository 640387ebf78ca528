"""`python -m kubomsd_b200 run ...`: the reference's `kubomsd run` option
surface (src/kubo_msd/cli.py:10-40, 73-95) for the stochastic-KPM solver on the
B200 backend.

Every option of the reference's `run` command is accepted under the same
name.  `--solver stochastic` is an alias of `stochastic-kpm`.  Two options are
added: `--precision {fp64,mixed}` and `--moment-doubling`.  Options selecting
paths outside this backend exit with status 2 and a message, as the reference
does for invalid input: the exact solver, the hybrid backend, and the
Cholesky / cluster-Jacobi / IC(0) metric solvers.  Multi-GPU runs use
`--transport-distribution torch` under torchrun, one process per GPU.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from . import __version__


def parser():
    p = argparse.ArgumentParser(prog="kubomsd-b200", description="Stochastic-KPM Kubo MSD transport on B200 GPUs; "
                                                                  "energies are absolute eV.")
    p.add_argument("--version", action="version", version="kubomsd-b200 " + __version__)
    sub = p.add_subparsers(dest="command", required=True)
    run = sub.add_parser("run", help="compute transport from model.json")
    run.add_argument("--input", required=True, type=Path)
    run.add_argument("--out", required=True, type=Path)
    run.add_argument("--solver", choices=["exact", "stochastic-kpm", "stochastic"], default="exact")
    run.add_argument("--backend", choices=["cpu", "hybrid", "gpu"], default="gpu")
    run.add_argument("--kernel", choices=["gaussian", "jackson"], default="gaussian")
    run.add_argument("--stochastic-method", choices=["auto", "stepwise", "spectral"], default="auto")
    run.add_argument("--metric-residual-policy", choices=["fixed", "adaptive"], default="fixed")
    run.add_argument("--metric-check-interval", type=int, default=32)
    run.add_argument("--metric-gap-ratio", type=float, default=.1)
    run.add_argument("--metric-solver", choices=["pcg", "cholesky"], default="pcg")
    run.add_argument("--metric-refine-maxiter", type=int, default=3)
    run.add_argument("--metric-partition-file")
    run.add_argument("--metric-ic-ordering", choices=["rcm", "natural"], default="rcm")
    run.add_argument("--metric-ic-shift-max", type=float, default=1e-2)
    run.add_argument("--metric-gpu-check-batch", type=int, default=1)
    run.add_argument("--cpu-kernel", choices=["cpp", "reference"], default="cpp")
    run.add_argument("--omp-threads", type=int, default=1)
    run.add_argument("--transport-distribution", choices=["serial", "mpi", "torch"], default="serial")
    run.add_argument("--emin", type=float)
    run.add_argument("--emax", type=float)
    run.add_argument("--n-energy", type=int, default=201)
    run.add_argument("--energy-grid", type=Path)
    run.add_argument("--time-grid", type=Path)
    run.add_argument("--tmax-fs", type=float)
    run.add_argument("--dt-fs", type=float)
    run.add_argument("--sigma-ev", type=float, default=.05)
    run.add_argument("--n-moments", type=int, default=256)
    run.add_argument("--spectral-min", type=float)
    run.add_argument("--spectral-max", type=float)
    run.add_argument("--axes", default="x,y,z")
    run.add_argument("--axes-vectors", type=Path)
    run.add_argument("--initial-state-selection", choices=["all", "window"], default="all")
    run.add_argument("--buffer-ev", type=float, default=0.)
    for name, default in [("nsamples", 64), ("seed", 20261019), ("sample-batch", 8), ("statistics-block", 8),
                          ("pair-block", 128), ("time-block", 16), ("energy-block", 256), ("metric-maxiter", 1000),
                          ("sampling-max-order", 4096), ("propagation-max-order", 4096)]:
        run.add_argument("--" + name, type=int, default=default)
    for name, default in [("metric-rtol", 1e-10), ("metric-atol", 0.), ("sampling-tol", 1e-10),
                          ("propagation-tol", 1e-12), ("segment-fs", 1.), ("integration-dt-fs", .01),
                          ("rho-abs", 0.), ("rho-rel", 1e-12), ("memory-limit-gb", 4.)]:
        run.add_argument("--" + name, type=float, default=default)
    run.add_argument("--preconditioner", choices=["diagonal", "block-jacobi", "full-cholesky", "cluster-jacobi",
                                                  "ic0"], default="diagonal")
    run.add_argument("--no-vac", action="store_true")
    run.add_argument("--exact-projection-kernel", choices=["sparse", "dense"], default="sparse")
    run.add_argument("--npz", action="store_true")
    run.add_argument("--efermi-ev", type=float)
    run.add_argument("--efermi-source")
    run.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    run.add_argument("--moment-doubling", action="store_true")
    run.add_argument("--spectral-bounds-method", choices=["arpack", "device-lanczos"], default="arpack",
                     help="host ARPACK (the reference's estimate) or Lanczos on the device")
    sub.add_parser("capabilities", help="report the B200 backend's availability")
    return p


def _config(args):
    from .config import RunConfig, resolve_output_grid, resolve_time_grid
    from .errors import KuboMSDError
    solver = "stochastic-kpm" if args.solver in ("stochastic", "stochastic-kpm") else args.solver
    if solver != "stochastic-kpm":
        raise KuboMSDError("the B200 backend implements --solver stochastic-kpm (exact stays in KuboMSD)")
    if args.backend == "hybrid":
        raise KuboMSDError("stochastic-kpm requires Jackson, cpu/gpu, full-space sampling")
    if args.kernel != "jackson":
        raise KuboMSDError("stochastic-kpm requires Jackson, cpu/gpu, full-space sampling")
    if args.metric_solver != "pcg" or args.preconditioner not in ("diagonal", "block-jacobi"):
        raise KuboMSDError("the B200 backend implements PCG with diagonal or block-jacobi preconditioning")
    if args.energy_grid:
        if args.emin is not None or args.emax is not None:
            raise KuboMSDError("--energy-grid excludes --emin/--emax")
        E = json.loads(args.energy_grid.read_text())
    else:
        if args.emin is None or args.emax is None:
            raise KuboMSDError("provide --emin and --emax, or --energy-grid")
        E = resolve_output_grid(args.emin, args.emax, args.n_energy)
    if args.time_grid:
        if args.tmax_fs is not None or args.dt_fs is not None:
            raise KuboMSDError("--time-grid excludes --tmax-fs/--dt-fs")
        T = json.loads(args.time_grid.read_text())
    else:
        T = resolve_time_grid(50. if args.tmax_fs is None else args.tmax_fs, .1 if args.dt_fs is None else args.dt_fs)
    if (args.spectral_min is None) != (args.spectral_max is None):
        raise KuboMSDError("both --spectral-min and --spectral-max required")
    bounds = None if args.spectral_min is None else (args.spectral_min, args.spectral_max)
    axes = tuple(a.strip() for a in args.axes.split(","))
    vectors = json.loads(args.axes_vectors.read_text()) if args.axes_vectors is not None else None
    return RunConfig(energy_eV=E, time_fs=T, solver=solver, backend="gpu", kernel=args.kernel,
                     sigma_eV=args.sigma_ev, n_moments=args.n_moments, spectral_bounds=bounds, axes=axes,
                     axes_vectors=vectors, initial_state_selection=args.initial_state_selection,
                     stochastic_method=args.stochastic_method, nsamples=args.nsamples, seed=args.seed,
                     sample_batch=args.sample_batch, statistics_block=args.statistics_block,
                     time_block=args.time_block, metric_rtol=args.metric_rtol, metric_atol=args.metric_atol,
                     metric_maxiter=args.metric_maxiter, metric_solver=args.metric_solver,
                     metric_residual_policy=args.metric_residual_policy,
                     metric_check_interval=args.metric_check_interval, metric_gap_ratio=args.metric_gap_ratio,
                     preconditioner=args.preconditioner, sampling_tol=args.sampling_tol,
                     sampling_max_order=args.sampling_max_order, propagation_tol=args.propagation_tol,
                     propagation_max_order=args.propagation_max_order, segment_fs=args.segment_fs,
                     integration_dt_fs=args.integration_dt_fs, include_vac=not args.no_vac, rho_abs=args.rho_abs,
                     rho_rel=args.rho_rel, memory_limit_gb=args.memory_limit_gb, precision=args.precision,
                     moment_doubling=args.moment_doubling, output_npz=args.npz,
                     bounds_method=args.spectral_bounds_method,
                     transport_distribution=args.transport_distribution)


def run_input(input_path, cfg, out):
    """Load, build, transport and write (src/kubo_msd/dispatch.py:21-62)."""
    from .io import ResultsWriter, load_model
    from .operators import build_operators
    from .parallel import ParallelContext
    from .stochastic import choose_stochastic_method, iter_stochastic_blocks
    ctx = ParallelContext(distributed=cfg.transport_distribution == "torch")
    start = time.perf_counter()
    sink = ResultsWriter(out, cfg) if ctx.root else None
    try:
        model = load_model(input_path)
        loaded = time.perf_counter()
        ops = build_operators(model, cfg)
        built = time.perf_counter()
        method = choose_stochastic_method(cfg)
        for block in iter_stochastic_blocks(ops, cfg, method, parallel=ctx):
            if ctx.root:
                sink.append(block)
        summary = {"output_path": str(out), "run_status": "complete", "method": method, "backend": "gpu (B200)",
                   "diagnostics": {"h_action_calls": ops.h_calls, "v_cov_calls": ops.v_calls,
                                   "metric": ops.metric.diagnostics(),
                                   "velocity_hermiticity": ops.velocity_hermiticity}}
        if ctx.root:
            sink.metadata["initialization"] = {"input_seconds": loaded - start,
                                               "operators_and_metric_seconds": built - loaded}
            sink.metadata["performance_end_to_end_seconds"] = time.perf_counter() - start
            sink.finalize(summary)
        return summary
    except BaseException:
        if sink is not None:
            sink.__exit__(*sys.exc_info())
        raise


def main(argv=None):
    args = parser().parse_args(argv)
    if args.command == "capabilities":
        info = {"version": __version__, "stochastic_kpm": "B200 CUDA engine (libkmsd_b200.so)"}
        try:
            from . import _abi
            lib = _abi.require_library()
            info["library"] = json.loads(lib.kmsd_build_info().decode())
            import torch
            info["gpu"] = torch.cuda.get_device_name() if torch.cuda.is_available() else "unavailable"
        except Exception as exc:  # noqa: BLE001
            info["library"] = {"available": False, "reason": str(exc)}
        print(json.dumps(info, indent=2))
        return 0
    try:
        cfg = _config(args)
        summary = run_input(args.input, cfg, args.out)
        print(json.dumps({"run_status": summary["run_status"], "method": summary["method"],
                          "backend": summary["backend"], "output": str(args.out),
                          "scientific_convergence": "separate; see metadata.json"}, indent=2))
        return 0
    except (ValueError, OSError, KeyError, TypeError, MemoryError) as exc:
        print(f"kubomsd-b200: {type(exc).__name__}: {exc}", file=sys.stderr)
        return 2


if __name__ == "__main__":
    raise SystemExit(main())
