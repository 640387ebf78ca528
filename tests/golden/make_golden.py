"""Generate the golden fixtures of tests/golden/ by running the REFERENCE.

Runs KuboMSD's own Python solver layer (src/kubo_msd: build_operators,
stepwise_samples, iter_stochastic_blocks, ...) on top of its compiled CPU
engine cpp/native.cpp, built into oracle/_ref/ by oracle/build_ref.sh, with
`cpu_kernel="cpp"` — the reference's production CPU path.  The outputs are
stored as small .npz files together with their inputs; tests compare the B200
engine and the oracle restatement against them.  Needs the reference checkout:
$KUBOMSD_REFERENCE, else a directory named `reference` beside this
repository; h5py is not needed because only the solver layer is driven.

    python tests/golden/make_golden.py            # every case
    python tests/golden/make_golden.py c3_fp64    # named cases only

The stated-configuration cases (c1_square64_full, c3_honeycomb_fp64,
c2_diamond10) run the full-size lattices of the precision form and the
nonorthogonal model at reduced moment and vector counts; they take minutes.
"""
from __future__ import annotations

import hashlib
import os
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np
import scipy.linalg as la
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
REF = Path(os.environ.get("KUBOMSD_REFERENCE", ROOT.parent / "reference"))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(REF / "src"))
sys.path.insert(0, str(REF))

from oracle import ref_native  # noqa: E402

ref_native.build()
import kubo_msd  # noqa: E402

kubo_msd.__path__.append(str(ref_native.REF_DIR))  # kubo_msd._native from oracle/_ref
import kubo_msd._native  # noqa: E402

ref_native._module = kubo_msd._native  # one registration of the pybind classes for both routes

from kubo_msd.config import RunConfig  # noqa: E402
from kubo_msd.contracts import ModelBundle  # noqa: E402
from kubo_msd.metric.sampling import MetricSampler, random_phases  # noqa: E402
from kubo_msd.metric.solve import MetricSolver  # noqa: E402
from kubo_msd.operators.velocity import build_operators  # noqa: E402
from kubo_msd.solvers.chebyshev import bessel_coefficients, scaling  # noqa: E402
from kubo_msd.solvers.stepwise import propagate, stepwise_samples  # noqa: E402
from kubo_msd.solvers.spectral import spectral_samples  # noqa: E402
from kubo_msd.solvers.stochastic import iter_stochastic_blocks  # noqa: E402
from kubo_msd.kernels.energy import jackson_coefficients, reconstruction_matrix  # noqa: E402

from kubomsd_b200 import lattices  # noqa: E402


def csr_arrays(prefix, A):
    A = sp.csr_matrix(A, dtype=np.complex128)
    A.sum_duplicates()
    A.sort_indices()
    return {f"{prefix}_indptr": A.indptr.astype(np.int64), f"{prefix}_indices": A.indices.astype(np.int64),
            f"{prefix}_data": A.data, f"{prefix}_shape": np.array(A.shape)}


def digest(A):
    A = sp.csr_matrix(A, dtype=np.complex128)
    A.sum_duplicates()
    A.sort_indices()
    h = hashlib.sha256()
    for v in (A.indptr.astype(np.int64), A.indices.astype(np.int64), A.data):
        h.update(np.ascontiguousarray(v).tobytes())
    return h.hexdigest()


def small_model(kind, n=10, seed=7331):
    """Dense complex Hermitian H, SPD S = I + 0.03 A^H A, position/velocity X."""
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    S = np.eye(n) + .03 * (A.conj().T @ A)
    H = (A + A.conj().T) / 10
    X = np.diag(np.linspace(-.6, .9, n)).astype(complex) + .02 * (A + A.conj().T)
    if kind == "velocity":
        return ModelBundle(H, S, velocity={"x": X}, atom_slices=[(0, 3), (3, 6), (6, 10)])
    if kind == "position":
        return ModelBundle(H, S, position={"x": X}, atom_slices=[(0, 3), (3, 6), (6, 10)])
    r = np.linspace(0, 2.5, n)
    comp = (H * (r[None, :] - r[:, None]), X - r[:, None] * S, X - S * r[None, :])
    return ModelBundle(H, S, composite={"x": comp}, atom_slices=[(0, 3), (3, 6), (6, 10)])


def base_config(**kw):
    values = dict(energy_eV=[-.4, -.1, .2, .5], time_fs=[0, .08, .2], solver="stochastic-kpm",
                  kernel="jackson", axes=("x",), spectral_bounds=(-2.5, 2.5), n_moments=24, metric_rtol=2e-13,
                  sampling_tol=1e-12, segment_fs=.07, include_vac=False, cpu_kernel="cpp",
                  stochastic_method="stepwise")
    values.update(kw)
    return RunConfig(**values)


def engine_case(kind, precond):
    m = small_model(kind)
    cfg = base_config(preconditioner=precond)
    ops = build_operators(m, cfg)
    assert ops.native is not None and ops.metric.native is not None
    rng = np.random.default_rng(4242)
    n = m.n_orbitals
    B = rng.normal(size=(n, 3)) + 1j * rng.normal(size=(n, 3))
    c, a = scaling(cfg)
    coeff, _ = bessel_coefficients(.07, cfg, weighted_tail=True)
    aug = np.concatenate([B, rng.normal(size=(n, 3)) + 1j * rng.normal(size=(n, 3))], axis=1)
    out = dict(B=B, aug=aug, coeff=coeff, center=c, half=a, rtol=cfg.metric_rtol,
               H=np.asarray(m.H_cov), S=np.asarray(m.S),
               blocks_L=np.array([np.pad(L, ((0, 4 - L.shape[0]), (0, 4 - L.shape[0])))
                                  for _, _, L in ops.metric.host_setup.blocks]) if precond == "block-jacobi"
               else np.zeros((0, 4, 4)),
               blocks_start=np.array([0] + [b for _, b, _ in ops.metric.host_setup.blocks]) if precond ==
               "block-jacobi" else np.zeros(0, np.int64))
    if kind == "velocity":
        out["V"] = np.asarray(m.velocity["x"])
    elif kind == "position":
        out["X"] = np.asarray(m.position["x"])
    else:
        out["bond"], out["xbar"], out["delta"] = (np.asarray(x) for x in m.composite["x"])
    out["h_action"] = ops.native.h_action(B)
    out["v_cov"] = ops.native.v_cov([1., 0., 0.], B)
    out["chain"] = ops.native.chain(B, 12, c, a)
    out["moments"] = ops.native.moments(B, 20, c, a)
    out["series_plain"] = ops.native.series(B, coeff, c, a)
    out["series_aug"] = ops.native.series(aug, coeff, c, a, [[1., 0., 0.]])
    y, rep = ops.metric.solve_s(B)
    out["solve"] = y
    out["solve_iterations"] = np.asarray(rep.iterations)
    out["solve_relative"] = np.asarray(rep.relative_residual)
    sampler = MetricSampler(ops.metric, cfg)
    xi = random_phases(n, 11, [0, 1, 2])
    out["xi"] = xi
    out["sample_coeff"] = np.asarray(sampler.coeff)
    out["sample_center"] = sampler.center
    out["sample_half"] = sampler.half
    out["sample"] = sampler.transform(xi)
    out["propagate"] = propagate(B, .2, ops, cfg)[0]
    dos, nums, _ = stepwise_samples(ops, cfg, B)
    out["dos"] = dos
    out["msd"] = nums["msd_A2/commutator"]
    vcfg = replace(cfg, include_vac=True, integration_dt_fs=.01)
    _, vac, _ = spectral_samples(ops, vcfg, B)
    for key, value in vac.items():
        out["spectral/" + key] = value
    out["integration_dt_fs"] = vcfg.integration_dt_fs
    out["energies"] = np.asarray(cfg.energy_eV)
    out["times"] = np.asarray(cfg.time_fs)
    out["n_moments"] = cfg.n_moments
    out["segment_fs"] = cfg.segment_fs
    out["bounds"] = np.asarray(cfg.spectral_bounds)
    return out


def pcg_known():
    out = {}
    cfg = base_config()
    from types import SimpleNamespace
    solver = MetricSolver(np.array([[1., .2], [.2, 2.]]), cfg)
    y, rep = solver.solve_s(np.ones((2, 1)), SimpleNamespace(rtol=.5, metric_atol=0., metric_maxiter=1))
    out["one_step"] = y
    out["one_step_iterations"] = np.asarray(rep.iterations)
    solver = MetricSolver(np.array([[1, .2j], [-.2j, 2]]), base_config(metric_maxiter=1))
    try:
        solver.solve_s(np.array([[0, 1], [0, 1]], complex))
    except ValueError as exc:
        d = exc.diagnostics
        out["fail_converged"] = np.array(d["converged"])
        out["fail_iterations"] = np.array(d["iterations"])
        out["fail_message"] = np.array(str(exc))
    rng = np.random.default_rng(97)
    A = rng.normal(size=(11, 11)) + 1j * rng.normal(size=(11, 11))
    S = A.conj().T @ A + 2 * np.eye(11)
    B = rng.normal(size=(11, 4)) + 1j * rng.normal(size=(11, 4))
    B *= [0, 1e-180, 1, 1e180]
    out["scaled_S"] = S
    out["scaled_B"] = B
    for pre in ("diagonal", "block-jacobi"):
        s = MetricSolver(S, base_config(preconditioner=pre), atom_slices=[(0, 3), (3, 7), (7, 11)])
        y, rep = s.solve_s(B)
        out[f"scaled_{pre}"] = y
        out[f"scaled_{pre}_iterations"] = np.asarray(rep.iterations)
    # a tridiagonal metric long enough to exercise the 32-iteration refresh
    n = 96
    T = sp.diags([-np.ones(n - 1), 2.03 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="csr", dtype=complex)
    Bt = (rng.normal(size=(n, 3)) + 1j * rng.normal(size=(n, 3)))
    s = MetricSolver(T, base_config(metric_rtol=1e-11, metric_maxiter=1000))
    y, rep = s.solve_s(Bt)
    out["tri_B"] = Bt
    out["tri"] = y
    out["tri_iterations"] = np.asarray(rep.iterations)
    out["tri_refreshes"] = s.diagnostics()["true_residual_refreshes"]
    for pol in ("adaptive",):
        s = MetricSolver(T, base_config(metric_rtol=1e-11, metric_maxiter=1000, metric_residual_policy=pol))
        y, rep = s.solve_s(Bt)
        out[f"tri_{pol}"] = y
        out[f"tri_{pol}_iterations"] = np.asarray(rep.iterations)
    return out


TIME_GRIDS = [(50., 1.), (1., .1), (.3, .1), (10., .7), (5., .5), (0., 1.), (2., 3.), (100., .01), (7.3, .25)]
ENERGY_GRIDS = [(-11., 11., 201), (-9., 9., 201), (-1., 1., 2), (-40., 40., 13), (.1, .7, 7)]


def config_case():
    """The reference's output grids (config.py:14-24): time grids from (tmax,
    dt) and energy grids from (emin, emax, n), which must match bit for bit."""
    from kubo_msd.config import resolve_output_grid, resolve_time_grid
    out = {}
    for i, (tmax, dt) in enumerate(TIME_GRIDS):
        out[f"time_{i}"] = np.asarray(resolve_time_grid(tmax, dt))
    for i, (a, b, n) in enumerate(ENERGY_GRIDS):
        out[f"energy_{i}"] = np.asarray(resolve_output_grid(a, b, n))
    out["time_inputs"] = np.asarray(TIME_GRIDS)
    out["energy_inputs"] = np.asarray(ENERGY_GRIDS)
    return out


def statistics_case():
    """The reference's paired block bootstrap (observables/statistics.py:5-22)
    on seeded block sums: 9 blocks of unequal counts over (axis, time,
    energy), a denominator of shape (blocks, 1) broadcast over the energies,
    and one energy whose denominator vanishes in some resamples."""
    from kubo_msd.observables.statistics import estimate_ratio
    rng = np.random.default_rng(3)
    out = {"A": rng.random((9, 2, 4, 7)), "D": rng.random((9, 7)) + .5, "counts": rng.integers(1, 5, 9)}
    out["value"], out["stderr"], _ = estimate_ratio(out["A"], out["D"], out["counts"])
    out["A2"], out["D2"], out["counts2"] = rng.random((5, 6)), rng.random((5, 1)) + .2, np.array([3, 1, 4, 1, 5])
    out["value2"], out["stderr2"], _ = estimate_ratio(out["A2"], out["D2"], out["counts2"])
    D3 = rng.random((4, 3)) + .1
    D3[1:, 2] = 0.
    out["A3"], out["D3"], out["counts3"] = rng.random((4, 3)), D3, np.array([2, 2, 2, 2])
    out["value3"], out["stderr3"], _ = estimate_ratio(out["A3"], out["D3"], out["counts3"])
    return out


def host_formulas():
    out = {}
    cfg = base_config(spectral_bounds=(-11.2, 11.2))
    for tag, dt, w in (("a", 1., True), ("b", .3, False), ("c", .07, True)):
        b, d = bessel_coefficients(dt, cfg, weighted_tail=w)
        out[f"bessel_{tag}"] = b
    for L in (1, 2, 64, 1024):
        out[f"jackson_{L}"] = jackson_coefficients(L)
    out["G"] = reconstruction_matrix(np.linspace(-11, 11, 41), (-11.2, 11.2), 128)
    out["phases"] = random_phases(16, 7, [0, 1, 2, 5])
    out["phases_c1_head"] = random_phases(4096, 20261019, [0, 7])[:256]
    return out


def square_pipeline(method="stepwise", include_vac=False):
    """Full reference stochastic pipeline on a 16x16 square lattice."""
    m = lattices.square_lattice(16, seed=99)
    model = ModelBundle(m.H, m.S, velocity=m.velocity)
    cfg = RunConfig(energy_eV=np.linspace(-9, 9, 19), time_fs=[0., 1., 2., 3.], solver="stochastic-kpm",
                    kernel="jackson", axes=("x",), spectral_bounds=(-11.5, 11.5), n_moments=64, nsamples=8,
                    sample_batch=4, statistics_block=2, include_vac=include_vac, stochastic_method=method,
                    cpu_kernel="cpp", seed=515, integration_dt_fs=.05)
    ops = build_operators(model, cfg)
    blocks = list(iter_stochastic_blocks(ops, cfg, method))
    out = {"H_digest": np.array(digest(m.H)), "V_digest": np.array(digest(m.velocity["x"]))}
    for blk in blocks:
        for k, v in {**blk.static, **blk.arrays}.items():
            out["arr/" + k] = np.asarray(v)
    return out


def c1_case():
    """Config-1 lattice: 64x64 square, R=8 phases, M=512 moments, short MSD."""
    m = lattices.square_lattice(64)
    model = ModelBundle(m.H, m.S, velocity=m.velocity)
    cfg = RunConfig(energy_eV=np.linspace(-11, 11, 201), time_fs=[0., 1., 2., 3.], solver="stochastic-kpm",
                    kernel="jackson", axes=("x",), spectral_bounds=(-11.2, 11.2), n_moments=512,
                    include_vac=False, stochastic_method="stepwise", cpu_kernel="cpp", omp_threads=8)
    ops = build_operators(model, cfg)
    B = random_phases(m.n, 20261019, range(8))
    c, a = scaling(cfg)
    out = {"H_digest": np.array(digest(m.H)), "V_digest": np.array(digest(m.velocity["x"]))}
    out["moments"] = ops.native.moments(B, 512, c, a)
    dos, nums, diag = stepwise_samples(ops, cfg, B)
    out["dos"] = dos
    out["msd"] = nums["msd_A2/commutator"]
    return out


def diamond_case():
    m = lattices.diamond_sp3(cells=2)
    model = ModelBundle(m.H, m.S, composite=m.composite, atom_slices=m.atom_slices)
    cfg = RunConfig(energy_eV=np.linspace(-8, 6, 8), time_fs=[0., .5, 1.], solver="stochastic-kpm",
                    kernel="jackson", axes=("x", "y", "z"), spectral_bounds=(-40., 40.), n_moments=32,
                    include_vac=False, stochastic_method="stepwise", cpu_kernel="cpp", metric_rtol=1e-12,
                    preconditioner="block-jacobi", segment_fs=.5, omp_threads=8)
    ops = build_operators(model, cfg)
    sampler = MetricSampler(ops.metric, cfg)
    xi = random_phases(m.n, 3, [0, 1])
    c, a = scaling(cfg)
    out = {"H_digest": np.array(digest(m.H)), "S_digest": np.array(digest(m.S)),
           "bounds": np.asarray(cfg.spectral_bounds)}
    out["xi"] = xi
    out["sample_coeff"] = np.asarray(sampler.coeff)
    out["sample_center"] = sampler.center
    out["sample_half"] = sampler.half
    out["sample"] = sampler.transform(xi)
    B = xi  # unit-modulus phases drive the transport checks below
    out["B"] = B
    out["moments"] = ops.native.moments(B, 32, c, a)
    out["v_cov_y"] = ops.native.v_cov([0., 1., 0.], B)
    dos, nums, _ = stepwise_samples(ops, cfg, B)
    out["dos"] = dos
    out["msd"] = nums["msd_A2/commutator"]
    out["metric_calls"] = ops.metric.diagnostics()["calls"]
    return out


def c1_full_case():
    """Config 1 in full: 64x64 square lattice, R=8, M=512, 201 energies,
    stepwise MSD along x over 0-50 fs at dt = 1 fs, no VAC."""
    m = lattices.square_lattice(64)
    model = ModelBundle(m.H, m.S, velocity=m.velocity)
    cfg = RunConfig(energy_eV=np.linspace(-11, 11, 201), time_fs=np.arange(51.), solver="stochastic-kpm",
                    kernel="jackson", axes=("x",), spectral_bounds=(-11.2, 11.2), n_moments=512,
                    include_vac=False, stochastic_method="stepwise", cpu_kernel="cpp", omp_threads=OMP)
    ops = build_operators(model, cfg)
    B = random_phases(m.n, 20261019, range(8))
    dos, nums, diag = stepwise_samples(ops, cfg, B)
    return {"H_digest": np.array(digest(m.H)), "V_digest": np.array(digest(m.velocity["x"])), "dos": dos,
            "msd": nums["msd_A2/commutator"], "time_fs": np.asarray(cfg.time_fs)}


def c3_fp64_case():
    """Precision-form lattice at full size: honeycomb 2048 x 1024 cells x 2 =
    4,194,304 sites, W = 1 eV; the reference engine's FP64 moments
    (Engine::moments, cpp/native.cpp:590-609) of R=8 phase vectors (sample ids
    0..7, seed 20261019), M=16, window (-9.2, 9.2) eV."""
    m = lattices.honeycomb(2048, 1024, with_velocity=False)
    eng = ref_native.RefEngine(m.H, sp.identity(m.n, format="csr"), threads=OMP)
    B = random_phases(m.n, 20261019, range(8))
    c, a = 0., 9.2
    return {"H_digest": np.array(digest(m.H)), "moments": eng.core.moments(B, 16, c, a), "center": c, "half": a}


def c2_full_case():
    """Config-2 model at full size: diamond sp3, 10^3 cells x 8 atoms x 4
    orbitals = 32,000 orbitals, kappa(S) = 50, block-Jacobi PCG.  The solves
    are tightened to rtol 1e-12 (the reference's own parity tests tighten
    theirs to 2e-13) so that solve tolerance does not mask the comparison.
    S^-1/2 sampling of R=4 phases, M=8 moments, v_cov along x, and a short
    stepwise MSD (x, y, z; 0, 0.5, 1 fs; M=16) of R=2 vectors."""
    m = lattices.diamond_sp3(cells=10)
    model = ModelBundle(m.H, m.S, composite=m.composite, atom_slices=m.atom_slices)
    cfg = RunConfig(energy_eV=np.linspace(-30, 30, 13), time_fs=[0., .5, 1.], solver="stochastic-kpm",
                    kernel="jackson", axes=("x", "y", "z"), spectral_bounds=(-40., 40.), n_moments=16,
                    include_vac=False, stochastic_method="stepwise", cpu_kernel="cpp", metric_rtol=1e-12,
                    preconditioner="block-jacobi", segment_fs=.5, omp_threads=OMP)
    ops = build_operators(model, cfg)
    sampler = MetricSampler(ops.metric, cfg)
    xi = random_phases(m.n, 20261019, range(4))
    c, a = scaling(cfg)
    out = {"H_digest": np.array(digest(m.H)), "S_digest": np.array(digest(m.S)),
           "sample_coeff": np.asarray(sampler.coeff), "sample_center": sampler.center,
           "sample_half": sampler.half}
    out["sample"] = sampler.transform(xi)
    out["moments"] = ops.native.moments(xi, 8, c, a)
    out["v_cov_x"] = ops.native.v_cov([1., 0., 0.], xi[:, :2])
    dos, nums, _ = stepwise_samples(ops, cfg, xi[:, :2])
    out["dos"] = dos
    out["msd"] = nums["msd_A2/commutator"]
    return compact_rows(out, ("sample", "v_cov_x"))


ROW_STRIDE = 16


def compact_rows(out, names):
    """Keeps the fixture small: for each (N, b) array, every ROW_STRIDE-th row
    plus the whole array's column sums and column norms."""
    for name in names:
        full = np.asarray(out.pop(name))
        out[name + "_rows"] = full[::ROW_STRIDE]
        out[name + "_colsum"] = full.sum(axis=0)
        out[name + "_colnorm"] = np.linalg.norm(full, axis=0)
    out["row_stride"] = np.array(ROW_STRIDE)
    return out


OMP = os.cpu_count() or 1

CASES = {
    **{f"engine_{kind}_{pre}": (lambda kind=kind, pre=pre: engine_case(kind, pre))
       for kind in ("velocity", "position", "composite") for pre in ("diagonal", "block-jacobi")},
    "pcg_known": pcg_known,
    "host_formulas": host_formulas,
    "statistics": statistics_case,
    "config": config_case,
    "square16_pipeline": square_pipeline,
    "square16_pipeline_vac": lambda: square_pipeline("stepwise", include_vac=True),
    "square16_pipeline_spectral": lambda: square_pipeline("spectral", include_vac=False),
    "c1_square64": c1_case,
    "diamond2": diamond_case,
    "c1_square64_full": c1_full_case,
    "c3_honeycomb_fp64": c3_fp64_case,
    "c2_diamond10": c2_full_case,
}


def main(names):
    import time
    for name in names or CASES:
        t0 = time.perf_counter()
        arrays = CASES[name]()
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print(name, sum(np.asarray(v).nbytes for v in arrays.values()), "bytes",
              f"{time.perf_counter() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
