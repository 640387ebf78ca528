"""Run controls of the stochastic path, field-compatible with KuboMSD's RunConfig.

`RunConfig` keeps the reference's field names, defaults and validation rules
for everything the stochastic-KPM transport reads (src/kubo_msd/config.py:26-147)
and adds two B200 fields:

* ``precision``: ``"fp64"`` (the reference's arithmetic) or ``"mixed"``
  (complex64 vectors and SpMM inside the Chebyshev recurrences; moment
  accumulation, solves, inner products and norms in FP64);
* ``moment_doubling``: compute moments with the product identity
  mu_2n = 2<T_n,T_n> - mu_0, mu_2n+1 = 2<T_n+1,T_n> - mu_1 (orthogonal basis
  only; halves the operator applications per moment set).

A reference RunConfig instance is accepted everywhere; the two extra fields
then take their defaults.
"""
from __future__ import annotations

from dataclasses import dataclass, fields

import numpy as np

from .errors import KuboMSDError


def grid(values, name, starts_zero=False):
    a = np.array(values, dtype=np.float64, copy=True)
    if a.ndim != 1 or not len(a) or not np.all(np.isfinite(a)) or np.any(np.diff(a) <= 0):
        raise KuboMSDError(f"{name} must be a finite, strictly increasing nonempty array")
    if starts_zero and a[0] != 0:
        raise KuboMSDError("time must start at zero")
    a.setflags(write=False)
    return a


def resolve_output_grid(emin, emax, n_energy):
    if not np.isfinite([emin, emax]).all() or emin >= emax or int(n_energy) != n_energy or n_energy < 2:
        raise KuboMSDError("require finite emin < emax and n_energy >= 2")
    return grid(np.linspace(emin, emax, int(n_energy)), "energy")


def resolve_time_grid(tmax, dt):
    if not np.isfinite([tmax, dt]).all() or tmax < 0 or dt <= 0:
        raise KuboMSDError("invalid tmax/dt")
    t = np.arange(int(np.floor(tmax / dt)) + 1, dtype=float) * dt
    if t[-1] < tmax and not np.isclose(t[-1], tmax, rtol=0, atol=8 * np.spacing(max(tmax, dt))):
        t = np.append(t, tmax)
    else:
        t[-1] = tmax
    return grid(t, "time", True)


@dataclass(frozen=True)
class RunConfig:
    energy_eV: object
    time_fs: object
    solver: str = "stochastic-kpm"
    backend: str = "gpu"
    cpu_kernel: str = "cpp"
    omp_threads: int = 1
    transport_distribution: str = "serial"
    kernel: str = "jackson"
    sigma_eV: float = .05
    n_moments: int = 256
    spectral_bounds: object = None
    axes: tuple = ("x", "y", "z")
    axes_vectors: object = None
    initial_state_selection: str = "all"
    stochastic_method: str = "auto"
    nsamples: int = 64
    seed: int = 20261019
    sample_batch: int = 8
    statistics_block: int = 8
    time_block: int = 16
    metric_rtol: float = 1e-10
    metric_atol: float = 0.
    metric_maxiter: int = 1000
    metric_solver: str = "pcg"
    metric_residual_policy: str = "fixed"
    metric_check_interval: int = 32
    metric_gap_ratio: float = .1
    preconditioner: str = "diagonal"
    sampling_tol: float = 1e-10
    sampling_max_order: int = 4096
    propagation_tol: float = 1e-12
    propagation_max_order: int = 4096
    segment_fs: float = 1.
    integration_dt_fs: float = .01
    include_vac: bool = True
    rho_abs: float = 0.
    rho_rel: float = 1e-12
    memory_limit_gb: float = 4.
    output_npz: bool = False
    bounds_method: str = "arpack"
    precision: str = "fp64"
    moment_doubling: bool = False

    def __post_init__(self):
        object.__setattr__(self, "energy_eV", grid(self.energy_eV, "energy"))
        object.__setattr__(self, "time_fs", grid(self.time_fs, "time", True))
        if self.solver != "stochastic-kpm":
            raise KuboMSDError("the B200 backend implements solver stochastic-kpm")
        if self.kernel != "jackson" or self.initial_state_selection != "all":
            raise KuboMSDError("stochastic-kpm requires Jackson, cpu/gpu, full-space sampling")
        if self.stochastic_method not in ("auto", "stepwise", "spectral"):
            raise KuboMSDError("unsupported stochastic method")
        for name in ("n_moments", "nsamples", "sample_batch", "statistics_block", "time_block", "metric_maxiter",
                     "sampling_max_order", "propagation_max_order"):
            v = getattr(self, name)
            if isinstance(v, bool) or not isinstance(v, (int, np.integer)) or v < 1:
                raise KuboMSDError(f"{name} must be a positive integer")
        if not isinstance(self.seed, (int, np.integer)) or self.seed < 0:
            raise KuboMSDError("seed must be a nonnegative integer")
        for name in ("sigma_eV", "metric_rtol", "sampling_tol", "propagation_tol", "segment_fs", "integration_dt_fs",
                     "memory_limit_gb"):
            if not np.isfinite(getattr(self, name)) or getattr(self, name) <= 0:
                raise KuboMSDError(f"{name} must be positive and finite")
        for name in ("metric_atol", "rho_abs", "rho_rel"):
            if not np.isfinite(getattr(self, name)) or getattr(self, name) < 0:
                raise KuboMSDError(f"{name} must be nonnegative and finite")
        if self.preconditioner not in ("diagonal", "block-jacobi"):
            raise KuboMSDError("the B200 backend supports the diagonal and block-jacobi preconditioners")
        if self.metric_solver != "pcg":
            raise KuboMSDError("the B200 backend implements metric_solver pcg")
        if self.metric_residual_policy not in ("fixed", "adaptive"):
            raise KuboMSDError("metric_residual_policy must be fixed or adaptive")
        if self.metric_check_interval < 1:
            raise KuboMSDError("metric_check_interval must be a positive integer")
        if not 0 < self.metric_gap_ratio < 1:
            raise KuboMSDError("metric_gap_ratio must be strictly between zero and one")
        if self.precision not in ("fp64", "mixed"):
            raise KuboMSDError("precision must be fp64 or mixed")
        if self.bounds_method not in ("arpack", "device-lanczos"):
            raise KuboMSDError("bounds_method must be arpack or device-lanczos")
        if self.spectral_bounds is not None:
            b = tuple(float(v) for v in self.spectral_bounds)
            if len(b) != 2 or not np.isfinite(b).all() or b[0] >= b[1]:
                raise KuboMSDError("invalid full spectral bounds")
            object.__setattr__(self, "spectral_bounds", b)
        axes = tuple(self.axes)
        if not axes or len(set(axes)) != len(axes):
            raise KuboMSDError("axes must be nonempty and unique")
        if self.axes_vectors is None:
            if any(a not in "xyz" or len(a) != 1 for a in axes):
                raise KuboMSDError("custom axes require axes_vectors")
            v = np.array([np.eye(3)["xyz".index(a)] for a in axes])
        else:
            v = np.array(self.axes_vectors, dtype=float, copy=True)
        if v.shape != (len(axes), 3) or not np.isfinite(v).all() or not np.allclose(v @ v.T, np.eye(len(axes)),
                                                                                    atol=1e-12, rtol=0):
            raise KuboMSDError("direction vectors must be orthonormal")
        v.setflags(write=False)
        object.__setattr__(self, "axes_vectors", v)
        object.__setattr__(self, "axes", axes)

    def as_dict(self):
        return {f.name: (getattr(self, f.name).tolist() if isinstance(getattr(self, f.name), np.ndarray)
                         else getattr(self, f.name)) for f in fields(self)}


def option(cfg, name, default):
    """Read a B200-only field from either config flavour."""
    return getattr(cfg, name, default)
