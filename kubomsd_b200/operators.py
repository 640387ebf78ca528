"""Operator bundle on the B200 engine (the reference's OperatorBundle,
src/kubo_msd/operators/velocity.py:10-124, with the metric set-up of
src/kubo_msd/metric/setup.py:46-92 and MetricSolver, metric/solve.py:11-58).

`build_operators(model, config)` validates H, S and the velocity operators
(Hermitian, finite, square), prepares the preconditioner (diagonal, or
block-Jacobi Cholesky factors per atom slice), uploads everything once to the
device, creates the engine, and runs the reference's velocity Hermiticity
probe through the engine.  The bundle exposes the reference's methods
(apply_h_action, apply_v_cov, apply_v_action, inner, solve_s, h_calls,
v_calls) on device tensors or host arrays.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import scipy.linalg as la

from .config import option
from .errors import KuboMSDError, NumericalError
from .kpm import hermitian, spd_bounds
from .native import B200Metric, B200Operators, as_device


class DeviceMetric:
    """MetricSolver surface over B200Metric (metric/solve.py:11-174)."""

    def __init__(self, S, config, atom_slices=None):
        self.config = config
        self.host_S = S
        self.s_lower, self.s_upper, self.bounds_report = spd_bounds(S)
        self.condition_estimate = self.s_upper / self.s_lower
        self.diagonal = S.diagonal().real.copy()
        blocks = []
        if config.preconditioner == "block-jacobi":
            slices = atom_slices or [(j, j + 1) for j in range(S.shape[0])]
            if [i for a, b in slices for i in range(a, b)] != list(range(S.shape[0])):
                raise NumericalError("atom_slices must partition orbitals")
            for a, b in slices:
                blocks.append((a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)))
        self.blocks = blocks
        self.native = B200Metric(S, self.diagonal, blocks, config)

    def solve_s(self, B, config=None):
        cfg = self.config if config is None else SimpleNamespace(**{**_as_dict(self.config), **vars(config)})
        return self.native.solve(B, cfg)

    def diagnostics(self):
        d = self.native.diagnostics()
        d.update(condition_upper_or_estimate=self.condition_estimate, bounds=self.bounds_report,
                 kernel="b200", solver="pcg", resolved_preconditioner=self.config.preconditioner)
        return d


def _as_dict(cfg):
    if hasattr(cfg, "as_dict"):
        return cfg.as_dict()
    return dict(vars(cfg))


class DeviceOperators:
    def __init__(self, model, config):
        self.config = config
        self.n = model.H.shape[0]
        self.host_H = hermitian(model.H, "Hamiltonian")
        self.host_S = hermitian(model.S, "overlap")
        if self.host_H.shape != self.host_S.shape:
            raise KuboMSDError("H/S dimensions disagree")
        self.metric = DeviceMetric(self.host_S, config, getattr(model, "atom_slices", None) or None)
        self.velocity = {a: hermitian(v, "velocity " + a) for a, v in (model.velocity or {}).items()}
        self.position = {a: hermitian(v, "position " + a) for a, v in (model.position or {}).items()}
        self.composite = {a: tuple(parts) for a, parts in (model.composite or {}).items()}
        for axis, parts in self.composite.items():
            if len(parts) != 3:
                raise KuboMSDError("composite velocity requires bond/xbar/delta")
        self.directions = {a: v for a, v in zip(config.axes, config.axes_vectors)}
        for direction in config.axes_vectors:
            for axis, c in zip("xyz", direction):
                if c and axis not in self.velocity and axis not in self.position and axis not in self.composite:
                    raise KuboMSDError(f"missing physical velocity/position/dipole for {axis}")
        self.native = B200Operators(self, config, precision=option(config, "precision", "fp64"))
        self.velocity_hermiticity = {}
        rng = np.random.default_rng(551)
        probe = (np.eye(self.n, dtype=complex) if self.n <= 64 else
                 rng.normal(size=(self.n, 8)) + 1j * rng.normal(size=(self.n, 8)))
        for axis in config.axes:
            self.velocity_hermiticity[axis] = self._check_velocity(axis, probe)

    def _check_velocity(self, axis, probe):
        """Hermiticity probe with tightened retries (velocity.py:57-88)."""
        cfg = self.config
        controls, attempts = None, []
        rtol, atol = cfg.metric_rtol, cfg.metric_atol
        retries = 2
        error = np.nan
        for attempt in range(retries + 1):
            try:
                v = probe.conj().T @ np.asarray(self.apply_v_cov(axis, probe, controls))
            except NumericalError as exc:
                attempts.append(dict(metric_rtol=rtol, metric_atol=atol, status="S_SOLVE_FAILED", reason=str(exc)))
                exc.diagnostics = {**(getattr(exc, "diagnostics", None) or {}),
                                   "velocity_probe": dict(axis=axis, threshold=1e-10, attempts=attempts)}
                raise
            error = float(np.linalg.norm(v - v.conj().T) / max(np.linalg.norm(v), 1e-300))
            attempts.append(dict(metric_rtol=rtol, metric_atol=atol, relative_error=error))
            if np.isfinite(error) and error <= 1e-10:
                return dict(relative_error=error, threshold=1e-10, attempts=attempts,
                            mode="full" if self.n <= 64 else "8-vector bilinear probe")
            if not np.isfinite(error) or attempt == retries:
                break
            rtol = min(rtol * .1, 1e-12 if attempt == 0 else 1e-13)
            atol *= .1
            controls = SimpleNamespace(metric_rtol=rtol, metric_atol=atol, metric_maxiter=cfg.metric_maxiter)
        failure = KuboMSDError(f"constructed velocity {axis} is not Hermitian (relative error {error:g}; "
                               f"probe attempts {attempts})")
        failure.diagnostics = {"velocity_probe": dict(axis=axis, threshold=1e-10, attempts=attempts)}
        raise failure

    # reference surface ------------------------------------------------------
    def solve_s(self, B, config=None):
        return self.metric.solve_s(B, config)

    @property
    def h_calls(self):
        return self.native.core.h_calls

    @property
    def v_calls(self):
        return self.native.core.v_calls

    def apply_h_cov(self, B):
        return self.native.H.matmul(B)

    def apply_h_action(self, B):
        return self.native.h_action(B)

    def apply_v_cov(self, axis, B, config=None):
        direction = self.directions.get(axis, np.eye(3)["xyz".index(axis)] if axis in "xyz" else None)
        if direction is None:
            raise KuboMSDError("unknown direction")
        return self.native.v_cov(direction, B, config)

    def apply_v_action(self, axis, B):
        return self.solve_s(self.apply_v_cov(axis, B))[0]

    def inner(self, A, B):
        return self.native.inner(A, B)


def build_operators(model, config):
    return DeviceOperators(model, config)


def to_device(B):
    return as_device(B)[0]
