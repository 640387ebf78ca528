"""Builders shared by the GPU tests (imported only inside gpu-marked tests)."""
from types import SimpleNamespace

import numpy as np
import scipy.sparse as sp

from tests.helpers import fixture_blocks, fixture_model


def controls(rtol=1e-10, precision="fp64", policy="fixed", doubling=False):
    return SimpleNamespace(metric_rtol=rtol, metric_atol=0., metric_maxiter=1000, metric_residual_policy=policy,
                           metric_check_interval=32, metric_gap_ratio=.1, metric_solver="pcg", precision=precision,
                           moment_doubling=doubling)


def engine(H, S, velocity=None, position=None, composite=None, blocks=(), rtol=1e-10, precision="fp64",
           policy="fixed"):
    from kubomsd_b200.native import B200Metric, B200Operators
    cfg = controls(rtol, precision, policy)
    S = sp.csr_matrix(S, dtype=complex)
    metric = B200Metric(S, S.diagonal().real.copy(), list(blocks), cfg)
    ops = SimpleNamespace(host_H=H, metric=SimpleNamespace(native=metric), velocity=velocity or {},
                          position=position or {}, composite=composite or {})
    eng = B200Operators(ops, cfg)

    def v_cov(axis, B, config=None):
        return eng.v_cov(np.eye(3)["xyz".index(axis)], B, config)

    def v_action(axis, B):
        return metric.solve(v_cov(axis, B), cfg)[0]

    return metric, eng, SimpleNamespace(native=eng, inner=eng.inner, apply_v_cov=v_cov, apply_v_action=v_action)


def fixture_engine(d, kind, pre, precision="fp64"):
    H, S, vel, pos, comp = fixture_model(d, kind)
    blocks = fixture_blocks(d) if pre == "block-jacobi" else ()
    return engine(H, S, vel, pos, comp, blocks, rtol=float(d["rtol"]), precision=precision)
