"""Shared test helpers: golden fixture access and tolerance checks."""
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"


def golden(name):
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as f:
        return {k: f[k] for k in f.files}


def csr_from(d, prefix):
    import scipy.sparse as sp
    return sp.csr_matrix((d[f"{prefix}_data"], d[f"{prefix}_indices"], d[f"{prefix}_indptr"]),
                         shape=tuple(d[f"{prefix}_shape"]))


def assert_rel(actual, expected, tol, what=""):
    """max |actual - expected| <= tol * max |expected| (norm-wise relative error)."""
    a = np.asarray(actual)
    e = np.asarray(expected)
    assert a.shape == e.shape, (what, a.shape, e.shape)
    scale = float(np.max(np.abs(e))) if e.size else 0.
    err = float(np.max(np.abs(a - e))) if e.size else 0.
    assert err <= tol * max(scale, 1e-300), f"{what}: max abs err {err:.3e} vs scale {scale:.3e} (tol {tol:g})"
    return err / max(scale, 1e-300)


def fixture_model(d, kind):
    """(H, S, velocity, position, composite) of an engine fixture."""
    vel, pos, comp = {}, {}, {}
    if kind == "velocity":
        vel = {"x": d["V"]}
    elif kind == "position":
        pos = {"x": d["X"]}
    else:
        comp = {"x": (d["bond"], d["xbar"], d["delta"])}
    return d["H"], d["S"], vel, pos, comp


def fixture_blocks(d):
    starts = [int(x) for x in d["blocks_start"]]
    return [(a, b, d["blocks_L"][i][:b - a, :b - a]) for i, (a, b) in enumerate(zip(starts[:-1], starts[1:]))]
