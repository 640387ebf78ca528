"""Test infrastructure: loader of the reference's compiled CPU engine.

`oracle/build_ref.sh` compiles KuboMSD's cpp/native.cpp (the pybind11 module
`kubo_msd._native`) into `oracle/_ref/`.  This module imports that binary
directly from there — the reference's own CSR / Metric / Engine classes —
for use as a parity checker and as the timed CPU baseline.  Product code never
imports this module.
"""
from __future__ import annotations

import importlib.machinery
import importlib.util
import subprocess
import sysconfig
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"


def library_path() -> Path:
    return REF_DIR / ("_native" + sysconfig.get_config_var("EXT_SUFFIX"))


def build() -> Path | None:
    """Compile the reference engine if its source is present (no-op otherwise)."""
    subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True, capture_output=True)
    path = library_path()
    return path if path.exists() else None


_module = None


def load():
    """Import the compiled reference module, or return None when absent."""
    global _module
    if _module is not None:
        return _module
    path = library_path()
    if not path.exists():
        return None
    loader = importlib.machinery.ExtensionFileLoader("_native", str(path))
    spec = importlib.util.spec_from_file_location("_native", str(path), loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    _module = mod
    return mod


def csr(mod, matrix, threads=1):
    """Canonical complex128 CSR exactly as the reference adapter builds it
    (src/kubo_msd/backends/native.py:42-46)."""
    host = sp.csr_matrix(matrix, dtype=np.complex128, copy=True)
    host.sum_duplicates()
    host.sort_indices()
    return mod.CSR(host.indptr.astype(np.int64), host.indices.astype(np.int64), host.data, host.shape[0], threads)


class RefEngine:
    """The reference Metric + Engine over host matrices (velocity kind 0/1/2)."""

    def __init__(self, H, S, velocity=None, position=None, composite=None, blocks=(), rtol=1e-10, atol=0.,
                 maxiter=1000, threads=1, hbar=0.6582119569509067, policy=("fixed", 32, .1)):
        mod = load()
        if mod is None:
            raise RuntimeError("reference engine not built (oracle/build_ref.sh)")
        self.mod = mod
        S = sp.csr_matrix(S, dtype=np.complex128)
        self.S = csr(mod, S, threads)
        diag = S.diagonal().real.copy()
        self.metric = mod.Metric(self.S, diag, list(blocks), threads)
        self.metric.set_residual_policy(*policy)
        self.H = csr(mod, H, threads)
        velocity, position, composite = velocity or {}, position or {}, composite or {}
        defs = []
        for axis in "xyz":
            if axis in velocity:
                defs.append((0, [csr(mod, velocity[axis], threads)]))
            elif axis in position:
                defs.append((1, [csr(mod, position[axis], threads)]))
            elif axis in composite:
                defs.append((2, [csr(mod, m, threads) for m in composite[axis]]))
            else:
                defs.append((-1, []))
        self.core = mod.Engine(self.H, self.metric, defs, rtol, atol, maxiter, hbar)
