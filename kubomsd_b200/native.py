"""Reference-facing adapter of the B200 engine.

`B200Metric` and `B200Operators` have the methods, arguments, return values
and error behaviour of KuboMSD's `NativeMetric` and `NativeOperators`
(src/kubo_msd/backends/native.py:49-133), so the reference's solvers can call
them where they call `ops.metric.native` / `ops.native`.  The work runs in
libkmsd_b200.so on the current CUDA device.  Arrays may be host NumPy arrays
(copied to the device and results copied back, as the reference returns NumPy
arrays) or CUDA torch tensors (results stay on the device).  There is no CPU
fallback: without the library or a CUDA device the constructors raise
BackendUnavailable.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any

import numpy as np
import scipy.sparse as sp

from . import _abi
from .errors import BackendUnavailable, NumericalError

try:  # the reference's report type, when KuboMSD is importable
    from kubo_msd.contracts import MetricSolveReport  # type: ignore
except Exception:  # noqa: BLE001
    @dataclass
    class MetricSolveReport:
        converged: Any
        iterations: Any
        true_residual: Any
        relative_residual: Any
        breakdown: Any

HBAR_EV_FS = 0.6582119569509067
MAX_COLS = 256          # FP64 columns per kernel launch (8 units x 32 lanes)
MAX_COLS_MIXED = 512    # complex64 columns per launch


class MetricFailure(RuntimeError):
    """A failed metric solve with its per-column diagnostics (cf. native.cpp:139-143)."""

    def __init__(self, message, diagnostics=None):
        super().__init__(message)
        self.diagnostics = diagnostics


def native_requested(config):
    """The GPU stochastic path is the B200 engine (cf. backends/native.py:11-13)."""
    return getattr(config, "backend", "gpu") == "gpu" and config.solver == "stochastic-kpm"


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise BackendUnavailable("B200 stochastic backend requires a CUDA device")
    return torch


def _call(function, *args, **kw):
    """Exception translation of backends/native.py:32-39."""
    try:
        return function(*args, **kw)
    except (ValueError, RuntimeError) as exc:
        failure = NumericalError(str(exc))
        if hasattr(exc, "diagnostics"):
            failure.diagnostics = exc.diagnostics
        raise failure from exc


def _check(lib, rc, diagnostics=None):
    if rc == _abi.KMSD_OK:
        return
    msg = _abi.last_error(lib)
    if rc == _abi.KMSD_EINVAL:
        raise ValueError(msg)
    if rc == _abi.KMSD_EMETRIC:
        raise MetricFailure(msg, diagnostics() if callable(diagnostics) else diagnostics)
    raise RuntimeError(msg)


def _stream(torch):
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def as_device(B, n=None, validate=True):
    """(N, b) complex128 contiguous CUDA tensor and whether the input was host
    memory.  Validation follows Dense(const Arr&) (cpp/native.cpp:31-40)."""
    torch = _torch()
    if isinstance(B, torch.Tensor):
        if B.ndim != 2 or B.shape[0] < 1 or B.shape[1] < 1:
            raise ValueError("expected nonempty finite (N,batch) array")
        t = B.to(device="cuda", dtype=torch.complex128).contiguous()
        if validate and not bool(torch.isfinite(torch.view_as_real(t)).all()):
            raise ValueError("expected finite (N,batch) array")
        host = False
    else:
        a = np.asarray(B)
        if a.ndim != 2 or a.shape[0] < 1 or a.shape[1] < 1:
            raise ValueError("expected nonempty finite (N,batch) array")
        a = np.ascontiguousarray(a, dtype=np.complex128)
        t = torch.from_numpy(a).to("cuda")
        # The finiteness check of the copied block runs on the device.
        if validate and not bool(torch.isfinite(torch.view_as_real(t)).all()):
            raise ValueError("expected finite (N,batch) array")
        host = True
    if n is not None and t.shape[0] != n:
        raise ValueError("CSR input dimension mismatch")
    return t, host


def _out(t, host):
    return t.cpu().numpy() if host else t


def canonical(matrix):
    """complex128 CSR, duplicates summed, sorted (backends/native.py:42-46)."""
    host = sp.csr_matrix(matrix, dtype=np.complex128, copy=True)
    host.sum_duplicates()
    host.sort_indices()
    return host


def _full_diagonal(X):
    """A position operator given by site coordinates (only diagonal entries,
    real) is stored with every diagonal entry explicit, zeros included, so
    the engine recognises it and applies i [H, X] / hbar from H's rows inside
    the Chebyshev step; any other matrix is returned unchanged."""
    A = sp.csr_matrix(X)
    if A.shape[0] != A.shape[1]:
        return X
    coo = A.tocoo()
    if np.any(coo.row != coo.col) or np.any(np.asarray(coo.data).imag != 0 if np.iscomplexobj(coo.data) else False):
        return X
    x = np.asarray(A.diagonal()).real.astype(np.float64)
    n = A.shape[0]
    return sp.csr_matrix((x, np.arange(n), np.arange(n + 1)), shape=(n, n))


class DeviceCSR:
    """A CSR matrix uploaded to the device; replaces `_native.CSR`."""

    def __init__(self, matrix, lib=None):
        self.lib = lib or _abi.require_library()
        _torch()
        A = canonical(matrix)
        self.n = A.shape[0]
        self.nnz = A.nnz
        indptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
        indices = np.ascontiguousarray(A.indices, dtype=np.int64)
        re = np.ascontiguousarray(A.data.real, dtype=np.float64)
        im = np.ascontiguousarray(A.data.imag, dtype=np.float64)
        handle = C.c_void_p()
        rc = self.lib.kmsd_csr_create(self.n, indptr.ctypes.data_as(C.POINTER(C.c_int64)),
                                      indices.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(re),
                                      _dptr(im) if np.any(im) else None, C.byref(handle))
        _check(self.lib, rc)
        self.handle = handle

    def matmul(self, B):
        torch = _torch()
        t, host = as_device(B, self.n)
        out = torch.empty_like(t)
        for j0 in range(0, t.shape[1], MAX_COLS):
            j1 = min(t.shape[1], j0 + MAX_COLS)
            x = t[:, j0:j1].contiguous()
            y = torch.empty_like(x)
            _check(self.lib, self.lib.kmsd_csr_matmul(self.handle, _ptr(x), _ptr(y), j1 - j0, _stream(torch)))
            out[:, j0:j1] = y
        return _out(out, host)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.kmsd_csr_destroy(h)
            self.handle = None


def vac_nodes(tables, coeffs, G, lib=None):
    """Per-node spectral tail on the device (kmsd_vac_nodes): `tables` the
    (b, length, kcols) device tensor of B200Operators.chain_correlate,
    `coeffs` a list of Bessel coefficient vectors (one per time node, each of
    at most kcols terms), G the (n_energy, n_moments) reconstruction matrix.
    Returns the (nodes, b, n_energy) float64 host array of VAC values."""
    torch = _torch()
    lib = lib or _abi.require_library()
    b, length, kcols = tables.shape
    m = len(coeffs)
    cf = np.zeros((m, kcols), np.complex128)
    orders = np.zeros(m, np.int32)
    for i, c in enumerate(coeffs):
        if len(c) > kcols:
            raise ValueError("internal spectral propagation order exceeded segment allocation")
        cf[i, :len(c)] = c
        orders[i] = len(c) - 1
    Gd = torch.from_numpy(np.ascontiguousarray(G, np.float64)).to(tables.device)
    L, ne = G.shape[1], G.shape[0]
    if length < L + int(orders.max()):
        raise ValueError("correlation tables shorter than the moments need")
    cfd = torch.from_numpy(cf).to(tables.device)
    od = torch.from_numpy(orders).to(tables.device)
    nbytes = m * b * (16 * length + 8 * L)
    work = torch.empty((nbytes + 15) // 16, dtype=torch.complex128, device=tables.device)
    vac = torch.empty((m, b, ne), dtype=torch.float64, device=tables.device)
    _check(lib, lib.kmsd_vac_nodes(_ptr(tables.contiguous()), b, length, kcols, L, _ptr(cfd), _ptr(od), m, _ptr(Gd),
                                   ne, _ptr(work), work.numel() * 16, _ptr(vac), _stream(torch)))
    return vac.cpu().numpy()


def _report_arrays(b):
    conv = np.zeros(b, np.uint8)
    brk = np.zeros(b, np.uint8)
    it = np.zeros(b, np.int64)
    res = np.zeros(b)
    rel = np.zeros(b)
    rep = _abi.SolveReport(conv.ctypes.data_as(C.POINTER(C.c_uint8)), brk.ctypes.data_as(C.POINTER(C.c_uint8)),
                           it.ctypes.data_as(C.POINTER(C.c_int64)), res.ctypes.data_as(C.POINTER(C.c_double)),
                           rel.ctypes.data_as(C.POINTER(C.c_double)))
    return rep, (conv, brk, it, res, rel)


def _diag_dict(arrays, m=None):
    conv, brk, it, res, rel = arrays
    sl = slice(None) if m is None else slice(0, m)
    return {"converged": [bool(x) for x in conv[sl]], "breakdown": [bool(x) for x in brk[sl]],
            "iterations": [int(x) for x in it[sl]], "true_residual": [float(x) for x in res[sl]],
            "relative_residual": [float(x) for x in rel[sl]]}


class B200Metric:
    """Drop-in for NativeMetric (src/kubo_msd/backends/native.py:49-92)."""

    def __init__(self, host, diagonal, blocks, config, preconditioner_data=None):
        self.lib = _abi.require_library()
        if getattr(config, "metric_solver", "pcg") != "pcg":
            raise BackendUnavailable("B200 metric implements the batched PCG solver (metric_solver=pcg)")
        if preconditioner_data is not None and getattr(preconditioner_data, "kind", None) in ("cluster-jacobi",
                                                                                              "ic0"):
            raise BackendUnavailable("B200 metric supports the diagonal and block-jacobi preconditioners")
        self.S = DeviceCSR(host, self.lib)
        self.n = self.S.n
        diag = np.ascontiguousarray(np.asarray(diagonal.get() if hasattr(diagonal, "get") else
                                               (diagonal.cpu().numpy() if hasattr(diagonal, "cpu") else diagonal),
                                               dtype=np.float64))
        blocks = list(blocks)
        nblocks = len(blocks)
        handle = C.c_void_p()
        if nblocks:
            start = np.zeros(nblocks + 1, np.int64)
            offs = np.zeros(nblocks, np.int64)
            facs, pos = [], 0
            for i, (a, b, L) in enumerate(blocks):
                L = np.asarray(L.get() if hasattr(L, "get") else L, dtype=np.complex128)
                start[i], start[i + 1] = a, b
                offs[i] = pos
                facs.append(L.ravel())
                pos += L.size
            fac = np.concatenate(facs)
            fre = np.ascontiguousarray(fac.real)
            fim = np.ascontiguousarray(fac.imag)
            rc = self.lib.kmsd_metric_create(self.S.handle, _dptr(diag), nblocks,
                                             start.ctypes.data_as(C.POINTER(C.c_int64)),
                                             offs.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(fre), _dptr(fim),
                                             C.byref(handle))
        else:
            rc = self.lib.kmsd_metric_create(self.S.handle, _dptr(diag), 0, None, None, None, None, C.byref(handle))
        _check(self.lib, rc)
        self.handle = handle
        self._create = (diag, blocks, config)
        self.policy = (getattr(config, "metric_residual_policy", "fixed"), getattr(config, "metric_check_interval", 32),
                       getattr(config, "metric_gap_ratio", .1))
        self._set_policy(*self.policy)
        self.identity = bool(self.lib.kmsd_metric_is_identity(handle))
        self.nseg = 1

    def replica(self):
        """A second metric over the same uploaded S with its own workspace, for
        concurrent use from another stream (handles are one-call-at-a-time)."""
        diag, blocks, config = self._create
        other = object.__new__(B200Metric)
        other.lib = self.lib
        other.S = self.S
        other.n = self.n
        B200Metric._init_handle(other, diag, blocks, config)
        if getattr(self, "storage", "fp64") == "mixed":
            other.set_storage("mixed")
        return other

    def _init_handle(self, diag, blocks, config):
        handle = C.c_void_p()
        nblocks = len(blocks)
        if nblocks:
            start = np.zeros(nblocks + 1, np.int64)
            offs = np.zeros(nblocks, np.int64)
            facs, pos = [], 0
            for i, (a, b, L) in enumerate(blocks):
                L = np.asarray(L, dtype=np.complex128)
                start[i], start[i + 1] = a, b
                offs[i] = pos
                facs.append(L.ravel())
                pos += L.size
            fac = np.concatenate(facs)
            fre, fim = np.ascontiguousarray(fac.real), np.ascontiguousarray(fac.imag)
            rc = self.lib.kmsd_metric_create(self.S.handle, _dptr(diag), nblocks,
                                             start.ctypes.data_as(C.POINTER(C.c_int64)),
                                             offs.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(fre), _dptr(fim),
                                             C.byref(handle))
        else:
            rc = self.lib.kmsd_metric_create(self.S.handle, _dptr(diag), 0, None, None, None, None, C.byref(handle))
        _check(self.lib, rc)
        self.handle = handle
        self._create = (diag, blocks, config)
        self.policy = (getattr(config, "metric_residual_policy", "fixed"), getattr(config, "metric_check_interval", 32),
                       getattr(config, "metric_gap_ratio", .1))
        self._set_policy(*self.policy)
        self.identity = bool(self.lib.kmsd_metric_is_identity(handle))
        self.nseg = 1

    def set_storage(self, precision):
        """Storage of the CG work vectors: "fp64" or "mixed" (complex64; all
        arithmetic, the solution, inner products and tests stay FP64)."""
        _check(self.lib, self.lib.kmsd_metric_set_storage(self.handle, _abi.KMSD_MIXED if precision == "mixed"
                                                          else _abi.KMSD_FP64))
        self.storage = precision

    def set_segments(self, offsets):
        """Declare S block-diagonal over the row ranges offsets[s]:offsets[s+1]
        (independent systems); later solves run one CG per (segment, column)
        and report nseg * b entries, segment-major (kmsd_metric_set_segments)."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        nseg = len(off) - 1
        _check(self.lib, self.lib.kmsd_metric_set_segments(self.handle, nseg,
                                                          off.ctypes.data_as(C.POINTER(C.c_int64))))
        self.nseg = max(nseg, 1)

    def _set_policy(self, policy, interval, gap):
        _check(self.lib, self.lib.kmsd_metric_set_residual_policy(
            self.handle, 1 if policy == "adaptive" else 0 if policy == "fixed" else -1, int(interval), float(gap)))

    def _solve(self, B, rtol, atol, maxiter):
        torch = _torch()
        t, host = as_device(B, self.n)
        out = torch.empty_like(t)
        b = t.shape[1]
        nseg = getattr(self, "nseg", 1)
        if nseg > 1 and b > MAX_COLS:
            raise ValueError(f"a segmented solve takes at most {MAX_COLS} columns per call")
        reps = []
        for j0 in range(0, b, MAX_COLS):
            j1 = min(b, j0 + MAX_COLS)
            x = t[:, j0:j1].contiguous()
            y = torch.empty_like(x)
            rep, arrays = _report_arrays(nseg * (j1 - j0))
            rc = self.lib.kmsd_metric_solve(self.handle, _ptr(x), _ptr(y), j1 - j0, float(rtol), float(atol),
                                            int(maxiter), C.byref(rep), _stream(torch))
            if rc == _abi.KMSD_EMETRIC:
                merged = [np.concatenate([r[i] for r in reps] + [arrays[i]]) for i in range(5)]
                _check(self.lib, rc, _diag_dict(merged))
            _check(self.lib, rc)
            reps.append(arrays)
            out[:, j0:j1] = y
        arrays = [np.concatenate([r[i] for r in reps]) for i in range(5)]
        return _out(out, host), arrays

    def solve(self, B, config):
        self._set_policy(config.metric_residual_policy, config.metric_check_interval, config.metric_gap_ratio)
        rtol = config.rtol if hasattr(config, "rtol") else config.metric_rtol
        try:
            values, arrays = _call(self._solve, B, max(rtol, 0), config.metric_atol, config.metric_maxiter)
        finally:
            self._set_policy(*self.policy)
        conv, brk, it, res, rel = arrays
        return values, MetricSolveReport(conv.astype(bool), it.astype(np.int64), res.astype(float),
                                         rel.astype(float), brk.astype(bool))

    def _sample(self, xi, coeff, center, half):
        torch = _torch()
        t, host = as_device(xi, self.n)
        coeff = np.ascontiguousarray(np.asarray(coeff, dtype=np.float64))
        if coeff.ndim != 1:
            raise ValueError("sampling coefficients must be 1D")
        out = torch.empty_like(t)
        for j0 in range(0, t.shape[1], MAX_COLS):
            j1 = min(t.shape[1], j0 + MAX_COLS)
            x = t[:, j0:j1].contiguous()
            y = torch.empty_like(x)
            _check(self.lib, self.lib.kmsd_metric_sample(self.handle, _ptr(x), _ptr(y), j1 - j0, _dptr(coeff),
                                                         len(coeff), float(center), float(half), _stream(torch)))
            out[:, j0:j1] = y
        return _out(out, host)

    def sample(self, xi, coeff, center, half):
        return _call(self._sample, xi, coeff, center, half)

    def stats(self):
        st = _abi.MetricStats()
        _check(self.lib, self.lib.kmsd_metric_stats_get(self.handle, C.byref(st)))
        return st

    def diagnostics(self):
        st = self.stats()
        values = {k: getattr(st, k) for k, _ in _abi.MetricStats._fields_}
        import json
        info = json.loads(self.lib.kmsd_build_info().decode())
        info.update(device=_torch().cuda.get_device_name())
        return {**values, "native": info}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.kmsd_metric_destroy(h)
            self.handle = None


class _Counters:
    def __init__(self, owner):
        self._owner = owner

    @property
    def h_calls(self):
        return self._owner._counters()[0]

    @property
    def v_calls(self):
        return self._owner._counters()[1]


class B200Operators:
    """Drop-in for NativeOperators (src/kubo_msd/backends/native.py:95-133).

    `ops` provides host_H, metric.native (a B200Metric) and the velocity /
    position / composite dictionaries of an OperatorBundle
    (src/kubo_msd/operators/velocity.py:10-47)."""

    def __init__(self, ops, config, precision=None):
        metric = ops.metric.native
        self.lib = metric.lib
        self.metric = metric
        self.H = DeviceCSR(ops.host_H, self.lib)
        self.S = metric.S
        self.n = self.H.n
        self.precision = precision or getattr(config, "precision", "fp64")
        # The mixed form on a nonorthogonal basis: the metric solve keeps its
        # CG work vectors in complex64 (FP64 arithmetic, solution, inner
        # products and tests) while the Chebyshev recurrence stays FP64.
        self.engine_precision = self.precision if metric.identity else "fp64"
        if self.precision == "mixed" and not metric.identity:
            metric.set_storage("mixed")
        self.doubling = bool(getattr(config, "moment_doubling", False))
        kinds = (C.c_int * 3)()
        mats = (C.c_void_p * 9)()
        self._keep = []
        for ai, axis in enumerate("xyz"):
            velocity = getattr(ops, "velocity", {}) or {}
            position = getattr(ops, "position", {}) or {}
            composite = getattr(ops, "composite", {}) or {}
            if axis in velocity:
                kind, ms = 0, [velocity[axis]]
            elif axis in position:
                kind, ms = 1, [position[axis]]
            elif axis in composite:
                kind, ms = 2, list(composite[axis])
            else:
                kind, ms = -1, []
            kinds[ai] = kind
            for j, m in enumerate(ms):
                m = m.get() if hasattr(m, "get") and not sp.issparse(m) else m
                if kind == 1:
                    m = _full_diagonal(m)
                d = DeviceCSR(m, self.lib)
                self._keep.append(d)
                mats[3 * ai + j] = d.handle
        self._kinds, self._mats, self._config = kinds, mats, config
        # work done, in applications of the scaled operator to one vector
        # (orbital.moment.vec / N): moment, propagation and chain steps
        self.vector_applications = 0
        self._create_engine()

    def _create_engine(self):
        handle = C.c_void_p()
        cfg = self._config
        rc = self.lib.kmsd_engine_create(self.H.handle, self.metric.handle, self._kinds, self._mats,
                                         float(cfg.metric_rtol), float(cfg.metric_atol), int(cfg.metric_maxiter),
                                         HBAR_EV_FS, _abi.KMSD_MIXED if self.engine_precision == "mixed" else _abi.KMSD_FP64,
                                         C.byref(handle))
        _check(self.lib, rc)
        self.handle = handle
        self.core = _Counters(self)

    def replica(self):
        """Another engine over the same uploaded H, S and velocity matrices with
        its own metric and workspace: a handle serves one call at a time, so
        concurrent streams each use their own replica."""
        other = object.__new__(B200Operators)
        other.__dict__.update({k: v for k, v in self.__dict__.items() if k not in ("handle", "core", "metric")})
        other.metric = self.metric.replica()
        other._create_engine()
        return other

    # -- helpers
    def _counters(self):
        h, v = C.c_int64(), C.c_int64()
        _check(self.lib, self.lib.kmsd_engine_counters(self.handle, C.byref(h), C.byref(v)))
        return h.value, v.value

    def _failure(self):
        cap = 512
        rep, arrays = _report_arrays(cap)
        m = C.c_int64()
        self.lib.kmsd_engine_failure_report(self.handle, C.byref(rep), cap, C.byref(m))
        return _diag_dict(arrays, m.value)

    def _cols(self):
        return MAX_COLS_MIXED if self.engine_precision == "mixed" else MAX_COLS

    # -- operations (same names and signatures as NativeOperators)
    def _h_action(self, B):
        torch = _torch()
        t, host = as_device(B, self.n)
        out = torch.empty_like(t)
        for j0 in range(0, t.shape[1], MAX_COLS):
            j1 = min(t.shape[1], j0 + MAX_COLS)
            x = t[:, j0:j1].contiguous()
            y = torch.empty_like(x)
            _check(self.lib, self.lib.kmsd_engine_h_action(self.handle, _ptr(x), _ptr(y), j1 - j0, _stream(torch)),
                   self._failure)
            out[:, j0:j1] = y
        return _out(out, host)

    def h_action(self, B):
        return _call(self._h_action, B)

    def _v_cov(self, direction, B, config=None):
        torch = _torch()
        d = np.ascontiguousarray(np.asarray(direction, dtype=np.float64))
        if d.shape != (3,):
            raise ValueError("direction must have three components")
        t, host = as_device(B, self.n)
        out = torch.empty_like(t)
        rt, at, mi = (config.metric_rtol, config.metric_atol, config.metric_maxiter) if config is not None else (
            0., 0., 0)
        for j0 in range(0, t.shape[1], MAX_COLS):
            j1 = min(t.shape[1], j0 + MAX_COLS)
            x = t[:, j0:j1].contiguous()
            y = torch.empty_like(x)
            _check(self.lib, self.lib.kmsd_engine_v_cov(self.handle, _dptr(d), _ptr(x), _ptr(y), j1 - j0, float(rt),
                                                        float(at), int(mi), _stream(torch)), self._failure)
            out[:, j0:j1] = y
        return _out(out, host)

    def v_cov(self, direction, B, config=None):
        return _call(self._v_cov, direction, B, config)

    def _series(self, B, coeff, center, half, directions=()):
        torch = _torch()
        t, host = as_device(B, self.n)
        c = np.asarray(coeff, dtype=np.complex128)
        if c.ndim != 1:
            raise ValueError("Chebyshev coefficients must be 1D")
        cc = np.ascontiguousarray(np.stack([c.real, c.imag], 1).ravel())
        dirs = np.ascontiguousarray(np.asarray([list(v) for v in directions], dtype=np.float64).reshape(-1, 3))
        nd = len(dirs)
        b = t.shape[1]
        if nd and b % (nd + 1):
            raise ValueError("invalid augmented block columns")
        nb = b // (nd + 1)
        step = max(1, self._cols() // (nd + 1))
        if self.engine_precision == "mixed" and nd:
            step -= step % 2
        out = torch.empty_like(t)
        for s0 in range(0, nb, step):
            s1 = min(nb, s0 + step)
            cols = np.concatenate([np.arange(a * nb + s0, a * nb + s1) for a in range(nd + 1)])
            idx = torch.as_tensor(cols, device=t.device)
            x = t.index_select(1, idx).contiguous() if (s0, s1) != (0, nb) else t
            y = torch.empty_like(x)
            _check(self.lib, self.lib.kmsd_engine_series(self.handle, _ptr(x), _ptr(y), x.shape[1], _dptr(cc),
                                                         len(c), float(center), float(half),
                                                         _dptr(dirs) if nd else None, nd, _stream(torch)),
                   self._failure)
            self.vector_applications += (len(c) - 1) * x.shape[1]
            if (s0, s1) != (0, nb):
                out[:, idx] = y
            else:
                out = y
        return _out(out, host)

    def series(self, B, coeff, center, half, directions=()):
        return _call(self._series, B, coeff, center, half, directions)

    def _chain(self, B, length, center, half):
        torch = _torch()
        t, host = as_device(B, self.n)
        if length < 1:
            raise ValueError("Chebyshev chain must be nonempty")
        b = t.shape[1]
        out = torch.empty((length, self.n, b), dtype=torch.complex128, device=t.device)
        for j0 in range(0, b, self._cols()):
            j1 = min(b, j0 + self._cols())
            x = t[:, j0:j1].contiguous()
            y = torch.empty((length, self.n, j1 - j0), dtype=torch.complex128, device=t.device)
            _check(self.lib, self.lib.kmsd_engine_chain(self.handle, _ptr(x), _ptr(y), j1 - j0, int(length),
                                                        float(center), float(half), _stream(torch)), self._failure)
            self.vector_applications += (length - 1) * (j1 - j0)
            out[:, :, j0:j1] = y
        return _out(out, host)

    def chain(self, B, length, center, half):
        return _call(self._chain, B, length, center, half)

    def _chain_correlate(self, B, cov, length, center, half):
        torch = _torch()
        t, _ = as_device(B, self.n)
        b = t.shape[1]
        cov = cov if isinstance(cov, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(cov, np.complex128))
        cov = cov.to(t.device, torch.complex128)
        if length < 1:
            raise ValueError("Chebyshev chain must be nonempty")
        if cov.ndim != 3 or cov.shape[0] != self.n or cov.shape[2] != b:
            raise ValueError("cov must be (N, kcols, batch)")
        kcols = cov.shape[1]
        # columns per call: at most 8, fewer when the right chain is long
        group = 8
        while group > 1 and kcols > 4 * (256 // group):
            group //= 2
        if self.engine_precision == "mixed":
            group = max(2, group - group % 2)
        if kcols > 4 * (256 // group):
            raise ValueError("too many right-chain terms for one correlation call")
        tables = torch.empty((b, length, kcols), dtype=torch.complex128, device=t.device)
        for j0 in range(0, b, group):
            j1 = min(b, j0 + group)
            x = t[:, j0:j1].contiguous()
            cv = cov[:, :, j0:j1].contiguous()
            out = torch.empty((j1 - j0, length, kcols), dtype=torch.complex128, device=t.device)
            _check(self.lib, self.lib.kmsd_engine_chain_correlate(self.handle, _ptr(x), _ptr(cv), j1 - j0,
                                                                  int(length), int(kcols), float(center),
                                                                  float(half), _ptr(out), _stream(torch)),
                   self._failure)
            self.vector_applications += (length - 1) * (j1 - j0)
            tables[j0:j1] = out
        return tables

    def chain_correlate(self, B, cov, length, center, half):
        """tables[c, j, k] = <T_j(Ht) B[:, c], cov[:, k, c]> (device tensor of
        shape (batch, length, kcols)); the chain is never stored whole."""
        return _call(self._chain_correlate, B, cov, length, center, half)

    def _moments(self, B, length, center, half, doubling=None):
        torch = _torch()
        t, host = as_device(B, self.n)
        if length < 1:
            raise ValueError("moment count must be positive")
        # the configured default applies the product identity where it holds (S = I);
        # an explicit doubling=True on a nonorthogonal engine is an error
        doubling = (self.doubling and self.metric.identity) if doubling is None else doubling
        flags = _abi.KMSD_MOMENTS_DOUBLING if doubling else _abi.KMSD_MOMENTS_DIRECT
        b = t.shape[1]
        mu = torch.empty((length, b), dtype=torch.float64, device=t.device)
        for j0 in range(0, b, self._cols()):
            j1 = min(b, j0 + self._cols())
            x = t[:, j0:j1].contiguous()
            m = torch.empty((length, j1 - j0), dtype=torch.float64, device=t.device)
            _check(self.lib, self.lib.kmsd_engine_moments(self.handle, _ptr(x), C.cast(C.c_void_p(m.data_ptr()),
                                                                                    C.POINTER(C.c_double)),
                                                          j1 - j0, int(length), float(center), float(half), flags,
                                                          _stream(torch)), self._failure)
            if length > 1:
                self.vector_applications += ((length + 1) // 2 if doubling else length - 1) * (j1 - j0)
            mu[:, j0:j1] = m
        return _out(mu, host)

    def moments(self, B, length, center, half, doubling=None):
        return _call(self._moments, B, length, center, half, doubling)

    def lanczos(self, v0, steps):
        """(alpha, beta) of `steps` Lanczos iterations of (H, S) in the S inner
        product from v0, run on the device (kmsd_engine_lanczos)."""
        torch = _torch()
        v, _ = as_device(v0, self.n, validate=False)
        v = v[:, :1].contiguous()
        alpha = np.zeros(int(steps))
        beta = np.zeros(int(steps))
        _check(self.lib, self.lib.kmsd_engine_lanczos(self.handle, _ptr(v), int(steps), _dptr(alpha), _dptr(beta),
                                                      _stream(torch)), self._failure)
        return alpha, beta

    def inner(self, A, B):
        """<A, S B> per column (OperatorBundle.inner, velocity.py:117)."""
        torch = _torch()
        a, host = as_device(A, self.n, validate=False)
        b_, _ = as_device(B, self.n, validate=False)
        out = torch.empty((a.shape[1],), dtype=torch.complex128, device=a.device)
        for j0 in range(0, a.shape[1], MAX_COLS):
            j1 = min(a.shape[1], j0 + MAX_COLS)
            x = a[:, j0:j1].contiguous()
            y = b_[:, j0:j1].contiguous()
            o = torch.empty((j1 - j0,), dtype=torch.complex128, device=a.device)
            _check(self.lib, self.lib.kmsd_engine_inner(self.handle, _ptr(x), _ptr(y), _ptr(o), j1 - j0,
                                                        _stream(torch)))
            out[j0:j1] = o
        return _out(out, host)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.kmsd_engine_destroy(h)
            self.handle = None
