"""Ragged batches of independent Hamiltonians (the batching form).

`B200Batch` wraps `kmsd_batch_*` (include/kmsd.h): many Hamiltonians of
uneven size, such as disorder realisations, concatenated block-diagonally on
the device (with their overlap matrices for a nonorthogonal basis).  One kernel per Chebyshev step covers all of
them, with per-instance spectral windows and per-instance moment reductions.
The whole step sequence is captured into a CUDA graph and replayed.  `tune()`
picks the row-tile size by timing.  The moments of every instance equal those
of a separate `B200Operators.moments` call on it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .native import DeviceCSR, _check, _ptr, _stream, _torch


class B200Batch:
    """Moments of many independent instances in one call.

    Orthogonal instances (`overlaps=None`): mixed or FP64, one step kernel per
    Chebyshev step over all instances, replayed from a CUDA graph.
    Nonorthogonal instances (`overlaps` = one S per instance, `blocks` = the
    block-Jacobi factors (a, b, L) of each instance in its own row numbering,
    or None for the diagonal preconditioner): direct moments
    mu_k = Re<S B, T_k> per instance with an FP64 recurrence, S^-1 applied by
    one segmented PCG per step over all instances (one CG per instance and
    column, as the reference solves each instance); precision="mixed" stores
    the CG work vectors in complex64.
    """

    def __init__(self, hamiltonians, precision="mixed", tile_rows=0, overlaps=None, blocks=None, rtol=1e-10,
                 atol=0., maxiter=1000, residual_policy="fixed", check_interval=32, gap_ratio=.1):
        self.lib = _abi.require_library()
        torch = _torch()
        # nonorthogonal instances: FP64 recurrence; precision="mixed" keeps
        # the CG work vectors of the segmented solve in complex64
        self.metric_storage = precision if overlaps is not None else None
        if overlaps is not None:
            precision = "fp64"
        self.parts = [DeviceCSR(H, self.lib) for H in hamiltonians]
        self.ninst = len(self.parts)
        handles = (C.c_void_p * self.ninst)(*[p.handle.value for p in self.parts])
        h = C.c_void_p()
        rc = self.lib.kmsd_batch_create(self.ninst, handles, _abi.KMSD_MIXED if precision == "mixed" else
                                        _abi.KMSD_FP64, int(tile_rows), C.byref(h))
        _check(self.lib, rc)
        self.handle = h
        self.precision = precision
        off = np.zeros(self.ninst + 1, np.int64)
        _check(self.lib, self.lib.kmsd_batch_rows(h, off.ctypes.data_as(C.POINTER(C.c_int64))))
        self.offsets = off
        self.n = int(off[-1])
        self.metric = None
        if overlaps is not None:
            self._attach_metric(hamiltonians, overlaps, blocks, rtol, atol, maxiter, residual_policy, check_interval,
                                gap_ratio)
        del torch

    def _attach_metric(self, hamiltonians, overlaps, blocks, rtol, atol, maxiter, policy, interval, gap):
        import scipy.sparse as sp
        from types import SimpleNamespace
        from .native import B200Metric
        if len(overlaps) != self.ninst:
            raise ValueError("one overlap matrix per instance is required")
        Hg = sp.block_diag([sp.csr_matrix(H) for H in hamiltonians], format="csr")
        Sg = sp.block_diag([sp.csr_matrix(S) for S in overlaps], format="csr")
        gblocks = []
        if blocks is not None:
            for off, bl in zip(self.offsets[:-1], blocks):
                gblocks += [(int(off) + a, int(off) + b, L) for a, b, L in bl]
        cfg = SimpleNamespace(metric_solver="pcg", metric_residual_policy=policy, metric_check_interval=interval,
                              metric_gap_ratio=gap)
        self.hglobal = DeviceCSR(Hg, self.lib)
        self.metric = B200Metric(Sg, Sg.diagonal().real.copy(), gblocks, cfg)
        self.metric.set_storage(self.metric_storage)
        _check(self.lib, self.lib.kmsd_batch_attach_metric(self.handle, self.hglobal.handle, self.metric.handle,
                                                           float(rtol), float(atol), int(maxiter)))

    def concat(self, blocks):
        """Concatenate per-instance (N_i, b) blocks into one device block."""
        torch = _torch()
        parts = [b if isinstance(b, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(b, np.complex128))
                 for b in blocks]
        return torch.cat([p.to("cuda", torch.complex128) for p in parts], dim=0).contiguous()

    col_block = 0  # vector-block width of one batch call (0: all columns), set by tune()

    def moments(self, B, length, centers, halves, doubling=True, use_graph=True):
        """(ninst, length, b) float64 device tensor of Jackson-KPM moments; the
        columns run in blocks of `col_block` vectors when tune() chose that."""
        torch = _torch()
        if isinstance(B, (list, tuple)):
            B = self.concat(B)
        if B.shape[0] != self.n:
            raise ValueError("batch block rows must equal the sum of instance sizes")
        w = self.col_block
        if w and w < B.shape[1]:
            parts = [self._moments_block(B[:, j0:j0 + w].contiguous(), length, centers, halves, doubling, use_graph)
                     for j0 in range(0, B.shape[1], w)]
            return torch.cat(parts, dim=2)
        return self._moments_block(B, length, centers, halves, doubling, use_graph)

    def _moments_block(self, B, length, centers, halves, doubling, use_graph):
        torch = _torch()
        b = B.shape[1]
        c = np.ascontiguousarray(np.broadcast_to(np.asarray(centers, float), (self.ninst,)))
        h = np.ascontiguousarray(np.broadcast_to(np.asarray(halves, float), (self.ninst,)))
        mu = getattr(self, "_mu", None)
        if mu is None or mu.shape != (self.ninst, length, b):
            mu = self._mu = torch.empty((self.ninst, length, b), dtype=torch.float64, device="cuda")
        if self.metric is not None:
            doubling = False  # the product identity needs S = I
        flags = _abi.KMSD_MOMENTS_DOUBLING if doubling else _abi.KMSD_MOMENTS_DIRECT
        rc = self.lib.kmsd_batch_moments(self.handle, _ptr(B), C.cast(C.c_void_p(mu.data_ptr()),
                                                                      C.POINTER(C.c_double)),
                                         b, int(length), c.ctypes.data_as(C.POINTER(C.c_double)),
                                         h.ctypes.data_as(C.POINTER(C.c_double)), flags, int(use_graph),
                                         _stream(torch))
        _check(self.lib, rc)
        return mu.clone()

    def tune(self, B, length, centers, halves, doubling=True):
        """Autotunes the row-tile size and the vector-block width: for each
        width (all columns, half, a quarter; even widths in the mixed form)
        the library sweeps the tile sizes, then whole calls with that width
        and its best tile are timed.  Keeps the fastest pair; returns the tile
        rows (the width is in `col_block`)."""
        torch = _torch()
        if isinstance(B, (list, tuple)):
            B = self.concat(B)
        b = B.shape[1]
        widths = [w for w in (b, b // 2, b // 4) if w >= 1 and b % w == 0 and
                  (self.precision != "mixed" or w % 2 == 0)]
        best = None
        for w in dict.fromkeys(widths):
            rows = self._tune_rows(B[:, :w].contiguous(), length, centers, halves, doubling)
            self.col_block = w
            self.moments(B, length, centers, halves, doubling)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.moments(B, length, centers, halves, doubling)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if best is None or ms < best[0]:
                best = (ms, w, rows)
        _, self.col_block, rows = best
        _check(self.lib, self.lib.kmsd_batch_set_tile_rows(self.handle, int(rows)))
        self.tuned = {"tile_rows": rows, "col_block": self.col_block, "ms": best[0]}
        return rows

    def _tune_rows(self, B, length, centers, halves, doubling):
        torch = _torch()
        b = B.shape[1]
        c = np.ascontiguousarray(np.broadcast_to(np.asarray(centers, float), (self.ninst,)))
        h = np.ascontiguousarray(np.broadcast_to(np.asarray(halves, float), (self.ninst,)))
        mu = torch.empty((self.ninst, length, b), dtype=torch.float64, device="cuda")
        chosen = C.c_int64()
        if self.metric is not None:
            doubling = False
        flags = _abi.KMSD_MOMENTS_DOUBLING if doubling else _abi.KMSD_MOMENTS_DIRECT
        rc = self.lib.kmsd_batch_tune(self.handle, _ptr(B), C.cast(C.c_void_p(mu.data_ptr()), C.POINTER(C.c_double)),
                                      b, int(length), c.ctypes.data_as(C.POINTER(C.c_double)),
                                      h.ctypes.data_as(C.POINTER(C.c_double)), flags, C.byref(chosen),
                                      _stream(torch))
        _check(self.lib, rc)
        return int(chosen.value)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.kmsd_batch_destroy(h)
            self.handle = None
