"""Device-resident stochastic-KPM transport driver.

The orchestration of KuboMSD's stepwise stochastic path
(src/kubo_msd/solvers/stepwise.py:8-38, chebyshev.py:50-54,
stochastic.py:21-228) with the vector blocks kept on the GPU between engine
calls: the augmented state [psi | phi_a] never leaves the device; only the
moment arrays (n_moments x batch float64), S-norms and the float64 block sums
come back to the host, where the Jackson projection, block statistics and the
paired bootstrap run in FP64 exactly as in the reference.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field, replace
from typing import Any

import numpy as np

from . import kpm
from .errors import BackendUnavailable, NumericalError
from .parallel import ParallelContext, owned_blocks

REASON_LOW_DOS, REASON_UNCERTAIN_TRACE, REASON_INTEGRATION_UNVERIFIED, REASON_INSUFFICIENT_BLOCKS = 1, 2, 16, 32


@dataclass
class TransportBlock:
    """Same fields as the reference's TransportBlock (contracts.py:41-47)."""
    start: int
    time_fs: Any
    arrays: dict
    static: dict = field(default_factory=dict)
    metadata: dict = field(default_factory=dict)


def _torch():
    import torch
    return torch


def projected_quadratic(B, ops, cfg):
    """(G mu)^T with mu the device moments of B (chebyshev.py:50-54)."""
    G = kpm.reconstruction_matrix(cfg.energy_eV, cfg.spectral_bounds, cfg.n_moments)
    c, a = kpm.scaling(cfg)
    mu = ops.native.moments(B, cfg.n_moments, c, a)
    mu = mu.cpu().numpy() if hasattr(mu, "cpu") else np.asarray(mu)
    return (G @ mu).T


def drift_tolerance(cfg):
    """S-norm drift guard: the reference's 1e-7 (stepwise.py:16-17, 35-36) for
    FP64; complex64 vectors carry ~6e-8 rounding per step, so the mixed form
    is held to 1e-5 instead."""
    return 1e-5 if getattr(cfg, "precision", "fp64") == "mixed" else 1e-7


def _snorm(ops, B):
    v = ops.inner(B, B)
    v = v.cpu().numpy() if hasattr(v, "cpu") else np.asarray(v)
    return v.real


def propagate(states, dt_fs, ops, cfg):
    """Segmented Bessel propagation with the S-norm drift guard (stepwise.py:8-18)."""
    torch = _torch()
    B = states if isinstance(states, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(states, dtype=np.complex128)).cuda()
    initial = _snorm(ops, B)
    nseg = max(1, int(np.ceil(abs(dt_fs) / cfg.segment_fs)))
    dt = dt_fs / nseg
    coeff, diag = kpm.bessel_coefficients(dt, cfg)
    c, a = kpm.scaling(cfg)
    for _ in range(nseg):
        B = ops.native.series(B, coeff, c, a)
    final = _snorm(ops, B)
    drift = float(np.max(np.abs(final - initial) / np.maximum(initial, np.finfo(float).tiny)))
    if drift > drift_tolerance(cfg):
        raise NumericalError(f"S-norm propagation drift {drift:g}; bounds/solver/propagation need correction")
    out = B if isinstance(states, torch.Tensor) else B.cpu().numpy()
    return out, {**diag, "segments": nseg, "relative_S_norm_drift": drift}


def stepwise_samples(ops, cfg, samples):
    """Velocity-driven augmented commutator MSD (stepwise.py:20-38) with the
    state resident on the device.  Returns (dos, {'msd_A2/commutator': ...}, diag)."""
    torch = _torch()
    initial = samples if isinstance(samples, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(samples, dtype=np.complex128))
    initial = initial.to("cuda", torch.complex128).contiguous()
    nb = initial.shape[1]
    na, nt, ne = len(cfg.axes), len(cfg.time_fs), len(cfg.energy_eV)
    t0 = time.perf_counter()
    dos = projected_quadratic(initial, ops, cfg)
    total = torch.cat([initial] + [torch.zeros_like(initial) for _ in cfg.axes], dim=1).contiguous()
    output = np.zeros((nb, na, nt, ne))
    c, a = kpm.scaling(cfg)
    orders = []
    norm0 = _snorm(ops, initial)
    drift = 0.
    segments = 0
    directions = [list(v) for v in cfg.axes_vectors]
    for j, t in enumerate(cfg.time_fs):
        if j:
            span = t - cfg.time_fs[j - 1]
            count = max(1, int(np.ceil(span / cfg.segment_fs)))
            coeff, report = kpm.bessel_coefficients(span / count, cfg, weighted_tail=True)
            orders.append(report["order"])
            for _ in range(count):
                total = ops.native.series(total, coeff, c, a, directions)
                segments += 1
            norm = _snorm(ops, total[:, :nb].contiguous())
            drift = max(drift, float(np.max(np.abs(norm - norm0) / np.maximum(norm0, np.finfo(float).tiny))))
            if drift > drift_tolerance(cfg):
                raise NumericalError(f"stepwise base propagation S-norm drift {drift:g}")
        for ai in range(na):
            output[:, ai, j, :] = projected_quadratic(total[:, (ai + 1) * nb:(ai + 2) * nb].contiguous(), ops, cfg)
    return dos, {"msd_A2/commutator": output}, {
        "algorithm": "velocity-driven augmented Chebyshev commutator", "segments": segments,
        "max_propagation_order": max(orders, default=0), "max_relative_S_norm_drift": drift,
        "seconds": time.perf_counter() - t0, "device_resident": True}


def spectral_samples(ops, cfg, samples):
    """Segmented trace-first Chebyshev product VAC (spectral.py:15-53).

    Per segment the anchors are propagated on the device, the left chain
    T_j(Ht) c (j < L+K) and the right chains T_k(Ht) v_a (k <= K) are built by
    the engine, the velocity is applied to the right chains on the device, and
    the correlation tables tables[b, j, k] = sum_n conj(left[j,n,b]) cov[k,n,b]
    are one batched complex GEMM per axis on the device.  The per-node Bessel
    contraction, product rule T_l T_p = (T_l+p + T_|l-p|)/2, Jackson projection
    and the M/D recurrence run in FP64 on the host in the reference's order.
    """
    from .config import resolve_time_grid
    torch = _torch()
    x = samples if isinstance(samples, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(samples, dtype=np.complex128))
    x = x.to("cuda", torch.complex128).contiguous()
    n, nb = x.shape
    na, ne, nt, L = len(cfg.axes), len(cfg.energy_eV), len(cfg.time_fs), cfg.n_moments
    t0 = time.perf_counter()
    dos = projected_quadratic(x, ops, cfg)
    keys = ("msd_A2/vac_integral", "diffusion_A2_per_fs/vac_integral", "vac_A2_per_fs2/vac_integral")
    output = {k: np.zeros((nb, na, nt, ne)) for k in keys}
    times = np.unique(np.r_[resolve_time_grid(cfg.time_fs[-1], cfg.integration_dt_fs), cfg.time_fs])
    output_indices = {float(t): j for j, t in enumerate(cfg.time_fs)}
    G = kpm.reconstruction_matrix(cfg.energy_eV, cfg.spectral_bounds, L)
    c_anchor = x
    v_anchor = [ops.apply_v_action(a, x) for a in cfg.axes]
    anchor, next_anchor, tables = 0., -1., None
    maxorder = segments = 0
    maxnorm = 0.
    c, a = kpm.scaling(cfg)
    M = np.zeros((nb, na, ne))
    D = np.zeros_like(M)
    previous, prev_t = None, 0.
    for t in times:
        if tables is None or t > next_anchor + 1e-14:
            new_anchor = 0. if tables is None else float(prev_t)
            if new_anchor > anchor:
                both = torch.cat([c_anchor] + v_anchor, dim=1).contiguous()
                both, report = propagate(both, new_anchor - anchor, ops, cfg)
                maxnorm = max(maxnorm, report["relative_S_norm_drift"])
                c_anchor = both[:, :nb].contiguous()
                v_anchor = [both[:, (i + 1) * nb:(i + 2) * nb].contiguous() for i in range(na)]
            anchor = new_anchor
            next_anchor = min(max(anchor + cfg.segment_fs, float(t)), float(times[-1]))
            coeff, _ = kpm.bessel_coefficients(next_anchor - anchor, cfg)
            K = len(coeff) - 1
            maxorder = max(maxorder, K)
            estimate = 16 * nb * (n * (L + 2 * K + 1) + na * (L + K) * (K + 1)) + 24 * nb * na * nt * ne
            if estimate > cfg.memory_limit_gb * 1024 ** 3:
                raise NumericalError("spectral workspace exceeds memory budget; reduce sample_batch/segment_fs or "
                                     "increase explicit budget")
            left = ops.native.chain(c_anchor, L + K, c, a)           # (L+K, n, nb) on the device
            lconj = left.permute(2, 0, 1).conj()                     # (nb, L+K, n)
            tables = []
            for ai, axis in enumerate(cfg.axes):
                right = ops.native.chain(v_anchor[ai], K + 1, c, a)  # (K+1, n, nb)
                cov = ops.apply_v_cov(axis, right.permute(1, 0, 2).reshape(n, -1).contiguous())
                cov = cov.reshape(n, K + 1, nb)                      # (n, K+1, nb)
                tables.append(torch.matmul(lconj, cov.permute(2, 0, 1)).cpu().numpy())  # (nb, L+K, K+1)
                del right, cov
            del left, lconj
            segments += 1
        b, _ = kpm.bessel_coefficients(float(t - anchor), cfg)
        Kt = len(b) - 1
        if Kt > tables[0].shape[-1] - 1:
            raise NumericalError("internal spectral propagation order exceeded segment allocation")
        vac = np.empty((nb, na, ne))
        l_ = np.arange(L)[:, None]
        p_ = np.arange(Kt + 1)[None, :]
        for ai, table in enumerate(tables):
            q = table[:, :, :Kt + 1] @ b
            moments = np.sum(.5 * (q[:, l_ + p_] + q[:, np.abs(l_ - p_)]) * b.conj()[None, None, :], axis=2).real
            vac[:, ai, :] = moments @ G.T
        if previous is not None:
            h = float(t - prev_t)
            M = M + 2 * h * D + h * h / 3 * (2 * previous + vac)
            D = D + h / 2 * (previous + vac)
        if float(t) in output_indices:
            j = output_indices[float(t)]
            output["msd_A2/vac_integral"][:, :, j, :] = M
            output["diffusion_A2_per_fs/vac_integral"][:, :, j, :] = D
            output["vac_A2_per_fs2/vac_integral"][:, :, j, :] = vac
        previous, prev_t = vac, t
    if not cfg.include_vac:
        output.pop("vac_A2_per_fs2/vac_integral")
    return dos, output, {"algorithm": "segmented trace-first Chebyshev product VAC", "segments": segments,
                         "max_propagation_order": maxorder, "max_relative_S_norm_drift": maxnorm,
                         "integration_scheme": "piecewise linear VAC, simultaneous M/D recurrence",
                         "internal_nodes": len(times), "integration_dt_fs": cfg.integration_dt_fs,
                         "integration_validation": "UNVERIFIED until step-size convergence",
                         "seconds": time.perf_counter() - t0, "device_resident": "chains, velocity, tables"}


class Sampler:
    """Metric-corrected random vectors D^-1/2 p(W) xi (metric/sampling.py:11-46)."""

    def __init__(self, ops, cfg):
        coeff, center, half, report = kpm.sampler_coefficients(ops.host_S, ops.metric.diagonal, cfg.sampling_tol,
                                                               cfg.sampling_max_order)
        self.coeff, self.center, self.half, self.report = coeff, center, half, report
        self.ops = ops

    def transform(self, xi):
        torch = _torch()
        x = xi if isinstance(xi, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(xi, np.complex128)).cuda()
        return self.ops.metric.native.sample(x, self.coeff, self.center, self.half)


def sample_metric(seed, sample_ids, ops, cfg):
    if not hasattr(ops, "sampler"):
        ops.sampler = Sampler(ops, cfg)
    return ops.sampler.transform(kpm.random_phases(ops.n, seed, sample_ids))


def _quantity_keys(cfg, method):
    keys = ["msd_A2/commutator"] if method == "stepwise" else []
    if method == "spectral" or cfg.include_vac:
        keys += ["msd_A2/vac_integral", "diffusion_A2_per_fs/vac_integral"]
        if cfg.include_vac:
            keys += ["vac_A2_per_fs2/vac_integral"]
    if len(cfg.time_fs) > 1:
        keys += ["diffusion_A2_per_fs/msd_gradient"]
    return keys


def choose_stochastic_method(config):
    """'auto' resolves to stepwise (src/kubo_msd/dispatch.py:17-19)."""
    return "stepwise" if config.stochastic_method == "auto" else config.stochastic_method


def iter_stochastic_blocks(ops, config, method="stepwise", samples=None, parallel=None, bounds_report=None):
    """Stochastic transport blocks with the reference's array names and
    statistics (stochastic.py:122-228): stepwise commutator MSD with the
    optional spectral VAC route, or the spectral method alone."""
    if method not in ("stepwise", "spectral"):
        raise BackendUnavailable(f"unsupported stochastic method {method!r}")
    primary = "commutator" if method == "stepwise" else "vac_integral"
    ctx = parallel or ParallelContext()
    cfg = config
    if bounds_report is None:
        if getattr(cfg, "bounds_method", "arpack") == "device-lanczos":
            bounds_report = kpm.lanczos_spectral_bounds(ops, cfg)
        else:
            bounds_report = ctx.root_call("spectral bounds", lambda: kpm.estimate_spectral_bounds(
                ops.host_H, ops.host_S, ops.metric.s_lower, cfg))
    cfg = replace(cfg, spectral_bounds=bounds_report["bounds"])
    ns = cfg.nsamples if samples is None else samples.shape[1]
    nbk = (ns + cfg.statistics_block - 1) // cfg.statistics_block
    block_ids = owned_blocks(ns, cfg.statistics_block, ctx.rank, ctx.size)
    counts = np.array([min(cfg.statistics_block, ns - i * cfg.statistics_block) for i in range(nbk)])
    keys = _quantity_keys(cfg, method)
    shape = (len(block_ids), len(cfg.axes), len(cfg.time_fs), len(cfg.energy_eV))
    accum = {k: np.zeros(shape) for k in keys}
    local_dos = np.zeros((len(block_ids), len(cfg.energy_eV)))
    diagnostics, ids_used = [], []
    t0 = time.perf_counter()

    def run():
        for local_block, global_block in enumerate(block_ids):
            first_id = global_block * cfg.statistics_block
            end_id = min(ns, first_id + cfg.statistics_block)
            for first in range(first_id, end_id, cfg.sample_batch):
                last = min(first + cfg.sample_batch, end_id)
                ids = np.arange(first, last)
                B = sample_metric(cfg.seed, ids, ops, cfg) if samples is None else samples[:, first:last]
                if method == "stepwise":
                    dos, nums, diag = stepwise_samples(ops, cfg, B)
                    if cfg.include_vac:
                        _, extra, extra_diag = spectral_samples(ops, cfg, B)
                        nums.update(extra)
                        diag["additional_vac_path"] = extra_diag
                        diag["additional_cost_recorded"] = True
                else:
                    dos, nums, diag = spectral_samples(ops, cfg, B)
                if len(cfg.time_fs) > 1:
                    nums["diffusion_A2_per_fs/msd_gradient"] = kpm.msd_gradient(cfg.time_fs, nums["msd_A2/" + primary],
                                                                               axis=2)
                diagnostics.append(diag)
                ids_used.extend(ids.tolist())
                if not np.isfinite(dos).all():
                    raise NumericalError("nonfinite stochastic DOS")
                local_dos[local_block] += dos.sum(0)
                for key, values in nums.items():
                    if not np.isfinite(values).all():
                        raise NumericalError("nonfinite stochastic numerator")
                    accum[key][local_block] += values.sum(0)

    ctx.stage("random sample transport", run)
    sample_seconds = time.perf_counter() - t0
    rank_records = ctx.allgather({"rank": ctx.rank, "block_ids": block_ids, "sample_ids": ids_used,
                                  "sample_seconds": sample_seconds, "metric": ops.metric.diagnostics()})
    dos_blocks = ctx.gather_blocks(local_dos, block_ids, nbk)
    normalized = None
    if ctx.root:
        rho, stderr_dos, stat = kpm.estimate_ratio(dos_blocks, counts[:, None], counts)
        threshold = kpm.dos_floor(ops.n, cfg.spectral_bounds[1] - cfg.spectral_bounds[0], cfg)
        valid = np.isfinite(rho) & (rho > threshold)
        reason = np.where(valid, 0, REASON_LOW_DOS).astype("uint32")
        if stderr_dos is not None:
            uncertain = ~np.isfinite(stderr_dos) | (rho - 1.96 * stderr_dos <= 0)
            valid &= ~uncertain
            reason[uncertain] |= REASON_UNCERTAIN_TRACE
        if nbk < 8:
            reason |= REASON_INSUFFICIENT_BLOCKS
        static = {"dos_states_per_eV": rho, "dos_block_sums": dos_blocks, "block_counts": counts,
                  "sample_count": np.array(ns), "sample_ids": np.arange(ns)}
        if stderr_dos is not None:
            static["stderr_dos_states_per_eV"] = stderr_dos
        metadata = {"primary_estimator": primary,
                    "primary_diffusion_estimator": "msd_gradient" if method == "stepwise" else "vac_integral",
                    "resolved_config": cfg.as_dict() if hasattr(cfg, "as_dict") else {}, "spectral_report":
                    bounds_report, "dos_floor": threshold, "statistical_method": stat,
                    "sample_generator": "NumPy PCG64 SeedSequence([seed,sample_id]); unit modulus complex phases",
                    "sampling": getattr(getattr(ops, "sampler", None), "report", {"source": "caller supplied"}),
                    "sample_batch_diagnostics": diagnostics, "parallel": {**ctx.metadata(), "ranks": rank_records},
                    "backend": "b200"}
        normalized = (valid, reason, static, metadata)
    for start in range(0, len(cfg.time_fs), cfg.time_block):
        stop = min(start + cfg.time_block, len(cfg.time_fs))
        arrays = {}
        for key in keys:
            raw = ctx.gather_blocks(accum[key][:, :, start:stop, :], block_ids, nbk)
            if ctx.root:
                valid = normalized[0]
                value, se, _ = kpm.estimate_ratio(raw, dos_blocks, counts)
                value[..., ~valid] = np.nan
                arrays.update({key: value, "numerator_" + key: raw.sum(0) / ns, "numerator_block_sums/" + key:
                               raw.copy()})
                if se is not None:
                    se[..., ~valid] = np.nan
                    arrays["stderr_" + key] = se
        if ctx.root:
            valid, reason, static, metadata = normalized
            for estimator in {k.split("/")[-1] for k in keys}:
                r = reason.copy()
                if estimator == "vac_integral":
                    r |= REASON_INTEGRATION_UNVERIFIED
                dims = (len(cfg.axes), stop - start, len(cfg.energy_eV))
                arrays["valid/" + estimator] = np.broadcast_to(valid, dims).copy()
                arrays["reason_code/" + estimator] = np.broadcast_to(r, dims).copy()
            yield TransportBlock(start, cfg.time_fs[start:stop], arrays, static if start == 0 else {},
                                 metadata if start == 0 else {})
        else:
            yield None
