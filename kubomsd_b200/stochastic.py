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

from . import devstats, kpm
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


def projected_quadratic(B, ops, cfg, device=False):
    """(G mu)^T with mu the device moments of B (chebyshev.py:50-54).  The
    projection runs on the device; device=True returns the device tensor
    (b, ne), otherwise a host array."""
    from . import devstats
    torch = _torch()
    c, a = kpm.scaling(cfg)
    Bd = B if isinstance(B, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(B, np.complex128)).cuda()
    mu = ops.native.moments(Bd, cfg.n_moments, c, a)
    if not isinstance(mu, torch.Tensor):
        mu = torch.from_numpy(np.ascontiguousarray(mu)).cuda()
    out = devstats.project(mu, devstats.reconstruction_matrix(cfg.energy_eV, cfg.spectral_bounds, cfg.n_moments))
    return out if device else out.cpu().numpy()


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


def _snorm_device(ops, B):
    return ops.inner(B, B).real


def stepwise_samples(ops, cfg, samples, device=False):
    """Velocity-driven augmented commutator MSD (stepwise.py:20-38) with the
    state resident on the device.  Returns (dos, {'msd_A2/commutator': ...},
    diag); with device=True the arrays stay device tensors.  The S-norm drift
    of every interval is kept on the device and checked once at the end,
    reporting the first interval over the tolerance as the reference does."""
    torch = _torch()
    initial = samples if isinstance(samples, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(samples, dtype=np.complex128))
    initial = initial.to("cuda", torch.complex128).contiguous()
    nb = initial.shape[1]
    na, nt, ne = len(cfg.axes), len(cfg.time_fs), len(cfg.energy_eV)
    t0 = time.perf_counter()
    dos = projected_quadratic(initial, ops, cfg, device=True)
    total = torch.cat([initial] + [torch.zeros_like(initial) for _ in cfg.axes], dim=1).contiguous()
    output = torch.zeros((nb, na, nt, ne), dtype=torch.float64, device=initial.device)
    c, a = kpm.scaling(cfg)
    orders = []
    norm0 = _snorm_device(ops, initial)
    tiny = np.finfo(float).tiny
    drifts = torch.zeros(max(nt, 1), dtype=torch.float64, device=initial.device)
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
            norm = _snorm_device(ops, total[:, :nb].contiguous())
            drifts[j] = torch.max(torch.abs(norm - norm0) / torch.clamp(norm0, min=tiny))
        for ai in range(na):
            output[:, ai, j, :] = projected_quadratic(total[:, (ai + 1) * nb:(ai + 2) * nb].contiguous(), ops, cfg,
                                                      device=True)
    d = drifts.cpu().numpy()
    over = np.nonzero(np.maximum.accumulate(d) > drift_tolerance(cfg))[0]
    if len(over):
        raise NumericalError(f"stepwise base propagation S-norm drift {float(np.max(d[:over[0] + 1])):g}")
    drift = float(d.max()) if len(d) else 0.
    if not device:
        dos, output = dos.cpu().numpy(), output.cpu().numpy()
    return dos, {"msd_A2/commutator": output}, {
        "algorithm": "velocity-driven augmented Chebyshev commutator", "segments": segments,
        "max_propagation_order": max(orders, default=0), "max_relative_S_norm_drift": drift,
        "seconds": time.perf_counter() - t0, "device_resident": True}


def _segment_nodes(times, segment_fs):
    """The reference's segmentation of the integration nodes (spectral.py:25-32):
    for each segment its anchor, its end, and the nodes it serves."""
    segs, anchor, next_anchor, have, prev_t = [], 0., -1., False, 0.
    for t in times:
        if not have or t > next_anchor + 1e-14:
            anchor = 0. if not have else float(prev_t)
            next_anchor = min(max(anchor + segment_fs, float(t)), float(times[-1]))
            segs.append([anchor, next_anchor, []])
            have = True
        segs[-1][2].append(float(t))
        prev_t = t
    return segs


def spectral_samples(ops, cfg, samples):
    """Segmented trace-first Chebyshev product VAC (spectral.py:15-53).

    Per segment the anchors are propagated on the device, the right chains
    T_k(Ht) v_a (k <= K) are built by the engine and the velocity is applied
    to them on the device.  The correlation tables
    tables[b, j, k] = sum_n conj(T_j(Ht) c)[n, b] cov[n, k, b] (j < L+K) are
    accumulated by the engine while it generates the left chain
    (kmsd_engine_chain_correlate: a ring of chain blocks contracted by a repo
    kernel, so the (L+K, N, b) chain is never stored).  The per-node Bessel
    contraction, product rule T_l T_p = (T_l+p + T_|l-p|)/2 and Jackson
    projection run on the device for all nodes of a segment at once
    (kmsd_vac_nodes); the M/D recurrence runs in FP64 on the host in the
    reference's order.
    """
    from .config import resolve_time_grid
    from .native import vac_nodes
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
    anchor = 0.
    maxorder = segments = 0
    maxnorm = 0.
    c, a = kpm.scaling(cfg)
    M = np.zeros((nb, na, ne))
    D = np.zeros_like(M)
    previous, prev_t = None, 0.
    for seg_anchor, seg_end, nodes in _segment_nodes(times, cfg.segment_fs):
        if seg_anchor > anchor:
            both = torch.cat([c_anchor] + v_anchor, dim=1).contiguous()
            both, report = propagate(both, seg_anchor - anchor, ops, cfg)
            maxnorm = max(maxnorm, report["relative_S_norm_drift"])
            c_anchor = both[:, :nb].contiguous()
            v_anchor = [both[:, (i + 1) * nb:(i + 2) * nb].contiguous() for i in range(na)]
        anchor = seg_anchor
        coeff, _ = kpm.bessel_coefficients(seg_end - anchor, cfg)
        K = len(coeff) - 1
        maxorder = max(maxorder, K)
        # device memory of the segment: the left-chain ring (32 blocks), the right
        # chains with their velocity, and the tables
        estimate = 16 * nb * (n * (32 + 2 * na * (K + 1) + 4) + na * (L + K) * (K + 1)) + 24 * nb * na * nt * ne
        if estimate > cfg.memory_limit_gb * 1024 ** 3:
            raise NumericalError("spectral workspace exceeds memory budget; reduce sample_batch/segment_fs or "
                                 "increase explicit budget")
        covs = []
        for ai, axis in enumerate(cfg.axes):
            right = ops.native.chain(v_anchor[ai], K + 1, c, a)  # (K+1, n, nb) on the device
            cov = ops.apply_v_cov(axis, right.permute(1, 0, 2).reshape(n, -1).contiguous())
            del right
            covs.append(cov.reshape(n, K + 1, nb))
        cov = covs[0] if na == 1 else torch.cat(covs, dim=1).contiguous()  # (n, na (K+1), nb)
        del covs
        tables = ops.native.chain_correlate(c_anchor, cov, L + K, c, a)  # (nb, L+K, na (K+1)) on the device
        del cov
        segments += 1
        node_coeffs = [kpm.bessel_coefficients(float(t - anchor), cfg)[0] for t in nodes]
        if max(len(b) for b in node_coeffs) > K + 1:
            raise NumericalError("internal spectral propagation order exceeded segment allocation")
        vac_all = np.empty((len(nodes), nb, na, ne))
        for ai in range(na):
            tab = tables[:, :, ai * (K + 1):(ai + 1) * (K + 1)].contiguous()
            vac_all[:, :, ai, :] = vac_nodes(tab, node_coeffs, G, ops.native.lib)
        del tables
        for t, vac in zip(nodes, vac_all):
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
                         "seconds": time.perf_counter() - t0,
                         "device_resident": "chains, velocity, correlation tables, per-node tail"}


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
    """Metric-corrected random vectors of the given sample ids, with the
    phases generated on the device (devstats.random_phases)."""
    if not hasattr(ops, "sampler"):
        ops.sampler = Sampler(ops, cfg)
    return ops.sampler.transform(devstats.random_phases(ops.n, seed, sample_ids))


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


def sample_working_bytes(cfg, n, method, batch):
    """Device bytes one sample batch holds at its peak: the augmented state
    and the engine's recurrence and series buffers (six blocks of the
    [psi | phi] width), the moment buffers, and for the VAC route the
    left-chain ring, the right chains with their velocity and the tables."""
    na, nt, ne = len(cfg.axes), len(cfg.time_fs), len(cfg.energy_eV)
    cols = batch * (1 + na)
    working = 16 * n * cols * 6 + 16 * n * batch * 4 + 8 * batch * na * nt * ne * 3
    if method == "spectral" or cfg.include_vac:
        a = .5 * (cfg.spectral_bounds[1] - cfg.spectral_bounds[0]) if cfg.spectral_bounds else 1.
        order = int(np.ceil(a * cfg.segment_fs / kpm.HBAR_EV_FS)) + 64
        working += 16 * n * batch * (32 + 3 * na * (order + 1)) + 16 * batch * na * (cfg.n_moments + order) * (
            order + 1)
    return working


def fit_sample_batch(cfg, n, method, ns):
    """The reference GPU edition's batch halving (kubo_msd_gpu/.../solvers/
    stochastic_gpu.py:31-45): the sample batch is halved until twice its
    working set fits both the configured memory budget and the device's free
    memory; a batch of one that does not fit is an error."""
    torch = _torch()
    batch = max(1, min(cfg.sample_batch, cfg.statistics_block, ns))
    limit = min(cfg.memory_limit_gb * 1024 ** 3, torch.cuda.mem_get_info()[0])
    while 2 * sample_working_bytes(cfg, n, method, batch) > limit:
        if batch == 1:
            raise NumericalError("stochastic sample workspace exceeds the device memory budget; raise "
                                 "memory_limit_gb or reduce the energy/time grids")
        batch = max(1, batch // 2)
    return batch


def check_transport_budget(cfg, keys, nblocks, nlocal, n, ctx):
    """The reference's transport workspace gate (stochastic.py:139-158), with
    the block sums held in device memory instead of a scratch file: the
    per-batch working set, the rank's block sums (against the device's free
    memory) and the root's merge and bootstrap slabs must fit
    cfg.memory_limit_gb, else NumericalError."""
    torch = _torch()
    na, nt, ne = len(cfg.axes), len(cfg.time_fs), len(cfg.energy_eV)
    working = min(cfg.sample_batch, cfg.statistics_block) * na * nt * ne * 8 * len(keys) * 2
    slab = nblocks * na * min(cfg.time_block, nt) * ne * 8
    root_working = slab * (len(keys) + 6) + nblocks * ne * 16
    if nblocks > 1:
        root_working += 4 * 256 * na * min(cfg.time_block, nt) * ne * 8 + 2 * 256 * nblocks * 8 + 2 * 256 * ne * 8
    if max(working, root_working if ctx.root else 0) > cfg.memory_limit_gb * 1024 ** 3:
        raise NumericalError("sample/merge/bootstrap workspace exceeds memory budget; reduce "
                             "sample_batch/time_block/energy count or raise explicit budget")
    block_sums = nlocal * na * nt * ne * 8 * len(keys) + nlocal * ne * 8
    free = torch.cuda.mem_get_info()[0]
    if block_sums > .8 * free:
        raise NumericalError("insufficient device memory for the paired statistical block sums")


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
    cfg = replace(cfg, sample_batch=fit_sample_batch(cfg, ops.n, method, ns))
    nbk = (ns + cfg.statistics_block - 1) // cfg.statistics_block
    block_ids = owned_blocks(ns, cfg.statistics_block, ctx.rank, ctx.size)
    counts = np.array([min(cfg.statistics_block, ns - i * cfg.statistics_block) for i in range(nbk)])
    keys = _quantity_keys(cfg, method)
    shape = (len(block_ids), len(cfg.axes), len(cfg.time_fs), len(cfg.energy_eV))
    torch = _torch()
    check_transport_budget(cfg, keys, nbk, len(block_ids), ops.n, ctx)
    # block sums stay on the device; the MSD gradient is linear, so it is taken
    # of the block sums once the samples are in
    gradient_key = "diffusion_A2_per_fs/msd_gradient"
    dev_keys = [k for k in keys if k != gradient_key]
    accum = {k: torch.zeros(shape, dtype=torch.float64, device="cuda") for k in dev_keys}
    local_dos = torch.zeros((len(block_ids), len(cfg.energy_eV)), dtype=torch.float64, device="cuda")
    diagnostics, ids_used = [], []
    t0 = time.perf_counter()

    def as_dev(x):
        return x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x, np.float64)).cuda()

    def run():
        for local_block, global_block in enumerate(block_ids):
            first_id = global_block * cfg.statistics_block
            end_id = min(ns, first_id + cfg.statistics_block)
            for first in range(first_id, end_id, cfg.sample_batch):
                last = min(first + cfg.sample_batch, end_id)
                ids = np.arange(first, last)
                B = sample_metric(cfg.seed, ids, ops, cfg) if samples is None else samples[:, first:last]
                if method == "stepwise":
                    dos, nums, diag = stepwise_samples(ops, cfg, B, device=True)
                    if cfg.include_vac:
                        _, extra, extra_diag = spectral_samples(ops, cfg, B)
                        nums.update(extra)
                        diag["additional_vac_path"] = extra_diag
                        diag["additional_cost_recorded"] = True
                else:
                    dos, nums, diag = spectral_samples(ops, cfg, B)
                diagnostics.append(diag)
                ids_used.extend(ids.tolist())
                local_dos[local_block] += as_dev(dos).sum(0)
                for key, values in nums.items():
                    accum[key][local_block] += as_dev(values).sum(0)
        # one check of the device sums: a nonfinite contribution leaves them nonfinite
        if not bool(torch.isfinite(local_dos).all()):
            raise NumericalError("nonfinite stochastic DOS")
        for values in accum.values():
            if not bool(torch.isfinite(values).all()):
                raise NumericalError("nonfinite stochastic numerator")
        if gradient_key in keys:
            grad = kpm.msd_gradient(cfg.time_fs, accum["msd_A2/" + primary].cpu().numpy(), axis=2)
            accum[gradient_key] = as_dev(grad) if grad is not None else torch.zeros(shape, dtype=torch.float64,
                                                                                    device="cuda")

    ctx.stage("random sample transport", run)
    sample_seconds = time.perf_counter() - t0
    rank_records = ctx.allgather({"rank": ctx.rank, "block_ids": block_ids, "sample_ids": ids_used,
                                  "sample_seconds": sample_seconds, "metric": ops.metric.diagnostics()})

    def gathered(local):
        """Global block sums on root as a device tensor (serial: the local ones)."""
        if ctx.dist is None:
            ctx.gather_blocks(np.empty((len(block_ids), 0)), block_ids, nbk)  # coverage check only
            return local
        full = ctx.gather_blocks(local.cpu().numpy(), block_ids, nbk)
        return as_dev(full) if ctx.root else None

    dos_dev = gathered(local_dos)
    dos_blocks = dos_dev.cpu().numpy() if ctx.root else None
    normalized = None
    if ctx.root:
        rho_d, se_d, stat = devstats.estimate_ratio(dos_dev, as_dev(counts[:, None].astype(float)), counts)
        rho = rho_d.cpu().numpy()
        stderr_dos = se_d.cpu().numpy() if se_d is not None else None
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
            raw_d = gathered(accum[key][:, :, start:stop, :].contiguous())
            if ctx.root:
                valid = normalized[0]
                value_d, se_d, _ = devstats.estimate_ratio(raw_d, dos_dev, counts)
                value = value_d.cpu().numpy()
                raw = raw_d.cpu().numpy()
                value[..., ~valid] = np.nan
                arrays.update({key: value, "numerator_" + key: raw.sum(0) / ns, "numerator_block_sums/" + key:
                               raw})
                if se_d is not None:
                    se = se_d.cpu().numpy()
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
