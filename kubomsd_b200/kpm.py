"""Host-side numerics of the stochastic-KPM path (small, FP64, NumPy/SciPy).

These are the scalar and small-array formulas around the device hot loop; each
follows the reference function it names so that the B200 path consumes the
same coefficients, grids and random phases as KuboMSD:

* spectral scaling and Bessel propagation coefficients
  (src/kubo_msd/solvers/chebyshev.py:8-30);
* Jackson damping and the reconstruction matrix G (src/kubo_msd/kernels/energy.py:12-37);
* random phases, NumPy PCG64 seeded by SeedSequence([seed, id])
  (src/kubo_msd/metric/sampling.py:8-9);
* SPD bounds, the metric inverse-square-root Chebyshev fit and the spectral
  bounds estimate (src/kubo_msd/metric/bounds.py:7-58, sampling.py:11-32);
* the paired block bootstrap and the MSD gradient
  (src/kubo_msd/observables/statistics.py:5-23, diffusion.py:4-6).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.fft import dct
from scipy.special import gammaln, jv

from .errors import KuboMSDError, NumericalError

HBAR_EV_FS = 0.6582119569509067  # eV fs (src/kubo_msd/units.py:1)


# ---------------------------------------------------------------- scaling
def scaling(cfg):
    if cfg.spectral_bounds is None:
        raise NumericalError("propagation needs resolved full spectral bounds")
    lo, hi = cfg.spectral_bounds
    return (lo + hi) / 2, (hi - lo) / 2


def bessel_coefficients(dt, cfg, weighted_tail=False):
    """b_m = J_m(a dt/hbar) (-i)^m (x2 for m >= 1) e^{-i c dt/hbar}; order from
    the absolute Bessel tail bound (weighted for the commutator)."""
    c, a = scaling(cfg)
    z = a * dt / HBAR_EV_FS
    az = abs(z)
    if az == 0:
        return np.array([1 + 0j]), {"order": 0, "tail_bound": 0.}
    chosen = None
    for k in range(max(1, int(np.ceil(az))), cfg.propagation_max_order + 1):
        n = k + 1
        ratio = az / (2 * (n + 1))
        if ratio >= 1:
            continue
        logbound = n * np.log(az / 2) - gammaln(n + 1) + az * az / (4 * (n + 1))
        bound = 2 * np.exp(min(logbound, 700)) / (1 - ratio)
        if weighted_tail:
            bound *= 4 * (n + 1) ** 2 / (1 - ratio) ** 2
        if bound <= cfg.propagation_tol:
            chosen = k
            break
    if chosen is None:
        raise NumericalError("propagation Bessel tail not converged before max order")
    m = np.arange(chosen + 1)
    b = jv(m, z) * (-1j) ** m
    b[1:] *= 2
    b *= np.exp(-1j * c * dt / HBAR_EV_FS)
    return b, {"order": chosen, "tail_bound": float(bound),
               "tail_policy": "absolute Bessel-series bound; weighted for commutator if requested"}


# ---------------------------------------------------------------- energy kernels
def validate_spectral_window(eps, bounds):
    e = np.asarray(eps, float)
    b = np.asarray(bounds, float)
    if b.shape != (2,) or not np.isfinite(b).all() or b[1] <= b[0]:
        raise KuboMSDError("invalid spectral bounds")
    if not np.isfinite(e).all() or np.any(e < b[0]) or np.any(e > b[1]):
        raise KuboMSDError("spectral bounds do not contain full spectrum")
    return float((b[0] + b[1]) / 2), float((b[1] - b[0]) / 2)


def jackson_coefficients(n_moments):
    L = int(n_moments)
    if L != n_moments or L < 1:
        raise KuboMSDError("n_moments must be positive integer")
    m = np.arange(L)
    theta = np.pi / (L + 1)
    g = ((L + 1 - m) * np.cos(m * theta) + np.sin(m * theta) / np.tan(theta)) / (L + 1)
    g[0] = 1.
    return g


def reconstruction_matrix(E, bounds, L):
    c, a = validate_spectral_window([], bounds)
    E = np.asarray(E, float)
    x = (E - c) / a
    if not np.isfinite(x).all() or np.any(np.abs(x) >= 1):
        raise KuboMSDError("Jackson output energies must lie strictly inside full spectral bounds")
    g = jackson_coefficients(L)
    g[1:] *= 2
    return np.cos(np.arccos(x)[:, None] * np.arange(L)) * g / (np.pi * a * np.sqrt(1 - x * x)[:, None])


def dos_floor(n_orbitals, width, cfg):
    w = cfg.sigma_eV if cfg.kernel == "gaussian" else (cfg.spectral_bounds[1] - cfg.spectral_bounds[0]) / (
        2 * cfg.n_moments)
    return max(cfg.rho_abs, cfg.rho_rel * n_orbitals / max(width, w))


# ---------------------------------------------------------------- sampling
def random_phases(n, seed, sample_ids):
    return np.column_stack([np.exp(2j * np.pi * np.random.Generator(np.random.PCG64(
        np.random.SeedSequence([int(seed), int(i)]))).random(n)) for i in sample_ids])


def hermitian(A, name="matrix", tol=1e-10):
    """Canonical complex CSR with the reference's Hermiticity check
    (src/kubo_msd/validation.py:13-18)."""
    A = sp.csr_matrix(A, dtype=np.complex128)
    A.sum_duplicates()
    A.sort_indices()
    if len(A.shape) != 2 or A.shape[0] != A.shape[1] or not A.shape[0] or not np.isfinite(A.data).all():
        raise KuboMSDError(f"{name}: invalid square finite matrix")
    n = sp.linalg.norm(A)
    err = sp.linalg.norm(A - A.getH())
    if err > (tol * n if n else 0):
        raise KuboMSDError(f"{name}: not Hermitian (relative error {err / max(n, np.finfo(float).tiny):g})")
    return A


def spd_bounds(S, *, allow_dense=True):
    S = hermitian(S, "overlap")
    diag = S.diagonal().real
    radii = np.asarray(abs(S).sum(axis=1)).ravel() - np.abs(diag)
    lo = float(np.min(diag - radii))
    hi = float(np.max(diag + radii))
    if lo > 0:
        return lo, hi, {"source": "Gershgorin", "certified": True}
    n = S.shape[0]
    if n <= 2 and not allow_dense:
        lo = float(diag[0]) if n == 1 else float((diag[0] + diag[1]) / 2 - np.hypot((diag[0] - diag[1]) / 2,
                                                                                   abs(S[0, 1])))
        source = "analytic one/two dimensional SPD check"
    elif n <= 128 and allow_dense:
        ev = np.linalg.eigvalsh(S.toarray())
        lo = float(ev[0])
        hi = float(ev[-1])
        source = "small-matrix eigenvalues of S"
    else:
        v0 = np.random.default_rng(9021).normal(size=n)
        e, V = sp.linalg.eigsh(S, k=1, which="SA", tol=1e-12, v0=v0)
        residual = float(np.linalg.norm(S @ V[:, 0] - e[0] * V[:, 0]))
        lo = float(e[0] - 10 * residual)
        source = "smallest Ritz value of S minus 10 residuals (estimated)"
    if lo <= 0 or not np.isfinite([lo, hi]).all():
        raise NumericalError("overlap is not positive definite or SPD verification failed")
    return lo * (1 - 1e-10), hi * (1 + 1e-10), {"source": source,
                                                 "certified": n <= 2 or (n <= 128 and allow_dense)}


def sampler_coefficients(S, diagonal, sampling_tol, sampling_max_order):
    """Chebyshev coefficients of w^-1/2 over the spectrum of D^-1/2 S D^-1/2
    (src/kubo_msd/metric/sampling.py:11-32): (coeff, center, half, report)."""
    z = 1 / np.sqrt(diagonal)
    W = sp.diags(z) @ sp.csr_matrix(S) @ sp.diags(z)
    lo, hi, breport = spd_bounds(W)
    center, half = (hi + lo) / 2, (hi - lo) / 2
    report = {"bounds": [lo, hi], "bounds_report": breport, "preconditioner": "diagonal congruence",
              "target": sampling_tol}
    if half < 1e-14 * center:
        report.update(order=0, max_relative_grid_error=0.)
        return np.array([1 / np.sqrt(center)]), center, half, report
    for order in (2 ** k for k in range(4, 20)):
        order = min(order, sampling_max_order)
        n = max(2 * order, 64)
        theta = np.pi * (np.arange(n) + .5) / n
        f = 1 / np.sqrt(center + half * np.cos(theta))
        coef = dct(f, type=2) / n
        coef[0] *= .5
        coef = coef[:order + 1]
        xx = np.cos(np.linspace(0, np.pi, max(4097, 8 * order + 1)))
        error = np.max(np.abs(np.polynomial.chebyshev.chebval(xx, coef) * np.sqrt(center + half * xx) - 1))
        if error < sampling_tol * .25:
            report.update(order=order, max_relative_grid_error=float(error))
            return coef, center, half, report
        if order >= sampling_max_order:
            break
    raise NumericalError("metric inverse sqrt polynomial failed sampling tolerance")


def estimate_spectral_bounds(H, S, s_lower, cfg):
    """Generalized extremal Ritz values with margin, or user bounds checked
    against them (src/kubo_msd/metric/bounds.py:26-58)."""
    n = H.shape[0]
    hnorm = float(np.asarray(abs(H).sum(axis=1)).max())
    b = hnorm / s_lower
    if b == 0 and cfg.spectral_bounds is None:
        raise NumericalError("fully degenerate zero spectrum needs explicit spectral bounds")
    conservative = (-b, b)
    if n <= 2:
        import scipy.linalg as la
        extremal = la.eigvalsh(H.toarray(), S.toarray(), subset_by_index=[0, n - 1])
        residuals = [0., 0.]
    else:
        extrema, residuals = [], []
        for which in ("SA", "LA"):
            vals = []
            for seed in (811, 812):
                e, v = sp.linalg.eigsh(H, M=S, k=1, which=which, tol=1e-11,
                                       v0=np.random.default_rng(seed).normal(size=n))
                r = np.linalg.norm(H @ v[:, 0] - e[0] * (S @ v[:, 0])) / np.linalg.norm(v[:, 0])
                vals.append(float(e[0]))
                residuals.append(float(r))
            extrema.append(min(vals) if which == "SA" else max(vals))
        extremal = np.array(extrema)
    lo = float(extremal[0])
    hi = float(extremal[-1])
    if cfg.spectral_bounds is not None:
        bounds = cfg.spectral_bounds
        if bounds[0] >= lo or bounds[1] <= hi:
            raise NumericalError("requested spectral bounds must enclose estimated full spectrum with margin")
        source = "user bounds checked against generalized extremal Ritz values"
        certified = False
    else:
        if hi - lo <= np.finfo(float).eps * max(abs(lo), abs(hi), 1):
            raise NumericalError("degenerate spectrum needs explicit bounds")
        margin = max(.01 * (hi - lo), 10 * max(residuals) / s_lower)
        bounds = (lo - margin, hi + margin)
        certified = False
        source = "two-start generalized Ritz extrema plus margin"
    return {"bounds": tuple(bounds), "source": source, "certified": certified, "residuals": residuals,
            "conservative_bounds": conservative, "extrema": [lo, hi]}


def lanczos_spectral_bounds(ops, cfg, steps=160, seed=811):
    """Extremal generalized eigenvalues of (H, S) by Lanczos on the device.

    The device replacement of the host ARPACK estimate (bounds.py:26-58) for
    large operators: `steps` Lanczos iterations in the S inner product
    (w = S^-1 H v, alpha = <v, H v>, beta = |w|_S) run on the device by
    kmsd_engine_lanczos with the scalars kept there, then the extreme Ritz
    values of the tridiagonal matrix and their residual bounds
    beta_k |e_k^T y|.  The result goes
    through the reference's margin rule: max(1 % of the width, 10 residuals /
    s_lower) on each side, or the enclosure check of user bounds.  Ritz values
    lie inside the spectrum, so the margin is what makes the window enclose
    it.
    """
    import torch
    n = ops.n
    rng = np.random.default_rng(seed)
    v = torch.from_numpy(rng.normal(size=(n, 1)) + 0j).cuda()
    # every step on the device, one read-back of the scalars at the end
    a_all, b_all = ops.native.lanczos(v, min(steps, n))
    alphas, betas = [], []
    for alpha, beta in zip(a_all, b_all):
        alphas.append(float(alpha))
        betas.append(float(beta))
        if beta <= 1e-14 * max(abs(alpha), 1.):
            break
    import scipy.linalg as la
    k = len(alphas)
    T = np.diag(alphas) + np.diag(betas[:k - 1], 1) + np.diag(betas[:k - 1], -1)
    e, y = la.eigh(T)
    res = np.abs(betas[k - 1] * y[-1, :])
    lo, hi = float(e[0]), float(e[-1])
    residuals = [float(res[0]), float(res[-1])]
    hnorm = float(np.asarray(abs(ops.host_H).sum(axis=1)).max())
    b = hnorm / ops.metric.s_lower
    if cfg.spectral_bounds is not None:
        bounds = cfg.spectral_bounds
        if bounds[0] >= lo or bounds[1] <= hi:
            raise NumericalError("requested spectral bounds must enclose estimated full spectrum with margin")
        source = "user bounds checked against device Lanczos extremal Ritz values"
    else:
        if hi - lo <= np.finfo(float).eps * max(abs(lo), abs(hi), 1):
            raise NumericalError("degenerate spectrum needs explicit bounds")
        margin = max(.01 * (hi - lo), 10 * max(residuals) / ops.metric.s_lower)
        bounds = (lo - margin, hi + margin)
        source = f"device Lanczos ({k} steps) extremal Ritz values plus margin"
    return {"bounds": tuple(bounds), "source": source, "certified": False, "residuals": residuals,
            "conservative_bounds": (-b, b), "extrema": [lo, hi], "lanczos_steps": k}


# ---------------------------------------------------------------- statistics
def estimate_ratio(block_numerators, block_dos, counts, n_resamples=256):
    A = np.asarray(block_numerators, float)
    D = np.asarray(block_dos, float)
    counts = np.asarray(counts, int)
    if A.shape[0] != len(counts) or D.shape[0] != len(counts) or np.any(counts <= 0):
        raise KuboMSDError("inconsistent statistical blocks/counts")
    if D.ndim != 2 or A.shape[-1] != D.shape[-1]:
        if D.shape == (len(counts), 1):
            D = np.broadcast_to(D, (len(counts), A.shape[-1]))
        else:
            raise KuboMSDError("statistical denominator must be (blocks,energy)")
    totalD = D.sum(0)
    totalA = A.sum(0)
    value = np.divide(totalA, totalD, out=np.full_like(totalA, np.nan), where=totalD != 0)
    status = {"method": "paired block bootstrap of sums", "n_blocks": len(counts), "counts": counts.tolist(),
              "reliable_interval": len(counts) >= 8, "bootstrap_seed": 21491, "n_resamples": n_resamples,
              "input_accumulation": "sum; actual unequal counts retained"}
    if len(counts) < 2:
        return value, None, status
    rng = np.random.default_rng(21491)
    indices = rng.integers(len(counts), size=(n_resamples, len(counts)))
    weights = np.zeros((n_resamples, len(counts)))
    for j, row in enumerate(indices):
        weights[j] = np.bincount(row, minlength=len(counts))
    resampledA = np.tensordot(weights, A, axes=(1, 0))
    resampledD = weights @ D
    resampledD = resampledD.reshape((n_resamples,) + (1,) * (A.ndim - 2) + (A.shape[-1],))
    ratios = np.divide(resampledA, resampledD, out=np.full_like(resampledA, np.nan), where=resampledD != 0)
    stderr = np.std(ratios, axis=0, ddof=1)
    return value, stderr, status


def msd_gradient(time_fs, msd, axis=1):
    if len(time_fs) < 2:
        return None
    return .5 * np.gradient(msd, np.asarray(time_fs), axis=axis, edge_order=2 if len(time_fs) > 2 else 1)
