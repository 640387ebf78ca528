"""ORACLE — test infrastructure only, never product code.

CPU restatement (NumPy/SciPy, complex128) of the reference's stochastic-KPM
transport hot path, used by tests/ and bench.py's CPU arm as the checker of the
B200 engine.  Each function cites the reference code it restates (paths are
within the KuboMSD project).  Parity of this restatement is pinned two ways
(tests/test_oracle_pin.py): against golden vectors produced by running the
reference itself (tests/golden/, generated by tests/golden/make_golden.py) and,
where `oracle/_ref` has been built, live against the reference's compiled
engine on random inputs.

Vector blocks are (N, b) complex128 arrays, as the reference's Dense.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.fft import dct
from scipy.special import gammaln, jv

HBAR_EV_FS = 0.6582119569509067  # src/kubo_msd/units.py:1


class MetricFailure(RuntimeError):
    """Restates MetricFailure (cpp/native.cpp:139-143) with its diagnostics."""

    def __init__(self, message, diagnostics):
        super().__init__(message)
        self.diagnostics = diagnostics


def canonical(A):
    """complex128 CSR with duplicates summed and sorted indices
    (src/kubo_msd/backends/native.py:42-46)."""
    A = sp.csr_matrix(A, dtype=np.complex128, copy=True)
    A.sum_duplicates()
    A.sort_indices()
    return A


def dense(B):
    """Dense(const Arr&) validation (cpp/native.cpp:31-40)."""
    B = np.asarray(B)
    if B.ndim != 2 or B.shape[0] < 1 or B.shape[1] < 1:
        raise ValueError("expected nonempty finite (N,batch) array")
    B = np.array(B, dtype=np.complex128, order="C")
    if not np.isfinite(B).all():
        raise ValueError("expected finite (N,batch) array")
    return B


class Metric:
    """Metric (cpp/native.cpp:150-480): diagonal or block-Jacobi PCG and sampling."""

    def __init__(self, S, diagonal, blocks=(), policy="fixed", interval=32, gap_ratio=.1):
        self.S = canonical(S)
        self.n = self.S.shape[0]
        self.diag = np.asarray(diagonal, float)
        if self.diag.shape != (self.n,) or not np.all(self.diag > 0) or not np.isfinite(self.diag).all():
            raise ValueError("invalid metric diagonal")
        self.blocks = [(int(a), int(b), np.asarray(L, complex)) for a, b, L in blocks]
        self.adaptive = policy == "adaptive"
        self.interval = interval
        self.gap_ratio = gap_ratio
        self.calls = self.iterations = self.refreshes = self.checks = self.restarts = 0
        self.max_relative = 0.

    def mul(self, X):
        return self.S @ X

    def precondition(self, r):
        """Diagonal z = r/d or per-block L L^H solves (native.cpp:259-297)."""
        if not self.blocks:
            return r / self.diag[:, None]
        z = np.empty_like(r)
        for a, b, L in self.blocks:
            y = np.linalg.solve(L, r[a:b])
            z[a:b] = np.linalg.solve(L.conj().T, y)
        return z

    @staticmethod
    def dot(a, b):
        return np.sum(a.conj() * b, axis=0)

    @staticmethod
    def norms(a):
        return np.sqrt(np.sum(np.abs(a) ** 2, axis=0))

    def solve(self, B, rtol, atol, maxiter):
        """Batched PCG, column by column semantics of Metric::solve
        (cpp/native.cpp:313-452)."""
        B = dense(B)
        if B.shape[0] != self.n or rtol < 0 or atol < 0 or maxiter < 1:
            raise ValueError("invalid metric RHS shape/tolerances")
        n, b = B.shape
        safe = np.max(np.maximum(np.abs(B.real), np.abs(B.imag)), axis=0)
        safe = np.where(safe == 0., 1., safe)
        q = B / safe
        bn = self.norms(q)
        threshold = np.maximum(rtol * bn, atol / safe)
        active = bn > threshold
        r = q.copy()
        y = np.zeros_like(q)
        z = self.precondition(r)
        p = z.copy()
        rz = self.dot(r, z).real
        p[:, ~active] = 0
        iterations = np.zeros(b, np.int64)
        breakdown = np.zeros(b, bool)
        any_breakdown = False
        for k in range(maxiter):
            if not active.any():
                break
            sp_ = self.mul(p)
            curv = self.dot(p, sp_)
            bad = active & (~(curv.real > 0) | ~np.isfinite(curv.real) | ~np.isfinite(curv.imag)
                            | (np.abs(curv.imag) > 1e-10 * np.maximum(np.abs(curv.real),
                                                                     np.finfo(float).tiny)))
            breakdown |= bad
            if bad.any():
                any_breakdown = True
                break
            alpha = np.where(active, rz / np.where(active, curv.real, 1.), 0.)
            y += p * alpha
            r -= sp_ * alpha
            iterations += active
            rn = self.norms(r)
            refresh = (k + 1) % self.interval == 0
            restart = np.zeros(b, bool)
            candidate = bool(np.any(active & (rn <= threshold)))
            if refresh or (self.adaptive and candidate):
                truth = q - self.mul(y)
                self.refreshes += 1
                self.checks += 1
                tn = self.norms(truth)
                for j in np.flatnonzero(active):
                    if self.adaptive:
                        gap = np.sqrt(np.sum(np.abs(truth[:, j] - r[:, j]) ** 2))
                        restart[j] = tn[j] > threshold[j] and (
                            gap > self.gap_ratio * max(tn[j], threshold[j]) or rn[j] <= threshold[j])
                    else:
                        restart[j] = True
                    active[j] = tn[j] > threshold[j]
                    if restart[j]:
                        self.restarts += 1
                        r[:, j] = truth[:, j]
            elif not self.adaptive:
                active &= rn > threshold
            z = self.precondition(r)
            newrz = self.dot(r, z).real
            beta = np.where(active, newrz / np.where(rz != 0, rz, 1.), 0.)
            rz = newrz
            p = np.where(active[None, :], z + np.where(restart[None, :], 0, p * beta), 0)
        residual = q - self.mul(y)
        self.checks += 1
        rn = self.norms(residual)
        converged = (rn <= threshold) & ~breakdown
        relative = np.where(bn > 0, rn / np.where(bn > 0, bn, 1.), 0.)
        true_residual = rn * safe
        self.max_relative = max(self.max_relative, float(relative.max()))
        finite = np.isfinite(y).all(axis=0)
        with np.errstate(over="ignore", invalid="ignore"):
            scaled = np.where(finite[None, :], y * safe, y)
        finite &= np.isfinite(scaled).all(axis=0)
        converged &= finite
        self.calls += 1
        self.iterations += int(iterations.max())
        report = dict(converged=converged.tolist(), breakdown=breakdown.tolist(), iterations=iterations.tolist(),
                      true_residual=true_residual.tolist(), relative_residual=relative.tolist())
        ok = converged.all() and not any_breakdown and finite.all()
        if not ok:
            message = ("S solve solution is nonfinite or not representable in complex128 after rescaling"
                       if not finite.all() else "PCG non-positive/complex curvature breakdown"
                       if any_breakdown else "S solve failed true-residual acceptance")
            raise MetricFailure(message, report)
        return scaled, report

    def sample(self, xi, coeff, center, half):
        """Clenshaw evaluation of D^-1/2 p(W) xi (cpp/native.cpp:453-479)."""
        xi = dense(xi)
        z = 1 / np.sqrt(self.diag)

        def action(a):
            return (z[:, None] * self.mul(a * z[:, None]) - center * a) / half

        coeff = np.asarray(coeff, float)
        if len(coeff) > 1:
            b1 = np.zeros_like(xi)
            b2 = np.zeros_like(xi)
            for k in range(len(coeff) - 1, 0, -1):
                b0 = 2. * action(b1) - b2 + coeff[k] * xi
                b2, b1 = b1, b0
            out = action(b1) - b2
        else:
            out = np.zeros_like(xi)
        return z[:, None] * (out + coeff[0] * xi)


class Engine:
    """Engine (cpp/native.cpp:488-610)."""

    def __init__(self, H, metric, definitions, rtol=1e-10, atol=0., maxiter=1000, hbar=HBAR_EV_FS):
        self.H = canonical(H)
        self.metric = metric
        self.defs = [(k, [canonical(m) for m in ms]) for k, ms in definitions]
        if len(self.defs) != 3 or self.H.shape != metric.S.shape:
            raise ValueError("invalid engine operators")
        self.rtol, self.atol, self.maxiter, self.hbar = rtol, atol, maxiter, hbar
        self.h_calls = self.v_calls = 0

    def solve(self, B, rtol=None, atol=None, maxiter=None):
        return self.metric.solve(B, self.rtol if rtol is None else rtol, self.atol if atol is None else atol,
                                 self.maxiter if maxiter is None else maxiter)[0]

    def h_action(self, B):  # native.cpp:505
        self.h_calls += 1
        return self.solve(self.H @ B)

    def v_cart(self, axis, B, ctl=()):  # native.cpp:506-523
        kind, m = self.defs[axis]
        if kind == 0 and len(m) == 1:
            return m[0] @ B
        if kind == 1 and len(m) == 1:
            out = self.H @ self.solve(m[0] @ B, *ctl)
            rhs = m[0] @ self.solve(self.H @ B, *ctl)
            return 1j * (out - rhs) / self.hbar
        if kind == 2 and len(m) == 3:
            out = m[0] @ B
            left = m[1] @ self.solve(self.H @ B, *ctl)
            right = self.H @ self.solve(m[2] @ B, *ctl)
            return 1j * (out - left + right) / self.hbar
        raise ValueError("missing Cartesian velocity")

    def v_cov(self, direction, B, ctl=()):  # native.cpp:524-533
        if len(direction) != 3:
            raise ValueError("direction must have three components")
        self.v_calls += 1
        out = np.zeros_like(B)
        for a in range(3):
            if direction[a] != 0.:
                out += direction[a] * self.v_cart(a, B, ctl)
        return out

    def scaled(self, B, center, half):  # native.cpp:534-539
        if not half > 0:
            raise ValueError("spectral half-width must be positive")
        return (self.h_action(B) - center * B) / half

    def augmented(self, B, center, half, directions):  # native.cpp:540-554
        out = self.scaled(B, center, half)
        if not len(directions):
            return out
        if B.shape[1] % (len(directions) + 1):
            raise ValueError("invalid augmented block columns")
        nb = B.shape[1] // (len(directions) + 1)
        initial = B[:, :nb]
        for a, d in enumerate(directions):
            v = self.solve(self.v_cov(d, initial))
            out[:, (a + 1) * nb:(a + 2) * nb] += (-1j * self.hbar / half) * v
        return out

    def series(self, B, coeff, center, half, directions=()):  # native.cpp:555-573
        coeff = np.asarray(coeff, complex)
        if len(coeff) == 0:
            raise ValueError("empty Chebyshev coefficients")
        out = B * coeff[0]
        if len(coeff) == 1:
            return out
        prev, curr = B, self.augmented(B, center, half, directions)
        out = out + coeff[1] * curr
        for k in range(2, len(coeff)):
            nxt = 2. * self.augmented(curr, center, half, directions) - prev
            out = out + coeff[k] * nxt
            prev, curr = curr, nxt
        if not np.isfinite(out).all():
            raise RuntimeError("nonfinite Chebyshev propagation; check bounds and solves")
        return out

    def chain(self, B, length, center, half):  # native.cpp:574-589
        if length < 1:
            raise ValueError("Chebyshev chain must be nonempty")
        out = np.empty((length,) + B.shape, complex)
        out[0] = B
        if length == 1:
            return out
        out[1] = self.scaled(B, center, half)
        for k in range(2, length):
            out[k] = 2. * self.scaled(out[k - 1], center, half) - out[k - 2]
        return out

    def moments(self, B, length, center, half):  # native.cpp:590-609
        if length < 1:
            raise ValueError("moment count must be positive")
        out = np.empty((length, B.shape[1]))
        sb = self.metric.mul(B)
        out[0] = np.sum(sb.conj() * B, axis=0).real
        if length == 1:
            return out
        prev, curr = B, self.scaled(B, center, half)
        out[1] = np.sum(sb.conj() * curr, axis=0).real
        for k in range(2, length):
            nxt = 2. * self.scaled(curr, center, half) - prev
            out[k] = np.sum(sb.conj() * nxt, axis=0).real
            prev, curr = curr, nxt
        return out


# ---------------------------------------------------------------- host formulas
def scaling(bounds):
    """(center, half) of the full spectral window (src/kubo_msd/solvers/chebyshev.py:8-11)."""
    lo, hi = bounds
    return (lo + hi) / 2, (hi - lo) / 2


def bessel_coefficients(dt, bounds, tol, max_order, weighted_tail=False):
    """Bessel propagation coefficients (src/kubo_msd/solvers/chebyshev.py:17-30)."""
    c, a = scaling(bounds)
    z = a * dt / HBAR_EV_FS
    az = abs(z)
    if az == 0:
        return np.array([1 + 0j]), 0
    chosen = None
    for k in range(max(1, int(np.ceil(az))), max_order + 1):
        n = k + 1
        ratio = az / (2 * (n + 1))
        if ratio >= 1:
            continue
        logbound = n * np.log(az / 2) - gammaln(n + 1) + az * az / (4 * (n + 1))
        bound = 2 * np.exp(min(logbound, 700)) / (1 - ratio)
        if weighted_tail:
            bound *= 4 * (n + 1) ** 2 / (1 - ratio) ** 2
        if bound <= tol:
            chosen = k
            break
    if chosen is None:
        raise ValueError("propagation Bessel tail not converged before max order")
    m = np.arange(chosen + 1)
    b = jv(m, z) * (-1j) ** m
    b[1:] *= 2
    b *= np.exp(-1j * c * dt / HBAR_EV_FS)
    return b, chosen


def jackson(L):
    """Jackson damping g_m (src/kubo_msd/kernels/energy.py:12-18)."""
    m = np.arange(L)
    theta = np.pi / (L + 1)
    g = ((L + 1 - m) * np.cos(m * theta) + np.sin(m * theta) / np.tan(theta)) / (L + 1)
    g[0] = 1.
    return g


def reconstruction(E, bounds, L):
    """G[e, m] (src/kubo_msd/kernels/energy.py:20-24)."""
    c, a = scaling(bounds)
    x = (np.asarray(E, float) - c) / a
    g = jackson(L)
    g[1:] *= 2
    return np.cos(np.arccos(x)[:, None] * np.arange(L)) * g / (np.pi * a * np.sqrt(1 - x * x)[:, None])


def random_phases(n, seed, sample_ids):
    """Unit-modulus random phases (src/kubo_msd/metric/sampling.py:8-9)."""
    return np.column_stack([np.exp(2j * np.pi * np.random.Generator(np.random.PCG64(
        np.random.SeedSequence([int(seed), int(i)]))).random(n)) for i in sample_ids])


def projected_quadratic(engine, B, energies, bounds, n_moments):
    """(G mu)^T (src/kubo_msd/solvers/chebyshev.py:50-54)."""
    c, a = scaling(bounds)
    G = reconstruction(energies, bounds, n_moments)
    return (G @ engine.moments(B, n_moments, c, a)).T


def propagate(engine, states, dt_fs, bounds, segment_fs, tol, max_order):
    """Segmented Bessel propagation with S-norm drift check
    (src/kubo_msd/solvers/stepwise.py:8-18)."""
    B = np.asarray(states, complex)
    initial = np.sum(B.conj() * engine.metric.mul(B), axis=0).real
    nseg = max(1, int(np.ceil(abs(dt_fs) / segment_fs)))
    dt = dt_fs / nseg
    coeff, order = bessel_coefficients(dt, bounds, tol, max_order)
    c, a = scaling(bounds)
    for _ in range(nseg):
        B = engine.series(B, coeff, c, a)
    final = np.sum(B.conj() * engine.metric.mul(B), axis=0).real
    drift = float(np.max(np.abs(final - initial) / np.maximum(initial, np.finfo(float).tiny)))
    if drift > 1e-7:
        raise ValueError(f"S-norm propagation drift {drift:g}")
    return B, drift


def stepwise_samples(engine, samples, energies, times, bounds, n_moments, axes_vectors, segment_fs=1.,
                     tol=1e-12, max_order=4096):
    """Velocity-driven augmented commutator MSD (src/kubo_msd/solvers/stepwise.py:20-38):
    returns (dos (R, ne), msd (R, na, nt, ne))."""
    initial = np.asarray(samples, complex)
    nb = initial.shape[1]
    na, nt, ne = len(axes_vectors), len(times), len(energies)
    dos = projected_quadratic(engine, initial, energies, bounds, n_moments)
    total = np.concatenate([initial] + [np.zeros_like(initial) for _ in range(na)], axis=1)
    out = np.zeros((nb, na, nt, ne))
    c, a = scaling(bounds)
    norm0 = np.sum(initial.conj() * engine.metric.mul(initial), axis=0).real
    for j, t in enumerate(times):
        if j:
            span = t - times[j - 1]
            count = max(1, int(np.ceil(span / segment_fs)))
            coeff, _ = bessel_coefficients(span / count, bounds, tol, max_order, weighted_tail=True)
            for _ in range(count):
                total = engine.series(total, coeff, c, a, [list(v) for v in axes_vectors])
            norm = np.sum(total[:, :nb].conj() * engine.metric.mul(total[:, :nb]), axis=0).real
            drift = float(np.max(np.abs(norm - norm0) / np.maximum(norm0, np.finfo(float).tiny)))
            if drift > 1e-7:
                raise ValueError(f"stepwise base propagation S-norm drift {drift:g}")
        for ai in range(na):
            out[:, ai, j, :] = projected_quadratic(engine, total[:, (ai + 1) * nb:(ai + 2) * nb], energies,
                                                   bounds, n_moments)
    return dos, out


def engine_from_model(H, S, velocity=None, position=None, composite=None, blocks=(), rtol=1e-10, atol=0.,
                      maxiter=1000, policy="fixed", interval=32, gap_ratio=.1):
    """Metric + Engine built the way NativeMetric / NativeOperators build theirs
    (src/kubo_msd/backends/native.py:49-114)."""
    S = canonical(S)
    metric = Metric(S, S.diagonal().real.copy(), blocks, policy, interval, gap_ratio)
    velocity, position, composite = velocity or {}, position or {}, composite or {}
    defs = []
    for axis in "xyz":
        if axis in velocity:
            defs.append((0, [velocity[axis]]))
        elif axis in position:
            defs.append((1, [position[axis]]))
        elif axis in composite:
            defs.append((2, list(composite[axis])))
        else:
            defs.append((-1, []))
    return Engine(H, metric, defs, rtol, atol, maxiter)


def sampler_coefficients(S, tol=1e-10, max_order=4096):
    """Chebyshev fit of w^-1/2 over the normalized metric spectrum
    (src/kubo_msd/metric/sampling.py:11-32); bounds from Gershgorin when it
    certifies (src/kubo_msd/metric/bounds.py:7-11), else dense eigenvalues."""
    S = canonical(S)
    z = 1 / np.sqrt(S.diagonal().real)
    W = (sp.diags(z) @ S @ sp.diags(z)).tocsr()
    d = W.diagonal().real
    radii = np.asarray(abs(W).sum(axis=1)).ravel() - np.abs(d)
    lo, hi = float(np.min(d - radii)), float(np.max(d + radii))
    if not lo > 0:
        ev = np.linalg.eigvalsh(W.toarray())
        lo, hi = float(ev[0]) * (1 - 1e-10), float(ev[-1]) * (1 + 1e-10)
    center, half = (hi + lo) / 2, (hi - lo) / 2
    if half < 1e-14 * center:
        return np.array([1 / np.sqrt(center)]), center, half
    for order in (2 ** k for k in range(4, 20)):
        order = min(order, max_order)
        n = max(2 * order, 64)
        theta = np.pi * (np.arange(n) + .5) / n
        f = 1 / np.sqrt(center + half * np.cos(theta))
        coef = dct(f, type=2) / n
        coef[0] *= .5
        coef = coef[:order + 1]
        xx = np.cos(np.linspace(0, np.pi, max(4097, 8 * order + 1)))
        err = np.max(np.abs(np.polynomial.chebyshev.chebval(xx, coef) * np.sqrt(center + half * xx) - 1))
        if err < tol * .25:
            return coef, center, half
        if order >= max_order:
            break
    raise ValueError("metric inverse sqrt polynomial failed sampling tolerance")


def resolve_time_grid(tmax, dt):
    """Uniform grid 0..tmax with tmax appended (src/kubo_msd/config.py:19-24)."""
    t = np.arange(int(np.floor(tmax / dt)) + 1, dtype=float) * dt
    if t[-1] < tmax and not np.isclose(t[-1], tmax, rtol=0, atol=8 * np.spacing(max(tmax, dt))):
        t = np.append(t, tmax)
    else:
        t[-1] = tmax
    return t


def spectral_samples(engine, samples, energies, times_out, bounds, n_moments, axes_vectors, integration_dt,
                     segment_fs=1., tol=1e-12, max_order=4096, include_vac=True):
    """Segmented trace-first Chebyshev product VAC
    (src/kubo_msd/solvers/spectral.py:15-53): returns (dos, outputs)."""
    x = np.asarray(samples, complex)
    n, nb = x.shape
    na, ne, nt, L = len(axes_vectors), len(energies), len(times_out), n_moments
    dos = projected_quadratic(engine, x, energies, bounds, n_moments)
    keys = ("msd_A2/vac_integral", "diffusion_A2_per_fs/vac_integral", "vac_A2_per_fs2/vac_integral")
    out = {k: np.zeros((nb, na, nt, ne)) for k in keys}
    times = np.unique(np.r_[resolve_time_grid(times_out[-1], integration_dt), times_out])
    index = {float(t): j for j, t in enumerate(times_out)}
    G = reconstruction(energies, bounds, L)
    c, a = scaling(bounds)
    c_anchor = x
    v_anchor = [engine.solve(engine.v_cov(list(d), x)) for d in axes_vectors]
    anchor, next_anchor, tables = 0., -1., None
    M = np.zeros((nb, na, ne))
    D = np.zeros_like(M)
    previous, prev_t = None, 0.
    for t in times:
        if tables is None or t > next_anchor + 1e-14:
            new_anchor = 0. if tables is None else float(prev_t)
            if new_anchor > anchor:
                both, _ = propagate(engine, np.concatenate([c_anchor] + v_anchor, axis=1), new_anchor - anchor,
                                    bounds, segment_fs, tol, max_order)
                c_anchor = both[:, :nb]
                v_anchor = [both[:, (i + 1) * nb:(i + 2) * nb] for i in range(na)]
            anchor = new_anchor
            next_anchor = min(max(anchor + segment_fs, float(t)), float(times[-1]))
            coeff, K = bessel_coefficients(next_anchor - anchor, bounds, tol, max_order)
            left = engine.chain(c_anchor, L + K, c, a)
            tables = []
            for ai, d in enumerate(axes_vectors):
                right = engine.chain(v_anchor[ai], K + 1, c, a)
                cov = engine.v_cov(list(d), right.transpose(1, 0, 2).reshape(n, -1)).reshape(n, K + 1, nb)
                tables.append(np.einsum("jnb,knb->bjk", left.conj(), cov.transpose(1, 0, 2)))
        b, Kt = bessel_coefficients(float(t - anchor), bounds, tol, max_order)
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
        if float(t) in index:
            j = index[float(t)]
            out["msd_A2/vac_integral"][:, :, j, :] = M
            out["diffusion_A2_per_fs/vac_integral"][:, :, j, :] = D
            out["vac_A2_per_fs2/vac_integral"][:, :, j, :] = vac
        previous, prev_t = vac, t
    if not include_vac:
        out.pop("vac_A2_per_fs2/vac_integral")
    return dos, out
