"""Error of the mixed form against the plain FP64 path on identical inputs.

The precision form (complex64 vectors and SpMM, FP64 moment accumulation) is
held to stated tolerances against FP64.  A norm-wise error over a whole
moment array is dominated by mu_0 = N and says little about the high orders
where FP32 rounding accumulates, so the comparison here is resolved:

* moments: for each order k, max_j |d mu_kj| / max_j |mu_kj| (the order's own
  scale), and the same normalised by mu_0 = N;
* DOS: the sample-averaged DOS per energy, relative to its own value, over
  the energies where the DOS is above 1e-3 of its maximum (the band);
* MSD(E, t): the sample-averaged MSD numerator per (energy, time), relative
  to its own value, over the points above 1e-3 of that time's maximum;
* D(E, t) = 1/2 dMSD/dt (kpm.msd_gradient, as the reference's
  observables/diffusion.py:4-6) the same way.

Both runs go through the product path (B200Operators and the stepwise driver
of kubomsd_b200.stochastic) on the same phases, bounds and grids.
"""
from __future__ import annotations

import time

import numpy as np

from . import kpm


def _resolved(test, ref, axis_scale, floor=1e-3):
    """max relative error over the points where |ref| >= floor x its scale along axis_scale."""
    test, ref = np.asarray(test), np.asarray(ref)
    scale = np.max(np.abs(ref), axis=axis_scale, keepdims=True)
    mask = np.abs(ref) >= floor * scale
    rel = np.abs(test - ref) / np.where(mask, np.abs(ref), 1.)
    return float(np.max(np.where(mask, rel, 0.))), float(np.mean(mask))


def moment_errors(mu_test, mu_ref):
    """Per-order errors of (M, R) moment arrays."""
    mu_test, mu_ref = np.asarray(mu_test), np.asarray(mu_ref)
    d = np.max(np.abs(mu_test - mu_ref), axis=1)
    per_order = d / np.maximum(np.max(np.abs(mu_ref), axis=1), np.finfo(float).tiny)
    n = float(np.max(np.abs(mu_ref[0])))
    return {"max_per_order": float(np.max(per_order)), "median_per_order": float(np.median(per_order)),
            "order_of_max": int(np.argmax(per_order)), "max_over_mu0": float(np.max(d) / n),
            "per_order": per_order}


def stepwise_errors(dos_t, msd_t, dos_r, msd_r, time_fs):
    """Per-energy DOS and per-(energy, time) MSD and D errors of stepwise outputs
    (dos: (R, ne); msd: (R, na, nt, ne))."""
    dos_t, dos_r = np.mean(dos_t, axis=0), np.mean(dos_r, axis=0)
    msd_t, msd_r = np.mean(msd_t, axis=0), np.mean(msd_r, axis=0)
    e_dos, f_dos = _resolved(dos_t, dos_r, 0)
    e_msd, f_msd = _resolved(msd_t[:, 1:], msd_r[:, 1:], -1)
    D_t = kpm.msd_gradient(np.asarray(time_fs), msd_t, axis=1) / 2.
    D_r = kpm.msd_gradient(np.asarray(time_fs), msd_r, axis=1) / 2.
    e_D, f_D = _resolved(D_t[:, 1:], D_r[:, 1:], -1)
    return {"dos_max_rel_per_energy": e_dos, "dos_band_fraction": f_dos,
            "msd_max_rel_per_point": e_msd, "msd_points_fraction": f_msd,
            "diffusion_max_rel_per_point": e_D, "diffusion_points_fraction": f_D,
            "dos_normwise": float(np.max(np.abs(dos_t - dos_r)) / np.max(np.abs(dos_r))),
            "msd_normwise": float(np.max(np.abs(msd_t - msd_r)) / np.max(np.abs(msd_r)))}


def mixed_vs_fp64(model, B, cfg, with_msd=True):
    """Runs the DOS moments and (with_msd) the stepwise MSD of `model` on the
    phase block B in FP64 and in the mixed form; returns the error report and
    the seconds each took."""
    import torch
    from dataclasses import replace
    from .operators import build_operators
    from . import stochastic
    out, res = {}, {}
    Bd = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    c, a = kpm.scaling(cfg)
    for prec in ("fp64", "mixed"):
        pc = replace(cfg, precision=prec)
        ops = build_operators(model, pc)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mu = ops.native.moments(Bd, cfg.n_moments, c, a)
        mu = mu.cpu().numpy() if hasattr(mu, "cpu") else np.asarray(mu)
        t_mu = time.perf_counter() - t0
        entry = {"moments": mu, "moments_s": t_mu}
        if with_msd:
            t0 = time.perf_counter()
            dos, nums, _ = stochastic.stepwise_samples(ops, pc, Bd)
            entry.update(dos=dos, msd=nums["msd_A2/commutator"], stepwise_s=time.perf_counter() - t0)
        res[prec] = entry
        del ops
        torch.cuda.empty_cache()
    m = moment_errors(res["mixed"]["moments"], res["fp64"]["moments"])
    out["moments"] = {k: v for k, v in m.items() if k != "per_order"}
    out["seconds"] = {p: {k: v for k, v in e.items() if k.endswith("_s")} for p, e in res.items()}
    if with_msd:
        out["stepwise"] = stepwise_errors(res["mixed"]["dos"], res["mixed"]["msd"], res["fp64"]["dos"],
                                          res["fp64"]["msd"], cfg.time_fs)
    out["_per_order"] = m["per_order"]
    return out
