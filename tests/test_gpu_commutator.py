"""Position-commutator velocity applied inside the Chebyshev step.

A position operator given by site coordinates, X = diag(x), on an
orthogonal basis makes the reference's kind-1 velocity
i (H S^-1 X B - X S^-1 H B) / hbar (cpp/native.cpp:506-523) equal to
i [H, X] B / hbar, whose row i is (i / hbar) sum_j H_ij (x_j - x_i) B_j.
The engine applies it from H's rows inside the augmented series step
instead of two SpMMs, two solves and a linear combination per step.  It is
checked against the oracle's kind-1 engine (FP64, 1e-10; mixed, the stated
tolerance), and the step count shows the fused path ran.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu


def _model(L=16):
    from kubomsd_b200 import lattices
    m = lattices.square_lattice(L, seed=21)
    x = (np.arange(m.n) // L).astype(float) * 1.0   # site coordinate along x (angstrom)
    y = (np.arange(m.n) % L).astype(float) * 1.0
    return m, {"x": sp.diags(x).tocsr(), "y": sp.diags(y).tocsr()}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_commutator_series_matches_oracle(cuda, precision):
    from kubomsd_b200 import _abi, kpm
    from kubomsd_b200.config import RunConfig
    from oracle import kpm_oracle as O
    from tests.gpu_util import engine
    m, pos = _model()
    B = kpm.random_phases(m.n, 3, range(4))
    aug = np.concatenate([B, np.zeros_like(B), np.zeros_like(B)], axis=1)
    cfg = RunConfig(energy_eV=[0.], time_fs=[0., 1.], spectral_bounds=(-11.5, 11.5), axes=("x", "y"))
    coeff, _ = kpm.bessel_coefficients(.5, cfg, weighted_tail=True)
    c, a = kpm.scaling(cfg)
    dirs = [[1., 0., 0.], [.6, .8, 0.]]
    _, eng, _ = engine(m.H, m.S, position=pos, precision=precision)
    lib = _abi.load()
    l0 = lib.kmsd_kernel_launches()
    got = eng.series(aug, coeff, c, a, dirs)
    launches = lib.kmsd_kernel_launches() - l0
    want = O.engine_from_model(m.H, m.S, position=pos).series(aug, coeff, c, a, dirs)
    assert_rel(got, want, 1e-10 if precision == "fp64" else 5e-5, f"fused commutator series {precision}")
    # one step kernel per Chebyshev term, plus a few copies / conversions
    assert launches <= len(coeff) + 4, launches


def test_fused_commutator_stepwise_matches_oracle(cuda):
    from kubomsd_b200 import kpm, stochastic
    from kubomsd_b200.config import RunConfig
    from oracle import kpm_oracle as O
    from tests.gpu_util import engine
    m, pos = _model()
    B = kpm.random_phases(m.n, 5, range(4))
    cfg = RunConfig(energy_eV=np.linspace(-9, 9, 13), time_fs=[0., 1., 2.], spectral_bounds=(-11.5, 11.5),
                    n_moments=64, axes=("x",), include_vac=False, stochastic_method="stepwise")
    _, eng, ops = engine(m.H, m.S, position=pos)
    dos, nums, _ = stochastic.stepwise_samples(ops, cfg, B)
    wdos, wmsd = O.stepwise_samples(O.engine_from_model(m.H, m.S, position=pos), B, cfg.energy_eV, cfg.time_fs,
                                    cfg.spectral_bounds, cfg.n_moments, [[1., 0., 0.]], segment_fs=cfg.segment_fs)
    assert_rel(dos, wdos, 1e-10, "dos")
    assert_rel(nums["msd_A2/commutator"], wmsd, 1e-9, "msd")


def _honeycomb(Lx=24, Ly=12):
    from kubomsd_b200 import lattices
    m = lattices.honeycomb(Lx, Ly, W=1., seed=5)
    acc = 1.42
    site = np.arange(m.n)
    cx, cy = np.divmod(site // 2, Ly)
    x = acc * 1.5 * (cx + cy) + acc * (site % 2)   # site coordinates along x (no minimum image)
    return m, {"x": sp.diags(x).tocsr()}


@pytest.mark.parametrize("form", ["velocity", "position"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ell_aligned_velocity_series_matches_oracle(cuda, form, precision):
    """On a lattice with a 4-wide ELL form the inline velocity (explicit V, or
    i [H, X] / hbar from coordinates) is applied from H's ELL row with values
    aligned to its columns; the augmented series matches the oracle."""
    from kubomsd_b200 import kpm
    from kubomsd_b200.config import RunConfig
    from oracle import kpm_oracle as O
    from tests.gpu_util import engine
    m, pos = _honeycomb()
    kw = {"velocity": m.velocity} if form == "velocity" else {"position": pos}
    B = kpm.random_phases(m.n, 9, range(4))
    aug = np.concatenate([B, np.zeros_like(B)], axis=1)
    cfg = RunConfig(energy_eV=[0.], time_fs=[0., 1.], spectral_bounds=(-9.6, 9.6), axes=("x",))
    coeff, _ = kpm.bessel_coefficients(.5, cfg, weighted_tail=True)
    c, a = kpm.scaling(cfg)
    _, eng, _ = engine(m.H, m.S, precision=precision, **kw)
    got = eng.series(aug, coeff, c, a, [[1., 0., 0.]])
    want = O.engine_from_model(m.H, m.S, **kw).series(aug, coeff, c, a, [[1., 0., 0.]])
    assert_rel(got, want, 1e-10 if precision == "fp64" else 5e-5, f"aligned {form} series {precision}")


@pytest.mark.parametrize("R", [16, 32, 64])
@pytest.mark.parametrize("form", ["velocity", "position"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ell_aligned_series_wide_blocks(cuda, R, form, precision):
    """[psi | phi] blocks of R columns each make row groups of 16 to 128 lanes
    (one to four warps); the psi lanes' velocity products reach the phi lanes
    through shared memory under a warp or named barrier.  The position form
    takes two directions (x and a diagonal), so two velocity matrices feed
    each of its two phi blocks."""
    from kubomsd_b200 import kpm
    from kubomsd_b200.config import RunConfig
    from oracle import kpm_oracle as O
    from tests.gpu_util import engine
    m, pos = _honeycomb()
    site = np.arange(m.n)
    cx, cy = np.divmod(site // 2, 12)
    pos["y"] = sp.diags(1.42 * .866 * (cy - cx) + .71 * (site % 2)).tocsr()
    if form == "velocity":
        kw, dirs, axes = {"velocity": m.velocity}, [[1., 0., 0.]], ("x",)
    else:
        kw, dirs, axes = {"position": pos}, [[1., 0., 0.], [.6, .8, 0.]], ("x", "y")
    B = kpm.random_phases(m.n, 11, range(R))
    aug = np.concatenate([B] + [np.zeros_like(B)] * len(dirs), axis=1)
    cfg = RunConfig(energy_eV=[0.], time_fs=[0., 1.], spectral_bounds=(-9.6, 9.6), axes=axes)
    coeff, _ = kpm.bessel_coefficients(.5, cfg, weighted_tail=True)
    c, a = kpm.scaling(cfg)
    _, eng, _ = engine(m.H, m.S, precision=precision, **kw)
    got = eng.series(aug, coeff, c, a, dirs)
    want = O.engine_from_model(m.H, m.S, **kw).series(aug, coeff, c, a, dirs)
    assert_rel(got, want, 1e-10 if precision == "fp64" else 5e-5, f"aligned {form} series R={R} {precision}")
