"""Parity on the stated configurations at their full lattice sizes.

* Config 1 in full: 64x64 square lattice, R=8, M=512, 201 energies, stepwise
  MSD over 0-50 fs at dt = 1 fs; FP64 against the reference's own run
  (1e-10 DOS, 1e-9 MSD), the mixed form within its stated tolerances.
* Config 3 lattice at full size (4,194,304-site honeycomb): FP64 moments of
  R=8 phase vectors, M=16, against the reference engine's (1e-10), with both
  moment methods; the mixed form within its stated moment tolerance, order by
  order.
* Config 3 precision form: the mixed form against FP64 on identical phases,
  M=4096, R=8, DOS and MSD(E, t) on config 1's time grid, with the errors
  resolved per moment order, per energy and per (energy, time) point.
* Config 2 model at full size (diamond sp3, 32,000 orbitals, kappa(S) = 50,
  block-Jacobi PCG): S^-1/2 sampling, moments, composite velocity and a short
  stepwise MSD against the reference (1e-10 / 1e-9), with the solves
  tightened to rtol 1e-12 as the golden run was.

The golden arrays come from the reference itself (tests/golden/make_golden.py).
"""
import numpy as np
import pytest
import scipy.linalg as la
import scipy.sparse as sp

from tests.helpers import assert_rel, golden

pytestmark = pytest.mark.gpu

# Mixed form (complex64 vectors / SpMM, FP64 accumulation) against FP64.
MIXED_MOMENTS_TOL = 5e-5     # norm-wise over a moment array
MIXED_MSD_TOL = 1e-4         # norm-wise over an MSD array (the precision form's target)
# Resolved errors of the precision form (C3, M=4096): per moment order against
# that order's own scale; per energy in the band (DOS above 1e-3 of its
# maximum); per (energy, time) point above 1e-3 of that time's maximum.
PF_MOMENT_PER_ORDER_TOL = 1e-3
PF_DOS_PER_ENERGY_TOL = 1e-4
PF_MSD_PER_POINT_TOL = 1e-3
PF_MSD_NORMWISE_TOL = 1e-4


def _eng(m, precision="fp64", doubling=False, **kw):
    from tests.gpu_util import engine
    metric, eng, ops = engine(m.H, m.S, velocity=m.velocity, precision=precision, **kw)
    eng.doubling = doubling
    return metric, eng, ops


# ------------------------------------------------------------------ config 1
@pytest.fixture(scope="module")
def c1_full(cuda):
    from kubomsd_b200 import kpm, lattices
    from kubomsd_b200.config import RunConfig
    m = lattices.square_lattice(64)
    B = kpm.random_phases(m.n, 20261019, range(8))

    def cfg(**kw):
        return RunConfig(energy_eV=np.linspace(-11, 11, 201), time_fs=np.arange(51.), spectral_bounds=(-11.2, 11.2),
                         n_moments=512, axes=("x",), include_vac=False, stochastic_method="stepwise", **kw)
    return m, B, cfg, golden("c1_square64_full")


def test_c1_full_time_grid_fp64(c1_full):
    from kubomsd_b200 import stochastic
    m, B, cfg, d = c1_full
    assert np.array_equal(d["time_fs"], np.arange(51.))
    _, _, ops = _eng(m)
    dos, nums, _ = stochastic.stepwise_samples(ops, cfg(), B)
    assert_rel(dos, d["dos"], 1e-10, "C1 dos, 0-50 fs")
    assert_rel(nums["msd_A2/commutator"], d["msd"], 1e-9, "C1 msd, 0-50 fs")


@pytest.mark.parametrize("doubling", [False, True])
def test_c1_full_time_grid_mixed(c1_full, doubling):
    from kubomsd_b200 import accuracy, stochastic
    m, B, cfg, d = c1_full
    _, _, ops = _eng(m, "mixed", doubling)
    dos, nums, _ = stochastic.stepwise_samples(ops, cfg(precision="mixed", moment_doubling=doubling), B)
    e1 = assert_rel(dos, d["dos"], MIXED_MOMENTS_TOL, "C1 dos mixed, 0-50 fs")
    e2 = assert_rel(nums["msd_A2/commutator"], d["msd"], MIXED_MSD_TOL, "C1 msd mixed, 0-50 fs")
    r = accuracy.stepwise_errors(dos, nums["msd_A2/commutator"], d["dos"], d["msd"], np.arange(51.))
    print(f"C1 mixed (doubling={doubling}): dos {e1:.2e} msd {e2:.2e} resolved {r}")


# ------------------------------------------------------------------ config 3
@pytest.fixture(scope="module")
def c3(cuda):
    from kubomsd_b200 import kpm, lattices
    torch = cuda
    m = lattices.honeycomb(2048, 1024, with_velocity=False)
    B = torch.from_numpy(kpm.random_phases(m.n, 20261019, range(8))).cuda()
    return m, B, golden("c3_honeycomb_fp64")


@pytest.mark.parametrize("doubling", [False, True])
def test_c3_full_size_moments_fp64(c3, doubling):
    m, B, d = c3
    _, eng, _ = _eng(m, "fp64", doubling)
    mu = eng.moments(B, 16, float(d["center"]), float(d["half"])).cpu().numpy()
    assert_rel(mu, d["moments"], 1e-10, f"C3 moments fp64 doubling={doubling}")
    per_order = np.max(np.abs(mu - d["moments"]), axis=1) / np.max(np.abs(d["moments"]), axis=1)
    assert np.all(per_order <= 1e-9), per_order


@pytest.mark.parametrize("doubling", [False, True])
def test_c3_full_size_moments_mixed(c3, doubling):
    from kubomsd_b200 import accuracy
    m, B, d = c3
    _, eng, _ = _eng(m, "mixed", doubling)
    mu = eng.moments(B, 16, float(d["center"]), float(d["half"])).cpu().numpy()
    assert_rel(mu, d["moments"], MIXED_MOMENTS_TOL, f"C3 moments mixed doubling={doubling}")
    r = accuracy.moment_errors(mu, d["moments"])
    assert r["max_per_order"] <= PF_MOMENT_PER_ORDER_TOL, r
    print(f"C3 mixed moments vs reference FP64: {r['max_per_order']:.2e} per order, "
          f"{r['max_over_mu0']:.2e} of mu0")


def test_c3_precision_form_resolved_errors(c3):
    """The precision-form configuration: M=4096, DOS and MSD(E, t) on config
    1's time grid (0-50 fs, dt = 1 fs), mixed against FP64 on the same R=8
    phase vectors; window (-9.2, 9.2) eV, 201 energies on [-9, 9] eV."""
    from kubomsd_b200 import accuracy, kpm, lattices
    from kubomsd_b200.config import RunConfig
    m = lattices.honeycomb(2048, 1024, with_velocity=True)
    B = kpm.random_phases(m.n, 20261019, range(8))
    cfg = RunConfig(energy_eV=np.linspace(-9, 9, 201), time_fs=np.arange(51.), spectral_bounds=(-9.2, 9.2),
                    n_moments=4096, axes=("x",), include_vac=False, stochastic_method="stepwise",
                    moment_doubling=True)
    rep = accuracy.mixed_vs_fp64(m, B, cfg)
    mo, st = rep["moments"], rep["stepwise"]
    print("C3 precision form, mixed vs FP64:", {k: v for k, v in rep.items() if not k.startswith("_")})
    assert mo["max_per_order"] <= PF_MOMENT_PER_ORDER_TOL, mo
    assert st["dos_max_rel_per_energy"] <= PF_DOS_PER_ENERGY_TOL, st
    assert st["msd_max_rel_per_point"] <= PF_MSD_PER_POINT_TOL, st
    assert st["msd_normwise"] <= PF_MSD_NORMWISE_TOL, st


# ------------------------------------------------------------------ config 2
@pytest.fixture(scope="module")
def c2_full(cuda):
    from kubomsd_b200 import kpm, lattices
    from tests.gpu_util import engine
    m = lattices.diamond_sp3(cells=10)
    S = sp.csr_matrix(m.S)
    blocks = [(a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)) for a, b in m.atom_slices]
    metric, eng, ops = engine(m.H, m.S, composite=m.composite, blocks=blocks, rtol=1e-12)
    xi = kpm.random_phases(m.n, 20261019, range(4))
    return m, metric, eng, ops, xi, golden("c2_diamond10")


def _compare_compact(full, d, name, tol):
    """An (N, b) array against the fixture's every-k-th row, column sums and
    column norms (the fixture stores those instead of the whole array)."""
    full = np.asarray(full)
    k = int(d["row_stride"])
    assert_rel(full[::k], d[name + "_rows"], tol, name + " rows")
    assert_rel(full.sum(axis=0), d[name + "_colsum"], tol, name + " column sums")
    assert_rel(np.linalg.norm(full, axis=0), d[name + "_colnorm"], tol, name + " column norms")


def test_c2_full_size_sampling_moments_velocity(c2_full):
    m, metric, eng, ops, xi, d = c2_full
    assert m.n == 32000
    _compare_compact(metric.sample(xi, d["sample_coeff"], float(d["sample_center"]), float(d["sample_half"])), d,
                     "sample", 1e-11)
    assert_rel(eng.moments(xi, 8, 0., 40.), d["moments"], 1e-10, "C2 moments")
    _compare_compact(eng.v_cov([1., 0., 0.], xi[:, :2]), d, "v_cov_x", 1e-10)


def test_c2_full_size_stepwise(c2_full):
    from kubomsd_b200 import stochastic
    from kubomsd_b200.config import RunConfig
    m, metric, eng, ops, xi, d = c2_full
    cfg = RunConfig(energy_eV=np.linspace(-30, 30, 13), time_fs=[0., .5, 1.], spectral_bounds=(-40., 40.),
                    n_moments=16, axes=("x", "y", "z"), include_vac=False, stochastic_method="stepwise",
                    metric_rtol=1e-12, preconditioner="block-jacobi", segment_fs=.5)
    dos, nums, _ = stochastic.stepwise_samples(ops, cfg, xi[:, :2])
    assert_rel(dos, d["dos"], 1e-10, "C2 dos")
    assert_rel(nums["msd_A2/commutator"], d["msd"], 1e-9, "C2 msd")
