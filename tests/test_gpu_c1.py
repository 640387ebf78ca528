"""Config-1 workload (64x64 square lattice, R=8 phases, M=512, Jackson,
201 energies): device moments and stepwise MSD vs the reference's outputs,
FP64 (1e-10) and the mixed form (stated tolerances)."""
import numpy as np
import pytest

from tests.helpers import assert_rel, golden

pytestmark = pytest.mark.gpu
BOUNDS = (-11.2, 11.2)
# Mixed form (complex64 vectors / SpMM, FP64 accumulation): norm-wise relative
# error bounds against the FP64 reference.
MIXED_MOMENTS_TOL = 5e-5
MIXED_MSD_TOL = 1e-4


@pytest.fixture(scope="module")
def c1(cuda):
    from kubomsd_b200 import kpm, lattices
    m = lattices.square_lattice(64)
    B = kpm.random_phases(m.n, 20261019, range(8))
    return m, B, golden("c1_square64")


def _ops(m, precision, doubling=False):
    from tests.gpu_util import engine
    metric, eng, ops = engine(m.H, m.S, velocity=m.velocity, precision=precision)
    eng.doubling = doubling
    return eng, ops


@pytest.mark.parametrize("doubling", [False, True])
def test_c1_moments_fp64(c1, doubling):
    m, B, d = c1
    eng, _ = _ops(m, "fp64", doubling)
    assert_rel(eng.moments(B, 512, 0., 11.2), d["moments"], 1e-10, "C1 moments fp64")


@pytest.mark.parametrize("doubling", [False, True])
def test_c1_moments_mixed(c1, doubling):
    m, B, d = c1
    eng, _ = _ops(m, "mixed", doubling)
    err = assert_rel(eng.moments(B, 512, 0., 11.2), d["moments"], MIXED_MOMENTS_TOL, "C1 moments mixed")
    print(f"mixed moments relative error {err:.2e}")


def _cfg(**kw):
    from kubomsd_b200.config import RunConfig
    return RunConfig(energy_eV=np.linspace(-11, 11, 201), time_fs=[0., 1., 2., 3.], spectral_bounds=BOUNDS,
                     n_moments=512, axes=("x",), include_vac=False, stochastic_method="stepwise", **kw)


def test_c1_stepwise_fp64(c1):
    from kubomsd_b200 import stochastic
    m, B, d = c1
    eng, ops = _ops(m, "fp64")
    dos, nums, diag = stochastic.stepwise_samples(ops, _cfg(), B)
    assert_rel(dos, d["dos"], 1e-10, "C1 dos")
    assert_rel(nums["msd_A2/commutator"], d["msd"], 1e-9, "C1 msd")
    assert diag["max_propagation_order"] > 0


def test_c1_stepwise_mixed_within_stated_tolerance(c1):
    from kubomsd_b200 import stochastic
    m, B, d = c1
    eng, ops = _ops(m, "mixed")
    dos, nums, _ = stochastic.stepwise_samples(ops, _cfg(precision="mixed"), B)
    e1 = assert_rel(dos, d["dos"], MIXED_MOMENTS_TOL, "C1 dos mixed")
    e2 = assert_rel(nums["msd_A2/commutator"], d["msd"], MIXED_MSD_TOL, "C1 msd mixed")
    print(f"mixed dos relerr {e1:.2e} msd relerr {e2:.2e}")
