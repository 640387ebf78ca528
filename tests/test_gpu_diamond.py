"""Nonorthogonal sp3 model (diamond, 4x4 atom blocks, kappa(S) = 50,
block-Jacobi PCG, composite velocity on x, y, z): the general-metric device
path vs the reference."""
import numpy as np
import pytest
import scipy.linalg as la
import scipy.sparse as sp

from tests.helpers import assert_rel, golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def diamond(cuda):
    from kubomsd_b200 import lattices
    from tests.gpu_util import engine
    m = lattices.diamond_sp3(cells=2)
    S = sp.csr_matrix(m.S)
    blocks = [(a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)) for a, b in m.atom_slices]
    metric, eng, ops = engine(m.H, m.S, composite=m.composite, blocks=blocks, rtol=1e-12)
    return m, metric, eng, ops, golden("diamond2")


def test_diamond_sampling_moments_velocity(diamond):
    m, metric, eng, ops, d = diamond
    c, a = 0., 40.
    assert_rel(metric.sample(d["xi"], d["sample_coeff"], float(d["sample_center"]), float(d["sample_half"])),
               d["sample"], 1e-11, "S^-1/2 sampling")
    assert_rel(eng.moments(d["B"], 32, c, a), d["moments"], 1e-10, "moments")
    assert_rel(eng.v_cov([0., 1., 0.], d["B"]), d["v_cov_y"], 1e-10, "composite v_cov")


def test_diamond_stepwise(diamond):
    from kubomsd_b200 import stochastic
    from kubomsd_b200.config import RunConfig
    m, metric, eng, ops, d = diamond
    cfg = RunConfig(energy_eV=np.linspace(-8, 6, 8), time_fs=[0., .5, 1.], spectral_bounds=(-40., 40.),
                    n_moments=32, axes=("x", "y", "z"), include_vac=False, stochastic_method="stepwise",
                    metric_rtol=1e-12, preconditioner="block-jacobi", segment_fs=.5)
    dos, nums, _ = stochastic.stepwise_samples(ops, cfg, d["B"])
    assert_rel(dos, d["dos"], 1e-10, "dos")
    assert_rel(nums["msd_A2/commutator"], d["msd"], 1e-9, "msd")
