"""Size-independent properties on a honeycomb lattice beyond the oracle's
reach: trace identity, moment-method equivalence, linearity, chain/moment
consistency, propagation round trips, mixed vs FP64 error."""
import numpy as np
import pytest

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu
BOUNDS = (-9.2, 9.2)


@pytest.fixture(scope="module")
def lattice(cuda):
    from kubomsd_b200 import kpm, lattices
    m = lattices.honeycomb(256, 128, seed=5)
    B = kpm.random_phases(m.n, 77, range(16))
    return m, B


def _eng(m, precision="fp64"):
    from tests.gpu_util import engine
    return engine(m.H, m.S, velocity=m.velocity, precision=precision)


def test_trace_identity_and_moment_methods(lattice):
    m, B = lattice
    _, eng, _ = _eng(m)
    direct = eng.moments(B, 256, 0., 9.2, doubling=False)
    np.testing.assert_allclose(direct[0], m.n, rtol=1e-13)  # mu_0 = sum |xi|^2 = N for unit phases
    doubled = eng.moments(B, 256, 0., 9.2, doubling=True)
    assert_rel(doubled, direct, 1e-11, "doubling vs direct")
    assert_rel(eng.moments(2 * B, 256, 0., 9.2), 4 * direct, 1e-12, "quadratic scaling")


def test_chain_consistent_with_moments(lattice):
    m, B = lattice
    _, eng, _ = _eng(m)
    ch = eng.chain(B[:, :4], 20, 0., 9.2)
    mu = eng.moments(B[:, :4], 20, 0., 9.2)
    proj = np.einsum("nb,knb->kb", B[:, :4].conj(), ch).real
    assert_rel(proj, mu, 1e-12, "chain projections")
    np.testing.assert_allclose(eng.h_action(B[:, :4]), eng.H.matmul(B[:, :4]), rtol=0, atol=1e-13)


def test_propagation_round_trip_and_norm(lattice):
    from kubomsd_b200 import stochastic
    from kubomsd_b200.config import RunConfig
    m, B = lattice
    _, eng, ops = _eng(m)
    cfg = RunConfig(energy_eV=[0.], time_fs=[0., 1.], spectral_bounds=BOUNDS, axes=("x",), include_vac=False)
    fwd, d1 = stochastic.propagate(B[:, :8], 1., ops, cfg)
    back, d2 = stochastic.propagate(fwd, -1., ops, cfg)
    assert_rel(back, B[:, :8], 1e-11, "round trip")
    assert d1["relative_S_norm_drift"] < 1e-12


def test_mixed_moments_error_vs_fp64(lattice):
    m, B = lattice
    _, e64, _ = _eng(m)
    _, e32, _ = _eng(m, "mixed")
    ref = e64.moments(B, 1024, 0., 9.2)
    for doubling in (False, True):
        # the stated moment tolerance of the mixed form (5e-5, norm-wise)
        err = assert_rel(e32.moments(B, 1024, 0., 9.2, doubling=doubling), ref, 5e-5, "mixed moments")
        print(f"M=1024 mixed (doubling={doubling}) moments relerr {err:.2e}")


def test_device_lanczos_bounds_match_arpack(lattice):
    from kubomsd_b200 import kpm
    from kubomsd_b200.config import RunConfig
    from kubomsd_b200.operators import build_operators
    m, _ = lattice
    cfg = RunConfig(energy_eV=[0.], time_fs=[0.], axes=("x",), include_vac=False)
    ops = build_operators(m, cfg)
    host = kpm.estimate_spectral_bounds(ops.host_H, ops.host_S, ops.metric.s_lower, cfg)
    dev = kpm.lanczos_spectral_bounds(ops, cfg)
    lo, hi = host["extrema"]
    # 160 Lanczos steps: extrema within ~1e-5 of ARPACK, far inside the 1 % margin
    np.testing.assert_allclose(dev["extrema"], host["extrema"], rtol=1e-4)
    assert dev["bounds"][0] < lo and dev["bounds"][1] > hi
