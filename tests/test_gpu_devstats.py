"""Device statistics against the host restatement of the reference's.

The paired block bootstrap on the device (kmsd_bootstrap_ratio) against
kpm.estimate_ratio (src/kubo_msd/observables/statistics.py:5-23) on the same
block sums, including blocks of unequal counts, a zero denominator (NaN) and
broadcast counts; the device energy projection against G @ mu; and the
spectral correlation tables of the ring contraction against a stored chain.
"""
import numpy as np
import pytest

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nblocks", [1, 2, 5, 9])
def test_device_bootstrap_matches_host(cuda, nblocks):
    from kubomsd_b200 import devstats, kpm
    torch = cuda
    rng = np.random.default_rng(nblocks)
    A = rng.normal(size=(nblocks, 2, 3, 7))
    D = rng.uniform(.5, 2., size=(nblocks, 7))
    D[:, 3] = 0.  # a zero denominator gives NaN in both
    counts = rng.integers(1, 5, nblocks)
    v_host, se_host, _ = kpm.estimate_ratio(A, D, counts)
    v, se, status = devstats.estimate_ratio(torch.from_numpy(A).cuda(), torch.from_numpy(D).cuda(), counts)
    v = v.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(v), np.isnan(v_host))
    ok = ~np.isnan(v_host)
    np.testing.assert_allclose(v[ok], v_host[ok], rtol=1e-13)
    if nblocks < 2:
        assert se is None and se_host is None
        return
    se = se.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(se), np.isnan(se_host))
    ok = ~np.isnan(se_host)
    np.testing.assert_allclose(se[ok], se_host[ok], rtol=1e-11)
    assert status["bootstrap_seed"] == 21491 and status["n_resamples"] == 256


def test_device_bootstrap_broadcast_counts(cuda):
    from kubomsd_b200 import devstats, kpm
    torch = cuda
    rng = np.random.default_rng(3)
    A = rng.normal(size=(6, 11))
    counts = np.array([4, 4, 4, 4, 4, 2])
    v_host, se_host, _ = kpm.estimate_ratio(A, counts[:, None], counts)
    v, se, _ = devstats.estimate_ratio(torch.from_numpy(A).cuda(), torch.from_numpy(counts[:, None] * 1.).cuda(),
                                       counts)
    np.testing.assert_allclose(v.cpu().numpy(), v_host, rtol=1e-13)
    np.testing.assert_allclose(se.cpu().numpy(), se_host, rtol=1e-11)


@pytest.mark.parametrize("tag", ["", "2", "3"])
def test_device_bootstrap_matches_reference_golden(cuda, tag):
    """The device bootstrap against the reference's estimate_ratio run on the
    same blocks (tests/golden/statistics.npz): unequal counts, a broadcast
    (blocks, 1) denominator, and resamples with a vanishing denominator."""
    from kubomsd_b200 import devstats
    from tests.helpers import golden
    torch = cuda
    d = golden("statistics")
    v, se, _ = devstats.estimate_ratio(torch.from_numpy(d["A" + tag]).cuda(), torch.from_numpy(d["D" + tag]).cuda(),
                                       d["counts" + tag])
    np.testing.assert_allclose(v.cpu().numpy(), d["value" + tag], rtol=1e-13)
    np.testing.assert_allclose(se.cpu().numpy(), d["stderr" + tag], rtol=1e-11, equal_nan=True)


def test_device_projection_matches_host(cuda):
    from kubomsd_b200 import devstats, kpm
    torch = cuda
    rng = np.random.default_rng(5)
    mu = rng.normal(size=(300, 5))
    E = np.linspace(-2, 2, 17)
    G = kpm.reconstruction_matrix(E, (-3., 3.), 300)
    got = devstats.project(torch.from_numpy(mu).cuda(), devstats.reconstruction_matrix(E, (-3., 3.), 300))
    assert_rel(got.cpu().numpy(), (G @ mu).T, 1e-13, "projection")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ring_correlation_matches_stored_chain(cuda, precision):
    """tables[b, j, k] from the ring contraction against the explicit
    sum_n conj(chain[j, n, b]) cov[n, k, b] over a stored FP64 chain, over
    several ring turns (length 77 > 2 x 32) and a length that is not a
    multiple of the ring."""
    from kubomsd_b200 import kpm, lattices
    from tests.gpu_util import engine
    torch = cuda
    m = lattices.square_lattice(24, seed=8)
    B = torch.from_numpy(kpm.random_phases(m.n, 2, range(6))).cuda()
    rng = np.random.default_rng(1)
    k1 = 13
    cov = torch.from_numpy(rng.normal(size=(m.n, k1, 6)) + 1j * rng.normal(size=(m.n, k1, 6))).cuda()
    _, eng, _ = engine(m.H, m.S, precision=precision)
    tables = eng.chain_correlate(B, cov, 77, 0., 11.5).cpu().numpy()
    _, e64, _ = engine(m.H, m.S)
    chain = e64.chain(B, 77, 0., 11.5).cpu().numpy()  # (77, n, 6)
    want = np.einsum("jnb,nkb->bjk", chain.conj(), cov.cpu().numpy())
    assert_rel(tables, want, 1e-12 if precision == "fp64" else 5e-5, "correlation tables")


@pytest.mark.parametrize("n", [1, 255, 256, 1000, 70001])
def test_device_phases_match_numpy_stream(cuda, n):
    """The device PCG64 stream (jump-ahead to each chunk, then steps) gives
    NumPy's draws: phases equal to the host sampler's to rounding of sin/cos."""
    from kubomsd_b200 import devstats, kpm
    ids = [0, 3, 17, 123456]
    got = devstats.random_phases(n, 20261019, ids).cpu().numpy()
    want = kpm.random_phases(n, 20261019, ids)
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-15)
    np.testing.assert_allclose(np.abs(got), 1., atol=1e-15)
