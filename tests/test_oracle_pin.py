"""The oracle restatement pinned to the reference: golden vectors produced by
running KuboMSD (tests/golden/make_golden.py) and, where oracle/_ref is
built, the reference's compiled engine itself on fresh random inputs."""
import numpy as np
import pytest
import scipy.sparse as sp

from tests.helpers import assert_rel, fixture_blocks, fixture_model, golden
from oracle import kpm_oracle as O
from oracle import ref_native

KINDS = ["velocity", "position", "composite"]
PRECONDS = ["diagonal", "block-jacobi"]


def oracle_engine(d, kind, pre):
    H, S, vel, pos, comp = fixture_model(d, kind)
    blocks = fixture_blocks(d) if pre == "block-jacobi" else ()
    return O.engine_from_model(H, S, vel, pos, comp, blocks=blocks, rtol=float(d["rtol"]))


@pytest.mark.parametrize("pre", PRECONDS)
@pytest.mark.parametrize("kind", KINDS)
def test_oracle_engine_matches_reference_golden(kind, pre):
    d = golden(f"engine_{kind}_{pre}")
    e = oracle_engine(d, kind, pre)
    B, c, a = d["B"], float(d["center"]), float(d["half"])
    assert_rel(e.h_action(B), d["h_action"], 1e-11, "h_action")
    assert_rel(e.v_cov([1., 0., 0.], B), d["v_cov"], 1e-10, "v_cov")
    assert_rel(e.chain(B, 12, c, a), d["chain"], 1e-10, "chain")
    assert_rel(e.moments(B, 20, c, a), d["moments"], 1e-10, "moments")
    assert_rel(e.series(B, d["coeff"], c, a), d["series_plain"], 1e-10, "series")
    assert_rel(e.series(d["aug"], d["coeff"], c, a, [[1., 0., 0.]]), d["series_aug"], 1e-10, "augmented series")
    assert_rel(e.metric.solve(B, float(d["rtol"]), 0., 1000)[0], d["solve"], 1e-11, "solve")
    assert_rel(e.metric.sample(d["xi"], d["sample_coeff"], float(d["sample_center"]), float(d["sample_half"])),
               d["sample"], 1e-12, "sample")
    bounds = tuple(d["bounds"])
    out, _ = O.propagate(e, B, .2, bounds, float(d["segment_fs"]), 1e-12, 4096)
    assert_rel(out, d["propagate"], 1e-10, "propagate")
    dos, msd = O.stepwise_samples(e, B, d["energies"], d["times"], bounds, int(d["n_moments"]), [[1., 0., 0.]],
                                  segment_fs=float(d["segment_fs"]))
    assert_rel(dos, d["dos"], 1e-10, "dos")
    assert_rel(msd, d["msd"], 1e-9, "msd")


def test_oracle_pcg_known_answers():
    d = golden("pcg_known")
    m = O.Metric(np.array([[1., .2], [.2, 2.]]), [1., 2.])
    y, rep = m.solve(np.ones((2, 1)), .5, 0., 1)
    np.testing.assert_allclose(y[:, 0], [15 / 17, 15 / 34], rtol=1e-14)
    np.testing.assert_allclose(y, d["one_step"], rtol=1e-14)
    assert rep["iterations"] == [1]
    m = O.Metric(np.array([[1, .2j], [-.2j, 2]]), [1., 2.])
    with pytest.raises(O.MetricFailure) as failed:
        m.solve(np.array([[0, 1], [0, 1]], complex), 2e-13, 0., 1)
    assert failed.value.diagnostics["converged"] == d["fail_converged"].tolist()
    assert failed.value.diagnostics["iterations"] == d["fail_iterations"].tolist()
    assert str(failed.value) == str(d["fail_message"])
    S, B = d["scaled_S"], d["scaled_B"]
    for pre in ("diagonal", "block-jacobi"):
        import scipy.linalg as la
        blocks = [] if pre == "diagonal" else [(a, b, la.cholesky(S[a:b, a:b], lower=True))
                                                for a, b in ((0, 3), (3, 7), (7, 11))]
        y, rep = O.Metric(S, S.diagonal().real, blocks).solve(B, 2e-13, 0., 1000)
        for j in range(4):
            assert_rel(y[:, j], d[f"scaled_{pre}"][:, j], 1e-11, f"{pre} column {j}")
        # iteration counts at a 2e-13 threshold depend on the last bits: +-1
        assert np.all(np.abs(np.array(rep["iterations"]) - d[f"scaled_{pre}_iterations"]) <= 1)
    n = 96
    T = sp.diags([-np.ones(n - 1), 2.03 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="csr", dtype=complex)
    m = O.Metric(T, T.diagonal().real)
    y, rep = m.solve(d["tri_B"], 1e-11, 0., 1000)
    assert_rel(y, d["tri"], 1e-9, "tridiagonal")
    assert abs(m.refreshes - int(d["tri_refreshes"])) <= 1
    m = O.Metric(T, T.diagonal().real, policy="adaptive")
    y, rep = m.solve(d["tri_B"], 1e-11, 0., 1000)
    assert_rel(y, d["tri_adaptive"], 1e-9, "tridiagonal adaptive")
    assert np.all(np.abs(np.array(rep["iterations"]) - d["tri_adaptive_iterations"]) <= 1)


def test_oracle_host_formulas():
    d = golden("host_formulas")
    bounds = (-11.2, 11.2)
    for tag, dt, w in (("a", 1., True), ("b", .3, False), ("c", .07, True)):
        b, _ = O.bessel_coefficients(dt, bounds, 1e-12, 4096, weighted_tail=w)
        np.testing.assert_allclose(b, d[f"bessel_{tag}"], rtol=1e-14, atol=1e-300)
    for L in (1, 2, 64, 1024):
        np.testing.assert_allclose(O.jackson(L), d[f"jackson_{L}"], rtol=1e-14)
    np.testing.assert_allclose(O.reconstruction(np.linspace(-11, 11, 41), bounds, 128), d["G"], rtol=1e-13)
    np.testing.assert_array_equal(O.random_phases(16, 7, [0, 1, 2, 5]), d["phases"])
    np.testing.assert_array_equal(O.random_phases(4096, 20261019, [0, 7])[:256], d["phases_c1_head"])


def test_oracle_c1_moments_and_short_msd():
    from kubomsd_b200 import lattices
    from tests.golden import make_golden_digest as dg
    d = golden("c1_square64")
    m = lattices.square_lattice(64)
    assert dg.digest(m.H) == str(d["H_digest"]) and dg.digest(m.velocity["x"]) == str(d["V_digest"])
    e = O.engine_from_model(m.H, m.S, m.velocity)
    B = O.random_phases(m.n, 20261019, range(8))
    c, a = O.scaling((-11.2, 11.2))
    assert_rel(e.moments(B, 512, c, a), d["moments"], 1e-11, "C1 moments")


def test_oracle_diamond_nonorthogonal():
    import scipy.linalg as la
    from kubomsd_b200 import lattices
    from tests.golden import make_golden_digest as dg
    d = golden("diamond2")
    m = lattices.diamond_sp3(cells=2)
    assert dg.digest(m.H) == str(d["H_digest"]) and dg.digest(m.S) == str(d["S_digest"])
    S = sp.csr_matrix(m.S)
    blocks = [(a, b, la.cholesky(S[a:b, a:b].toarray(), lower=True)) for a, b in m.atom_slices]
    e = O.engine_from_model(m.H, m.S, composite=m.composite, blocks=blocks, rtol=1e-12)
    c, a = O.scaling(tuple(d["bounds"]))
    assert_rel(e.moments(d["B"], 32, c, a), d["moments"], 1e-10, "diamond moments")
    assert_rel(e.v_cov([0., 1., 0.], d["B"]), d["v_cov_y"], 1e-10, "diamond v_cov y")
    assert_rel(e.metric.sample(d["xi"], d["sample_coeff"], float(d["sample_center"]), float(d["sample_half"])),
               d["sample"], 1e-11, "diamond sample")


@pytest.mark.skipif(ref_native.load() is None, reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_matches_compiled_reference_live(seed):
    """Fresh random nonorthogonal models: oracle vs the reference's own binary."""
    rng = np.random.default_rng(seed)
    n = 14
    A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    S = np.eye(n) + .02 * (A.conj().T @ A)
    H = (A + A.conj().T) / 9
    V = (A - A.conj().T) * .1j
    ref = ref_native.RefEngine(H, S, velocity={"y": V}, rtol=2e-13)
    e = O.engine_from_model(H, S, velocity={"y": V}, rtol=2e-13)
    B = rng.normal(size=(n, 4)) + 1j * rng.normal(size=(n, 4))
    assert_rel(e.moments(B, 30, .1, 2.), ref.core.moments(B, 30, .1, 2.), 1e-10, "moments")
    coeff = np.exp(1j * np.arange(9)) / (1 + np.arange(9)) ** 3
    aug = np.concatenate([B, B[:, ::-1]], axis=1)
    assert_rel(e.series(aug, coeff, .1, 2., [[0., 1., 0.]]), ref.core.series(aug, coeff, .1, 2., [[0., 1., 0.]]),
               1e-10, "series")
    assert_rel(e.chain(B, 7, .1, 2.), ref.core.chain(B, 7, .1, 2.), 1e-10, "chain")
    y, rep = ref.metric.solve(B, 2e-13, 0., 1000)
    assert_rel(e.metric.solve(B, 2e-13, 0., 1000)[0], y, 1e-11, "solve")


@pytest.mark.parametrize("kind", KINDS)
def test_oracle_spectral_vac_matches_reference(kind):
    d = golden(f"engine_{kind}_diagonal")
    e = oracle_engine(d, kind, "diagonal")
    dos, out = O.spectral_samples(e, d["B"], d["energies"], d["times"], tuple(d["bounds"]), int(d["n_moments"]),
                                  [[1., 0., 0.]], float(d["integration_dt_fs"]), segment_fs=float(d["segment_fs"]))
    assert_rel(dos, d["dos"], 1e-10, "dos")
    for key, value in out.items():
        assert_rel(value, d["spectral/" + key], 1e-9, key)
