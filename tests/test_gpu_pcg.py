"""Batched device PCG vs the reference's known answers and failure reports."""
import numpy as np
import pytest
import scipy.sparse as sp

from tests.helpers import assert_rel, golden

pytestmark = pytest.mark.gpu


def metric(S, blocks=(), rtol=2e-13, maxiter=1000, policy="fixed"):
    from kubomsd_b200.native import B200Metric
    from tests.gpu_util import controls
    cfg = controls(rtol, policy=policy)
    cfg.metric_maxiter = maxiter
    S = sp.csr_matrix(S, dtype=complex)
    return B200Metric(S, S.diagonal().real.copy(), list(blocks), cfg), cfg


def test_one_jacobi_step_known_answer(cuda):
    # One Jacobi-preconditioned CG step from p = (1, .5): y = (15/17, 15/34).
    m, cfg = metric(np.array([[1., .2], [.2, 2.]]))
    cfg.metric_rtol, cfg.metric_maxiter = .5, 1
    y, rep = m.solve(np.ones((2, 1)), cfg)
    np.testing.assert_allclose(y[:, 0], [15 / 17, 15 / 34], rtol=1e-14, atol=1e-14)
    assert rep.iterations.tolist() == [1] and rep.converged.tolist() == [True]
    assert 1e-12 < rep.relative_residual[0] < .5


def test_failure_report_matches_reference(cuda):
    from kubomsd_b200.errors import NumericalError
    d = golden("pcg_known")
    m, cfg = metric(np.array([[1, .2j], [-.2j, 2]]), maxiter=1)
    with pytest.raises(NumericalError) as failed:
        m.solve(np.array([[0, 1], [0, 1]], complex), cfg)
    assert str(failed.value) == str(d["fail_message"])
    assert failed.value.diagnostics["converged"] == d["fail_converged"].tolist()
    assert failed.value.diagnostics["iterations"] == d["fail_iterations"].tolist()


@pytest.mark.parametrize("pre", ["diagonal", "block-jacobi"])
def test_extreme_column_scales(cuda, pre):
    import scipy.linalg as la
    d = golden("pcg_known")
    S, B = d["scaled_S"], d["scaled_B"]
    blocks = [] if pre == "diagonal" else [(a, b, la.cholesky(S[a:b, a:b], lower=True))
                                            for a, b in ((0, 3), (3, 7), (7, 11))]
    m, cfg = metric(S, blocks)
    y, rep = m.solve(B, cfg)
    for j in range(4):
        assert_rel(y[:, j], d[f"scaled_{pre}"][:, j], 1e-11, f"column {j}")
    np.testing.assert_array_equal(y[:, 0], 0)
    assert rep.converged.all()
    assert np.all(np.abs(rep.iterations - d[f"scaled_{pre}_iterations"]) <= 1)


@pytest.mark.parametrize("policy", ["fixed", "adaptive"])
def test_true_residual_refresh(cuda, policy):
    d = golden("pcg_known")
    n = 96
    T = sp.diags([-np.ones(n - 1), 2.03 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="csr", dtype=complex)
    m, cfg = metric(T, rtol=1e-11, policy=policy)
    y, rep = m.solve(d["tri_B"], cfg)
    want = d["tri"] if policy == "fixed" else d["tri_adaptive"]
    assert_rel(y, want, 1e-9, policy)
    assert np.all(rep.relative_residual <= 1e-11)
    st = m.stats()
    assert st.true_residual_refreshes >= 1
    if policy == "fixed":
        assert abs(st.true_residual_refreshes - int(d["tri_refreshes"])) <= 1


def test_unrepresentable_solution_is_rejected(cuda):
    from kubomsd_b200.errors import NumericalError
    m, cfg = metric(.25 * np.eye(2))
    with pytest.raises(NumericalError, match="representable") as failed:
        m.solve(np.array([[1e308, 1.], [1., 1.]], dtype=complex), cfg)
    assert failed.value.diagnostics["converged"] == [False, True]


def test_extreme_finite_rhs_keeps_representable_solution(cuda):
    m, cfg = metric(np.eye(2))
    y, rep = m.solve(np.array([[complex(1.3e308, 1.3e308)], [1. + 0j]]), cfg)
    assert np.isfinite(y).all()
    np.testing.assert_allclose(y[0].real / 1.3e308, [1.], rtol=1e-14)
    np.testing.assert_allclose(y[1], [1.], rtol=1e-14, atol=0)
    assert rep.converged.tolist() == [True]


@pytest.mark.parametrize("cplx", [False, True])
def test_block_sparse_spmm_and_solve(cuda, cplx):
    # An atom-block operator (dense 4x4 blocks on a ring of 40 atoms, each
    # coupled to its two neighbours) is stored as 4x4 block-CSR: the SpMM and
    # every S product of the PCG walk block rows.  Both must agree with SciPy.
    import scipy.linalg as la
    import scipy.sparse.linalg as spla
    from kubomsd_b200 import _abi
    from kubomsd_b200.native import DeviceCSR
    rng = np.random.default_rng(7 + cplx)
    na, nb = 40, 4
    n = na * nb
    rows = []
    for a in range(na):
        for b in (a - 1, a + 1):
            blk = .08 * rng.standard_normal((nb, nb))
            if cplx:
                blk = blk + .08j * rng.standard_normal((nb, nb))
            rows.append((a, b % na, blk))
    S = sp.lil_matrix((n, n), dtype=complex)
    for a, b, blk in rows:
        S[a * nb:(a + 1) * nb, b * nb:(b + 1) * nb] += blk
    S = S.tocsr()
    S = S + S.conj().T
    for a in range(na):
        d = rng.standard_normal((nb, nb)) + (1j * rng.standard_normal((nb, nb)) if cplx else 0)
        S[a * nb:(a + 1) * nb, a * nb:(a + 1) * nb] += d @ d.conj().T + 2 * np.eye(nb)
    S = sp.csr_matrix(S)
    if not cplx:
        S = sp.csr_matrix(S.real.astype(complex))
    A = DeviceCSR(S)
    assert A.lib.kmsd_csr_forms(A.handle) & _abi.KMSD_FORM_BSR4
    X = rng.standard_normal((n, 8)) + 1j * rng.standard_normal((n, 8))
    assert_rel(A.matmul(X), S @ X, 1e-14, "block SpMM")
    blocks = [(a * nb, (a + 1) * nb, la.cholesky(S[a * nb:(a + 1) * nb, a * nb:(a + 1) * nb].toarray(), lower=True))
              for a in range(na)]
    m, cfg = metric(S, blocks, rtol=1e-12)
    y, rep = m.solve(X, cfg)
    assert rep.converged.all()
    ref = spla.spsolve(S.tocsc(), X)
    assert_rel(y, ref, 1e-10, "block-sparse metric solve")


def _hermitian_blocks(sizes, seed, coupling=0.):
    """A complex Hermitian positive definite S whose diagonal blocks have the
    given sizes, plus an optional sparse Hermitian coupling between them
    (diagonally shifted so that S stays positive definite)."""
    rng = np.random.default_rng(seed)
    off = np.cumsum([0] + list(sizes))
    n = int(off[-1])
    S = np.zeros((n, n), complex)
    for a, b in zip(off[:-1], off[1:]):
        X = rng.standard_normal((b - a, b - a)) + 1j * rng.standard_normal((b - a, b - a))
        S[a:b, a:b] = X @ X.conj().T / (b - a) + np.eye(b - a)
    if coupling:
        C = coupling * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        C = np.where(rng.random((n, n)) < .2, C, 0.)
        C = np.triu(C, 1)
        C = C + C.conj().T
        S += C + np.diag(np.abs(C).sum(axis=1))
    return S, off


@pytest.mark.parametrize("sizes", [(1, 2, 5, 8, 3, 4, 7, 6), (12, 9, 4, 1, 10)])
def test_block_jacobi_of_a_block_diagonal_metric_is_exact(cuda, sizes):
    # Blocks of up to 8 rows are applied as stored block inverses, larger
    # ones by substitution with the Cholesky factor: either way M^-1 = S^-1
    # here, so one iteration converges.
    import scipy.linalg as la
    S, off = _hermitian_blocks(sizes, 40 + len(sizes))
    blocks = [(int(a), int(b), la.cholesky(S[a:b, a:b], lower=True)) for a, b in zip(off[:-1], off[1:])]
    m, cfg = metric(S, blocks)
    rng = np.random.default_rng(3)
    B = rng.standard_normal((S.shape[0], 3)) + 1j * rng.standard_normal((S.shape[0], 3))
    y, rep = m.solve(B, cfg)
    assert rep.iterations.tolist() == [1, 1, 1] and rep.converged.all()
    assert_rel(y, np.linalg.solve(S, B), 1e-12, "solution")


@pytest.mark.parametrize("sizes", [(1, 2, 5, 8, 3, 4, 7, 6) * 3, (12, 9, 4, 1, 10) * 2])
def test_block_jacobi_on_a_coupled_complex_metric(cuda, sizes):
    import scipy.linalg as la
    S, off = _hermitian_blocks(sizes, 50 + len(sizes), coupling=.05)
    blocks = [(int(a), int(b), la.cholesky(S[a:b, a:b], lower=True)) for a, b in zip(off[:-1], off[1:])]
    m, cfg = metric(S, blocks, rtol=1e-12)
    md, _ = metric(S, (), rtol=1e-12)
    rng = np.random.default_rng(4)
    B = rng.standard_normal((S.shape[0], 5)) + 1j * rng.standard_normal((S.shape[0], 5))
    y, rep = m.solve(B, cfg)
    yd, repd = md.solve(B, cfg)
    assert rep.converged.all() and repd.converged.all()
    want = np.linalg.solve(S, B)
    assert_rel(y, want, 1e-10, "block-Jacobi solution")
    assert_rel(yd, want, 1e-10, "diagonal solution")
    assert rep.iterations.max() <= repd.iterations.max()  # the blocks precondition at least as well
