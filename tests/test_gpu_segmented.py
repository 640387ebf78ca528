"""Segmented metric solves and the nonorthogonal ragged batch.

A metric over a block-diagonal S with declared segments runs one CG per
(instance, column) in shared launches; each instance must get what its own
solve gives (the reference solves one instance per Metric).  The batch built
on it must give every instance the moments of the oracle's Engine on that
instance alone."""
import numpy as np
import pytest
import scipy.linalg as la
import scipy.sparse as sp

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu

SIZES = (10, 37, 5, 64, 23)  # atoms per instance


def atom_model(na, seed, nb=4, cplx=False):
    """H and S of `na` atoms with `nb` orbitals on a ring, coupled to the
    first and second neighbours by dense nb x nb blocks; S is SPD."""
    rng = np.random.default_rng(seed)
    n = na * nb
    rows, cols, sv, hv = [], [], [], []

    def put(a, b, s_blk, h_blk):
        r, c = np.meshgrid(np.arange(nb) + a * nb, np.arange(nb) + b * nb, indexing="ij")
        rows.append(r.ravel())
        cols.append(c.ravel())
        sv.append(s_blk.ravel())
        hv.append(h_blk.ravel())

    def rnd(scale):
        m = scale * rng.standard_normal((nb, nb))
        return m + 1j * scale * rng.standard_normal((nb, nb)) if cplx else m.astype(complex)

    for a in range(na):
        d = rnd(1.)
        put(a, a, d @ d.conj().T / nb + 2. * np.eye(nb), (lambda x: x + x.conj().T)(rnd(1.)))
        for step in (1, 2):
            b = (a + step) % na
            s_blk, h_blk = rnd(.06), rnd(.5)
            put(a, b, s_blk, h_blk)
            put(b, a, s_blk.conj().T, h_blk.conj().T)
    r, c = np.concatenate(rows), np.concatenate(cols)
    S = sp.coo_matrix((np.concatenate(sv), (r, c)), shape=(n, n)).tocsr()
    H = sp.coo_matrix((np.concatenate(hv), (r, c)), shape=(n, n)).tocsr()
    blocks = [(a * nb, (a + 1) * nb, la.cholesky(S[a * nb:(a + 1) * nb, a * nb:(a + 1) * nb].toarray(), lower=True))
              for a in range(na)]
    return H, S, blocks


def make_metric(S, blocks, rtol, policy="fixed", maxiter=1000):
    from kubomsd_b200.native import B200Metric
    from tests.gpu_util import controls
    cfg = controls(rtol, policy=policy)
    cfg.metric_maxiter = maxiter
    S = sp.csr_matrix(S, dtype=complex)
    return B200Metric(S, S.diagonal().real.copy(), list(blocks), cfg), cfg


def global_system(models):
    off = np.cumsum([0] + [m[1].shape[0] for m in models])
    Sg = sp.block_diag([m[1] for m in models], format="csr")
    blocks = [(int(o) + a, int(o) + b, L) for o, m in zip(off, models) for a, b, L in m[2]]
    return Sg, blocks, off


@pytest.mark.parametrize("nb,cplx,policy", [(4, False, "fixed"), (4, True, "fixed"), (4, False, "adaptive"),
                                            (3, False, "fixed")])
def test_segmented_solve_equals_separate_solves(cuda, nb, cplx, policy):
    from kubomsd_b200 import _abi
    models = [atom_model(na, 30 + i, nb, cplx) for i, na in enumerate(SIZES)]
    Sg, blocks, off = global_system(models)
    mg, cfg = make_metric(Sg, blocks, 1e-12, policy)
    if nb == 4:  # the S products of every segment walk 4x4 block rows
        assert mg.lib.kmsd_csr_forms(mg.S.handle) & _abi.KMSD_FORM_BSR4
    mg.set_segments(off)
    rng = np.random.default_rng(5)
    B = rng.standard_normal((Sg.shape[0], 8)) + 1j * rng.standard_normal((Sg.shape[0], 8))
    B[:, 3] *= 1e-30  # tiny columns keep their own scaling per segment
    y, rep = mg.solve(B, cfg)
    y2, _ = mg.solve(B, cfg)
    np.testing.assert_array_equal(y, y2)  # deterministic
    its = rep.iterations.reshape(len(models), 8)
    assert rep.converged.shape == (len(models) * 8,) and rep.converged.all()
    for s, m in enumerate(models):
        mi, _ = make_metric(m[1], m[2], 1e-12, policy)
        yi, ri = mi.solve(B[off[s]:off[s + 1]], cfg)
        assert_rel(y[off[s]:off[s + 1]], yi, 1e-11, f"segment {s}")
        assert np.all(np.abs(its[s] - ri.iterations) <= 1), (its[s], ri.iterations)
    # the segmented solve is a true solve of the block-diagonal system
    assert_rel(Sg @ y, B, 1e-10, "residual")


def test_segmented_failure_reports_every_column(cuda):
    from kubomsd_b200.errors import NumericalError
    models = [atom_model(na, 60 + i) for i, na in enumerate(SIZES[:3])]
    Sg, blocks, off = global_system(models)
    mg, cfg = make_metric(Sg, blocks, 1e-12, maxiter=2)
    mg.set_segments(off)
    B = np.ones((Sg.shape[0], 4), complex)
    with pytest.raises(NumericalError) as failed:
        mg.solve(B, cfg)
    assert str(failed.value) == "S solve failed true-residual acceptance"
    assert len(failed.value.diagnostics["converged"]) == 3 * 4
    assert all(i == 2 for i in failed.value.diagnostics["iterations"])


def test_segments_must_not_couple(cuda):
    models = [atom_model(na, 70 + i) for i, na in enumerate(SIZES[:2])]
    Sg, blocks, off = global_system(models)
    Sg = Sg.tolil()
    Sg[0, Sg.shape[0] - 1] = Sg[Sg.shape[0] - 1, 0] = .01
    mg, _ = make_metric(Sg.tocsr(), blocks, 1e-12)
    with pytest.raises(ValueError, match="couples two segments"):
        mg.set_segments(off)
    with pytest.raises(ValueError, match="cross a segment boundary"):
        mg.set_segments([0, 6, Sg.shape[0]])


def test_nonorthogonal_batch_equals_each_instance(cuda):
    from kubomsd_b200 import kpm
    from kubomsd_b200.batch import B200Batch
    from oracle import kpm_oracle as O
    models = [atom_model(na, 80 + i) for i, na in enumerate(SIZES)]
    windows = []
    for H, S, _ in models:
        ev = la.eigh(H.toarray(), S.toarray(), eigvals_only=True)
        windows.append(((ev[-1] + ev[0]) / 2, (ev[-1] - ev[0]) / 2 * 1.05))
    c = [w[0] for w in windows]
    a = [w[1] for w in windows]
    phases = [kpm.random_phases(H.shape[0], 11 + i, range(8)) for i, (H, _, _) in enumerate(models)]
    bt = B200Batch([m[0] for m in models], precision="fp64", tile_rows=64, overlaps=[m[1] for m in models],
                   blocks=[m[2] for m in models], rtol=1e-12)
    B = bt.concat(phases)
    got = bt.moments(B, 40, c, a).cpu().numpy()  # captured: every solve a device-driven loop
    np.testing.assert_array_equal(bt.moments(B, 40, c, a).cpu().numpy(), got)  # graph replay
    np.testing.assert_array_equal(bt.moments(B, 40, c, a, use_graph=False).cpu().numpy(), got)
    for i, (H, S, blocks) in enumerate(models):
        eng = O.engine_from_model(H, S, blocks=blocks, rtol=1e-12)
        want = eng.moments(phases[i], 40, c[i], a[i])
        assert_rel(got[i], want, 1e-9, f"instance {i}")


def test_device_driven_solve_equals_host_polled(cuda):
    # Engine operations run their solves as captured graphs whose iterations
    # are a device-driven WHILE node; kmsd_metric_solve polls from the host.
    # Same kernels and the same iteration rule: the results must be
    # bit-identical, and the launches inside the device loop must be counted.
    from tests.gpu_util import engine
    H, S, blocks = atom_model(40, 21)
    rng = np.random.default_rng(3)
    B = rng.standard_normal((S.shape[0], 8)) + 1j * rng.standard_normal((S.shape[0], 8))
    metric, eng, _ = engine(H, S, blocks=blocks, rtol=1e-12)
    cfg = metric._create[2]
    rhs = eng.H.matmul(B)  # H B by the same device SpMM the engine uses
    host = metric.solve(rhs, cfg)[0]  # host-polled S^-1 (H B)
    lib = metric.lib
    before = lib.kmsd_kernel_launches()
    dev = eng.h_action(B)  # S^-1 H B through the device-driven solve
    counted = lib.kmsd_kernel_launches() - before
    np.testing.assert_array_equal(dev, host)
    assert counted >= 3 * 10  # spmv, update and direction in every iteration
