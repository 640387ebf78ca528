"""The mixed form on a nonorthogonal basis: the CG work vectors of the metric
solve stored as complex64, with FP64 arithmetic, solution, inner products,
norms and acceptance.  It must reach the same tolerance as the FP64 solve,
and the moments built on it must agree with the FP64 ones."""
import numpy as np
import pytest

from tests.helpers import assert_rel
from tests.test_gpu_segmented import SIZES, atom_model, global_system, make_metric

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cplx", [False, True])
def test_mixed_storage_solve_reaches_the_fp64_tolerance(cuda, cplx):
    H, S, blocks = atom_model(64, 3, cplx=cplx)
    rng = np.random.default_rng(2)
    B = rng.standard_normal((S.shape[0], 16)) + 1j * rng.standard_normal((S.shape[0], 16))
    m64, cfg = make_metric(S, blocks, 1e-10)
    m32, _ = make_metric(S, blocks, 1e-10)
    m32.set_storage("mixed")
    y64, r64 = m64.solve(B, cfg)
    y32, r32 = m32.solve(B, cfg)
    assert r32.converged.all() and r64.converged.all()
    assert np.all(r32.relative_residual <= 1e-10)  # true residual, computed in FP64
    assert_rel(y32, y64, 1e-8, "mixed vs FP64 solution")
    assert r32.iterations.max() <= 1.5 * r64.iterations.max() + 8, (r32.iterations, r64.iterations)


def test_mixed_segmented_solve(cuda):
    models = [atom_model(na, 30 + i) for i, na in enumerate(SIZES)]
    Sg, blocks, off = global_system(models)
    mg, cfg = make_metric(Sg, blocks, 1e-10)
    mg.set_storage("mixed")
    mg.set_segments(off)
    rng = np.random.default_rng(6)
    B = rng.standard_normal((Sg.shape[0], 8)) + 1j * rng.standard_normal((Sg.shape[0], 8))
    y, rep = mg.solve(B, cfg)
    assert rep.converged.all() and np.all(rep.relative_residual <= 1e-10)
    assert_rel(Sg @ y, B, 1e-9, "residual")


def test_mixed_engine_moments_on_a_nonorthogonal_basis(cuda):
    from tests.gpu_util import engine
    H, S, blocks = atom_model(48, 9)
    rng = np.random.default_rng(1)
    B = np.exp(2j * np.pi * rng.random((S.shape[0], 8)))
    _, e64, _ = engine(H, S, blocks=blocks, rtol=1e-10, precision="fp64")
    _, e32, _ = engine(H, S, blocks=blocks, rtol=1e-10, precision="mixed")
    assert e32.metric.storage == "mixed" and e32.engine_precision == "fp64"
    want = e64.moments(B, 64, 0., 12.)
    got = e32.moments(B, 64, 0., 12.)
    assert_rel(got, want, 1e-8, "moments")


def test_mixed_nonorthogonal_batch(cuda):
    from kubomsd_b200 import kpm
    from kubomsd_b200.batch import B200Batch
    models = [atom_model(na, 80 + i) for i, na in enumerate(SIZES)]
    phases = [kpm.random_phases(m[0].shape[0], 11 + i, range(8)) for i, m in enumerate(models)]
    kw = dict(tile_rows=64, overlaps=[m[1] for m in models], blocks=[m[2] for m in models], rtol=1e-10)
    b64 = B200Batch([m[0] for m in models], precision="fp64", **kw)
    b32 = B200Batch([m[0] for m in models], precision="mixed", **kw)
    B = b64.concat(phases)
    want = b64.moments(B, 32, 0., 12.).cpu().numpy()
    got = b32.moments(B, 32, 0., 12.).cpu().numpy()
    for i in range(len(models)):
        assert_rel(got[i], want[i], 1e-8, f"instance {i}")
