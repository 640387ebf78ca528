"""Doubling moments on lattices with a real 4-wide ELL form, across shapes.

The product identity mu_2n = 2<T_n,T_n> - mu_0, mu_2n+1 = 2<T_n+1,T_n> - mu_1
on honeycomb lattices of one and many resident waves of row groups, odd and
even moment counts, narrow and wide vector blocks, FP64 and the mixed form,
against the oracle's Engine::moments (FP64 at 1e-10, mixed at its stated
5e-5), the direct moments alongside; and two calls agree bit for bit (fixed
row ownership and reduction order).
"""
import numpy as np
import pytest

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,R,M", [((24, 12), 8, 37), ((256, 64), 16, 64), ((2048, 32), 64, 11),
                                       ((40, 20), 6, 2), ((40, 20), 6, 5)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_doubling_matches_oracle(cuda, shape, R, M, precision):
    from kubomsd_b200 import _abi, kpm, lattices
    from oracle import kpm_oracle as O
    from tests.gpu_util import engine
    m = lattices.honeycomb(*shape, W=1.5, seed=31, with_velocity=False)
    B = kpm.random_phases(m.n, 7, range(R))
    _, eng, _ = engine(m.H, m.S, precision=precision)
    lib = _abi.load()
    assert lib.kmsd_csr_forms(eng.H.handle) & _abi.KMSD_FORM_ELL
    got = eng.moments(B, M, 0., 9.6, doubling=True)
    got = got.cpu().numpy() if hasattr(got, "cpu") else got
    direct = eng.moments(B, M, 0., 9.6, doubling=False)
    direct = direct.cpu().numpy() if hasattr(direct, "cpu") else direct
    want = O.engine_from_model(m.H, m.S).moments(B, M, 0., 9.6)
    tol = 1e-10 if precision == "fp64" else 5e-5
    assert_rel(got, want, tol, f"doubling {shape} R={R} M={M} {precision}")
    assert_rel(direct, want, tol, "direct")


def test_doubling_moments_repeat_bit_for_bit(cuda):
    """Fixed row ownership and reduction order: two calls agree exactly."""
    from kubomsd_b200 import kpm, lattices
    from tests.gpu_util import engine
    m = lattices.honeycomb(512, 64, seed=3, with_velocity=False)
    B = kpm.random_phases(m.n, 1, range(32))
    _, eng, _ = engine(m.H, m.S, precision="mixed")
    a = eng.moments(B, 200, 0., 9.2, doubling=True)
    b = eng.moments(B, 200, 0., 9.2, doubling=True)
    np.testing.assert_array_equal(a, b)
