"""The whole stochastic pipeline — seeded phases, metric sampling, stepwise
MSD, block sums, paired bootstrap, validity masks — through the B200 operator
bundle vs the reference's iter_stochastic_blocks output arrays."""
import numpy as np
import pytest

from tests.helpers import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,method,vac", [("square16_pipeline", "stepwise", False),
                                              ("square16_pipeline_vac", "stepwise", True),
                                              ("square16_pipeline_spectral", "spectral", False)])
def test_square16_pipeline_matches_reference(cuda, name, method, vac):
    from kubomsd_b200 import lattices, stochastic
    from kubomsd_b200.config import RunConfig
    from kubomsd_b200.operators import build_operators
    from tests.golden.make_golden_digest import digest
    d = golden(name)
    m = lattices.square_lattice(16, seed=99)
    assert digest(m.H) == str(d["H_digest"])
    cfg = RunConfig(energy_eV=np.linspace(-9, 9, 19), time_fs=[0., 1., 2., 3.], axes=("x",),
                    spectral_bounds=(-11.5, 11.5), n_moments=64, nsamples=8, sample_batch=4, statistics_block=2,
                    include_vac=vac, stochastic_method=method, seed=515, integration_dt_fs=.05)
    ops = build_operators(m, cfg)
    blocks = list(stochastic.iter_stochastic_blocks(ops, cfg, method))
    got = {}
    for blk in blocks:
        got.update(blk.static)
        got.update(blk.arrays)
    want = {k[4:]: v for k, v in d.items() if k.startswith("arr/")}
    assert set(want) <= set(got), set(want) - set(got)
    for key, value in want.items():
        g = np.asarray(got[key])
        if value.dtype.kind in "biu":
            np.testing.assert_array_equal(g, value, err_msg=key)
        else:
            np.testing.assert_allclose(g, value, rtol=1e-9, atol=1e-12 * np.nanmax(np.abs(value)), equal_nan=True,
                                       err_msg=key)
