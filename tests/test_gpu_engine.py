"""B200 engine vs the reference (golden vectors from KuboMSD's own engine):
every operation of the reference Engine / Metric on nonorthogonal models with
all three velocity kinds and both preconditioners, FP64."""
import numpy as np
import pytest

from tests.helpers import assert_rel, golden

pytestmark = pytest.mark.gpu
KINDS = ["velocity", "position", "composite"]
PRECONDS = ["diagonal", "block-jacobi"]


@pytest.mark.parametrize("pre", PRECONDS)
@pytest.mark.parametrize("kind", KINDS)
def test_engine_operations_match_reference(cuda, kind, pre):
    from tests.gpu_util import fixture_engine
    d = golden(f"engine_{kind}_{pre}")
    metric, eng, _ = fixture_engine(d, kind, pre)
    B, c, a = d["B"], float(d["center"]), float(d["half"])
    assert_rel(eng.h_action(B), d["h_action"], 1e-11, "h_action")
    assert_rel(eng.v_cov([1., 0., 0.], B), d["v_cov"], 1e-10, "v_cov")
    assert_rel(eng.chain(B, 12, c, a), d["chain"], 1e-10, "chain")
    assert_rel(eng.moments(B, 20, c, a), d["moments"], 1e-10, "moments")
    assert_rel(eng.series(B, d["coeff"], c, a), d["series_plain"], 1e-10, "series")
    assert_rel(eng.series(d["aug"], d["coeff"], c, a, [[1., 0., 0.]]), d["series_aug"], 1e-10, "augmented")
    cfg = type("C", (), dict(metric_rtol=float(d["rtol"]), metric_atol=0., metric_maxiter=1000,
                             metric_residual_policy="fixed", metric_check_interval=32, metric_gap_ratio=.1))()
    y, rep = metric.solve(B, cfg)
    assert_rel(y, d["solve"], 1e-11, "solve")
    assert rep.converged.all()
    assert np.all(np.abs(rep.iterations - d["solve_iterations"]) <= 1)
    assert np.all(rep.relative_residual <= float(d["rtol"]))
    assert_rel(metric.sample(d["xi"], d["sample_coeff"], float(d["sample_center"]), float(d["sample_half"])),
               d["sample"], 1e-12, "sample")


@pytest.mark.parametrize("pre", PRECONDS)
@pytest.mark.parametrize("kind", KINDS)
def test_propagation_and_stepwise_match_reference(cuda, kind, pre):
    from kubomsd_b200 import stochastic
    from kubomsd_b200.config import RunConfig
    from tests.gpu_util import fixture_engine
    d = golden(f"engine_{kind}_{pre}")
    _, eng, ops = fixture_engine(d, kind, pre)
    cfg = RunConfig(energy_eV=d["energies"], time_fs=d["times"], spectral_bounds=tuple(d["bounds"]),
                    n_moments=int(d["n_moments"]), axes=("x",), segment_fs=float(d["segment_fs"]),
                    metric_rtol=float(d["rtol"]), include_vac=False, stochastic_method="stepwise", preconditioner=pre)
    out, diag = stochastic.propagate(d["B"], .2, ops, cfg)
    assert_rel(out, d["propagate"], 1e-10, "propagate")
    dos, nums, _ = stochastic.stepwise_samples(ops, cfg, d["B"])
    assert_rel(dos, d["dos"], 1e-10, "dos")
    assert_rel(nums["msd_A2/commutator"], d["msd"], 1e-9, "msd")


def test_h_action_of_nonfinite_input_is_rejected(cuda):
    from kubomsd_b200.errors import NumericalError
    from tests.gpu_util import fixture_engine
    d = golden("engine_velocity_diagonal")
    _, eng, _ = fixture_engine(d, "velocity", "diagonal")
    B = d["B"].copy()
    B[1, 1] = np.nan
    with pytest.raises(NumericalError, match="finite"):
        eng.h_action(B)


def test_engine_counters_follow_reference_semantics(cuda):
    from tests.gpu_util import fixture_engine
    d = golden("engine_velocity_diagonal")
    _, eng, _ = fixture_engine(d, "velocity", "diagonal")
    eng.moments(d["B"], 20, float(d["center"]), float(d["half"]))
    assert eng.core.h_calls == 19
    eng.series(d["aug"], d["coeff"], float(d["center"]), float(d["half"]), [[1., 0., 0.]])
    assert eng.core.h_calls == 19 + len(d["coeff"]) - 1
    assert eng.core.v_calls == len(d["coeff"]) - 1


@pytest.mark.parametrize("pre", PRECONDS)
@pytest.mark.parametrize("kind", KINDS)
def test_spectral_vac_matches_reference(cuda, kind, pre):
    from kubomsd_b200 import stochastic
    from kubomsd_b200.config import RunConfig
    from tests.gpu_util import fixture_engine
    d = golden(f"engine_{kind}_{pre}")
    _, eng, ops = fixture_engine(d, kind, pre)
    cfg = RunConfig(energy_eV=d["energies"], time_fs=d["times"], spectral_bounds=tuple(d["bounds"]),
                    n_moments=int(d["n_moments"]), axes=("x",), segment_fs=float(d["segment_fs"]),
                    metric_rtol=float(d["rtol"]), include_vac=True, stochastic_method="spectral",
                    integration_dt_fs=float(d["integration_dt_fs"]), preconditioner=pre)
    dos, out, diag = stochastic.spectral_samples(ops, cfg, d["B"])
    assert_rel(dos, d["dos"], 1e-10, "dos")
    for key in ("msd_A2/vac_integral", "diffusion_A2_per_fs/vac_integral", "vac_A2_per_fs2/vac_integral"):
        assert_rel(out[key], d["spectral/" + key], 1e-9, key)
