"""`python -m kubomsd_b200 run` end to end (model.json in, results out) with the
reference's option names, against the reference pipeline's output arrays."""
import numpy as np
import pytest

from tests.helpers import golden

pytestmark = pytest.mark.gpu


def test_cli_run_matches_reference_pipeline(cuda, tmp_path):
    from kubomsd_b200 import cli, io, lattices
    d = golden("square16_pipeline")
    m = lattices.square_lattice(16, seed=99)
    model = io.save_model(m, tmp_path / "model")
    out = tmp_path / "run"
    rc = cli.main(["run", "--input", str(model), "--out", str(out), "--solver", "stochastic-kpm", "--backend", "gpu",
                   "--kernel", "jackson", "--stochastic-method", "stepwise", "--no-vac", "--axes", "x",
                   "--emin", "-9", "--emax", "9", "--n-energy", "19", "--tmax-fs", "3", "--dt-fs", "1",
                   "--n-moments", "64", "--nsamples", "8", "--sample-batch", "4", "--statistics-block", "2",
                   "--seed", "515", "--spectral-min", "-11.5", "--spectral-max", "11.5"])
    assert rc == 0
    res = io.read_results(out)
    assert res["metadata"]["run_status"] == "complete"
    arrays = res["arrays"]
    for key in ("msd_A2/commutator", "dos_states_per_eV", "numerator_block_sums/msd_A2/commutator",
                "stderr_msd_A2/commutator", "diffusion_A2_per_fs/msd_gradient"):
        want = d["arr/" + key]
        np.testing.assert_allclose(arrays[key], want, rtol=1e-9, atol=1e-12 * np.nanmax(np.abs(want)),
                                   equal_nan=True, err_msg=key)
    assert "msd_x_A2" in arrays and "diffusion_direction_average_A2_per_fs" in arrays


def test_cli_rejects_exact_solver(tmp_path):
    from kubomsd_b200 import cli
    rc = cli.main(["run", "--input", str(tmp_path / "m.json"), "--out", str(tmp_path / "o"), "--solver", "exact",
                   "--emin", "-1", "--emax", "1"])
    assert rc == 2
