"""Continuous-batching service: requests that arrive while others run are
admitted as slots and HBM budget free up, their work overlaps on the device,
and every result is the same alone and in the mix."""
import numpy as np
import pytest

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def models(cuda):
    from kubomsd_b200 import lattices
    from kubomsd_b200.serving import ResidentModel
    sq = lattices.square_lattice(48, seed=2)
    hc = lattices.honeycomb(96, 48, seed=4)
    dm = lattices.diamond_sp3(cells=2)
    return {"square": ResidentModel("square", sq, (-11.5, 11.5), precision="mixed"),
            "honeycomb": ResidentModel("honeycomb", hc, (-9.2, 9.2), precision="mixed"),
            "diamond": ResidentModel("diamond", dm, (-40., 40.), precision="fp64")}


def test_results_identical_alone_and_in_the_mix(models):
    from kubomsd_b200.serving import Request, Server, latency_summary
    reqs = []
    rng = np.random.default_rng(8)
    names = ["square", "honeycomb", "diamond"]
    for i in range(12):
        kind = "msd" if i % 4 == 3 else "dos"
        reqs.append(Request(.01 * i, i, names[i % 3], kind, int(rng.choice([128, 256])), int(rng.choice([8, 16])),
                            1000 + i, [0., .5, 1.] if kind == "msd" else None))
    srv = Server(models, slots=4)
    mixed = srv.serve(reqs)
    assert not srv.errors, srv.errors
    assert len(mixed) == len(reqs)
    alone = []
    for r in reqs:  # one at a time, nothing else on the device
        alone += Server(models, slots=1).serve([r])
    for a, b in zip(mixed, alone):
        assert a.rid == b.rid
        assert_rel(a.value, b.value, 1e-12, f"request {a.rid}")
    # work of different requests overlapped in time on the device
    spans = sorted((r.start, r.end) for r in mixed)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    s = latency_summary(mixed)
    assert s["requests"] == 12 and s["p99_s"] >= s["p50_s"] > 0


def test_admission_waits_for_hbm_budget(models):
    from kubomsd_b200.serving import Request, Server
    srv = Server(models, slots=4)
    one = models["honeycomb"].job_bytes(Request(0., 0, "honeycomb", "dos", 64, 16, 1))
    srv.budget = int(1.5 * one)  # room for one honeycomb job at a time
    reqs = [Request(0., i, "honeycomb", "dos", 256, 16, i) for i in range(3)]
    res = srv.serve(reqs)
    assert len(res) == 3
    spans = sorted((r.start, r.end) for r in res)
    assert all(spans[i + 1][0] >= spans[i][1] - 1e-3 for i in range(2))  # admitted one after another


@pytest.mark.parametrize("kind", ["moments", "series"])
def test_replicas_first_use_concurrently(cuda, kind):
    """Engine replicas share one uploaded model and build its complex64 copy on
    first use.  Replicas whose first mixed-precision calls start at the same
    time on two host threads and streams return exactly what one call alone
    returns (the copy is published only once it is complete)."""
    import threading
    from kubomsd_b200 import kpm, lattices
    from kubomsd_b200.config import RunConfig
    from kubomsd_b200.operators import build_operators
    torch = cuda
    m = lattices.honeycomb(256, 128, seed=9)
    cfg = RunConfig(energy_eV=[0.], time_fs=[0., 1.], spectral_bounds=(-9.2, 9.2), axes=("x",), include_vac=False,
                    precision="mixed", moment_doubling=True)
    c, a = kpm.scaling(cfg)
    B = torch.from_numpy(kpm.random_phases(m.n, 4, range(8))).cuda()
    coeff, _ = kpm.bessel_coefficients(.5, cfg, weighted_tail=True)
    aug = torch.cat([B, torch.zeros_like(B)], dim=1).contiguous()

    def call(eng):
        if kind == "moments":
            return eng.moments(B, 64, c, a).cpu().numpy()
        return eng.series(aug, coeff, c, a, [[1., 0., 0.]]).cpu().numpy()

    engines = [build_operators(m, cfg).native]
    engines.append(engines[0].replica())
    out, errors = [None, None], []
    gate = threading.Barrier(2)

    def worker(i):
        try:
            with torch.cuda.stream(torch.cuda.Stream()):
                gate.wait(timeout=30)
                out[i] = call(engines[i])
        except Exception as exc:  # noqa: BLE001
            errors.append(exc)

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=120)
    assert not errors, errors
    alone = call(engines[0])
    for got in out:
        assert np.isfinite(got).all()
        np.testing.assert_array_equal(got, alone)
