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
