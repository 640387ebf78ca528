"""Host-side logic of the package, on the CPU: the KPM host formulas against
the reference's golden values, the accuracy report, the workspace gates,
the segmentation of integration nodes, the request stream of the service
and the bench's sizing rules.  Nothing here launches a kernel."""
import numpy as np
import pytest

from tests.helpers import golden


def _cfg(**kw):
    from kubomsd_b200.config import RunConfig
    base = dict(energy_eV=np.linspace(-9, 9, 21), time_fs=[0., 1., 2.], spectral_bounds=(-11.2, 11.2),
                n_moments=128, axes=("x",))
    base.update(kw)
    return RunConfig(**base)


# ------------------------------------------------------------ host formulas
def test_bessel_coefficients_match_reference_golden():
    from kubomsd_b200 import kpm
    d = golden("host_formulas")
    for tag, dt, w in (("a", 1., True), ("b", .3, False), ("c", .07, True)):
        b, info = kpm.bessel_coefficients(dt, _cfg(propagation_tol=1e-12, propagation_max_order=4096),
                                          weighted_tail=w)
        np.testing.assert_allclose(b, d[f"bessel_{tag}"], rtol=1e-14, atol=1e-300)
        assert info["order"] == len(b) - 1


def test_jackson_and_reconstruction_match_reference_golden():
    from kubomsd_b200 import kpm
    d = golden("host_formulas")
    for L in (1, 2, 64, 1024):
        np.testing.assert_allclose(kpm.jackson_coefficients(L), d[f"jackson_{L}"], rtol=1e-14)
    G = kpm.reconstruction_matrix(np.linspace(-11, 11, 41), (-11.2, 11.2), 128)
    np.testing.assert_allclose(G, d["G"], rtol=1e-13)


def test_host_phases_match_reference_golden():
    from kubomsd_b200 import kpm
    d = golden("host_formulas")
    np.testing.assert_array_equal(kpm.random_phases(16, 7, [0, 1, 2, 5]), d["phases"])
    np.testing.assert_array_equal(kpm.random_phases(4096, 20261019, [0, 7])[:256], d["phases_c1_head"])


@pytest.mark.parametrize("bounds,energies,message", [
    ((1., -1.), [0.], "invalid spectral bounds"),
    ((-1., np.inf), [0.], "invalid spectral bounds"),
    ((-1., 1.), [1.5], "do not contain full spectrum"),
])
def test_spectral_window_errors(bounds, energies, message):
    from kubomsd_b200 import kpm
    with pytest.raises(Exception, match=message):
        kpm.validate_spectral_window(energies, bounds)


def test_reconstruction_rejects_energies_on_the_window_edge():
    from kubomsd_b200 import kpm
    with pytest.raises(Exception, match="strictly inside"):
        kpm.reconstruction_matrix([-11.2, 0.], (-11.2, 11.2), 16)


@pytest.mark.parametrize("tag", ["", "2", "3"])
def test_bootstrap_ratio_matches_reference_golden(tag):
    """The host paired block bootstrap (kpm.estimate_ratio) against the
    reference's own estimate_ratio on the same blocks: unequal counts, a
    broadcast (blocks, 1) denominator, and resamples whose denominator
    vanishes (NaN kept, as the reference keeps it)."""
    from kubomsd_b200 import kpm
    d = golden("statistics")
    v, se, st = kpm.estimate_ratio(d["A" + tag], d["D" + tag], d["counts" + tag])
    np.testing.assert_allclose(v, d["value" + tag], rtol=1e-14)
    np.testing.assert_allclose(se, d["stderr" + tag], rtol=1e-12, equal_nan=True)
    assert st["bootstrap_seed"] == 21491 and st["n_blocks"] == len(d["counts" + tag])


def test_bootstrap_single_block_and_bad_counts():
    from kubomsd_b200 import kpm
    d = golden("statistics")
    v, se, _ = kpm.estimate_ratio(d["A"][:1], d["D"][:1], d["counts"][:1])
    assert se is None
    np.testing.assert_allclose(v, d["A"][0] / d["D"][0], rtol=1e-14)
    with pytest.raises(Exception, match="inconsistent statistical blocks"):
        kpm.estimate_ratio(d["A"], d["D"], np.r_[d["counts"][:-1], 0])
    with pytest.raises(Exception, match="must be \\(blocks,energy\\)"):
        kpm.estimate_ratio(d["A"], d["D"][:, :3], d["counts"])


# ------------------------------------------------------------ accuracy report
def test_moment_errors_resolve_a_planted_high_order_error():
    """An error planted at one high order shows in the per-order figure at
    its own scale, while the norm-wise figure (over mu_0) stays small."""
    from kubomsd_b200 import accuracy
    rng = np.random.default_rng(1)
    ref = rng.normal(size=(64, 4)) * np.exp(-np.arange(64) / 8.)[:, None]
    ref[0] = 1000.
    test = ref.copy()
    test[50] *= 1 + 1e-3
    r = accuracy.moment_errors(test, ref)
    assert r["order_of_max"] == 50
    assert abs(r["max_per_order"] - 1e-3) < 1e-9
    assert r["max_over_mu0"] < 1e-6


def test_stepwise_errors_mask_and_diffusion():
    from kubomsd_b200 import accuracy
    rng = np.random.default_rng(2)
    t = np.arange(6.)
    dos = rng.random((3, 9)) + .1
    msd = rng.random((3, 1, 6, 9)) + t[None, None, :, None]
    msd[:, :, 0] = 0.
    r0 = accuracy.stepwise_errors(dos, msd, dos, msd, t)
    assert r0["dos_max_rel_per_energy"] == 0. and r0["msd_max_rel_per_point"] == 0.
    pert = msd.copy()
    pert[:, :, 3, 4] *= 1 + 2e-4
    r = accuracy.stepwise_errors(dos, pert, dos, msd, t)
    assert abs(r["msd_max_rel_per_point"] - 2e-4) < 1e-9
    assert r["diffusion_max_rel_per_point"] > 0. and r["dos_normwise"] == 0.


# ------------------------------------------------------------ segmentation
@pytest.mark.parametrize("times,segment", [
    ([0., .5, 1., 2.5, 3.], 1.), ([0., 1., 2., 3.], 1.), ([0., .2, 5.], 2.), ([0., 3.], .5)])
def test_segment_nodes_cover_every_node_in_order(times, segment):
    """Every node is served by one segment; segments are contiguous from 0,
    each spans at most max(segment, the gap to its first node), and a node
    never lies beyond its segment's end (the reference's spectral.py:25-32)."""
    from kubomsd_b200.stochastic import _segment_nodes
    segs = _segment_nodes(np.asarray(times), segment)
    served = [t for _, _, nodes in segs for t in nodes]
    assert served == list(times)
    assert segs[0][0] == 0.
    for (a0, e0, _), (a1, _, _) in zip(segs, segs[1:]):
        assert a1 >= a0 and e0 <= times[-1] + 1e-14
    for a, e, nodes in segs:
        assert all(a - 1e-14 <= t <= e + 1e-14 for t in nodes)


# ------------------------------------------------------------ workspace gates
def test_sample_working_bytes_grow_with_batch_and_vac():
    from kubomsd_b200.stochastic import sample_working_bytes
    cfg = _cfg(include_vac=False)
    b1, b2 = (sample_working_bytes(cfg, 10000, "stepwise", b) for b in (1, 2))
    assert b2 > b1 > 16 * 10000 * 2 * 6
    vac = sample_working_bytes(_cfg(include_vac=True), 10000, "stepwise", 1)
    assert vac > b1
    assert sample_working_bytes(_cfg(include_vac=False), 10000, "spectral", 1) > b1


# ------------------------------------------------------------ serving stream
def test_poisson_stream_is_seeded_and_within_window():
    from kubomsd_b200.serving import poisson_stream
    models = {"a": None, "b": None}
    r1 = poisson_stream(20., 3., models, seed=5, msd_fraction=.25)
    r2 = poisson_stream(20., 3., models, seed=5, msd_fraction=.25)
    assert [(r.arrival, r.model, r.kind, r.n_moments, r.vectors) for r in r1] == \
           [(r.arrival, r.model, r.kind, r.n_moments, r.vectors) for r in r2]
    assert all(0 < r.arrival <= 3. for r in r1) and [r.rid for r in r1] == list(range(len(r1)))
    assert 30 <= len(r1) <= 95
    assert {r.kind for r in r1} <= {"dos", "msd"}
    assert all((r.times_fs is not None) == (r.kind == "msd") for r in r1)


def test_latency_summary_percentiles():
    from kubomsd_b200.serving import Result, latency_summary
    res = [Result(i, 0., float(i), float(i) + 1., None, "a", "dos", 0) for i in range(100)]
    s = latency_summary(res)
    assert s["requests"] == 100 and s["mean_service_s"] == 1.
    assert abs(s["p50_s"] - np.percentile(np.arange(100) + 1., 50)) < 1e-12
    assert latency_summary([])["p50_s"] is None


# ------------------------------------------------------------ bench sizing
def test_reference_arm_sample_rule():
    import bench
    assert bench.reference_sample_ly(2048, 1024, 3, 3) == 1024     # the default run: full lattice
    assert bench.reference_sample_ly(2048, 1024, 20, 5) == 256      # long runs: a quarter of the rows
    assert bench.reference_sample_ly(64, 64, 1000, 5) == 64         # small lattices stay whole
    assert bench.reference_sample_ly(2048, 4, 1000, 5) == 4


def test_series_row_bytes():
    import bench
    # complex64 [psi | phi] of 2 x 64 columns on a 4-wide ELL operator
    assert bench.series_row_bytes(128, 4, 4) == 5 * 128 * 8 + 4 * 8 + 2 * 4 * 4
    assert bench.series_row_bytes(64, 8, 4) == 5 * 64 * 16 + 4 * 12 + 2 * 4 * 8


# ------------------------------------------------------------ output grids
def test_output_grids_match_reference_bit_for_bit():
    """Time and energy grids from the reference's resolve_time_grid /
    resolve_output_grid (tests/golden/config.npz): identical bits, since every
    moment, propagation and MSD array is indexed by them."""
    from kubomsd_b200.config import resolve_output_grid, resolve_time_grid
    d = golden("config")
    for i, (tmax, dt) in enumerate(d["time_inputs"]):
        np.testing.assert_array_equal(resolve_time_grid(float(tmax), float(dt)), d[f"time_{i}"])
    for i, (a, b, n) in enumerate(d["energy_inputs"]):
        np.testing.assert_array_equal(resolve_output_grid(float(a), float(b), int(n)), d[f"energy_{i}"])


@pytest.mark.parametrize("call,message", [
    (lambda c: c.resolve_time_grid(-1., 1.), "invalid tmax/dt"),
    (lambda c: c.resolve_time_grid(1., 0.), "invalid tmax/dt"),
    (lambda c: c.resolve_time_grid(np.inf, 1.), "invalid tmax/dt"),
    (lambda c: c.resolve_output_grid(1., 1., 5), "require finite emin < emax"),
    (lambda c: c.resolve_output_grid(0., 1., 1), "require finite emin < emax"),
    (lambda c: c.grid([0., 1., 1.], "energy"), "energy must be a finite, strictly increasing"),
    (lambda c: c.grid([.5, 1.], "time", True), "time must start at zero"),
])
def test_grid_errors_match_reference_messages(call, message):
    from kubomsd_b200 import config
    with pytest.raises(Exception, match=message):
        call(config)
