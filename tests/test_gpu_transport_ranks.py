"""Distributed transport equals serial transport.

Two ranks (gloo process group, host-side exchange only) share cuda:0 and run
iter_stochastic_blocks on the same model and configuration; their statistics
blocks are owned round robin and gathered to rank 0, which normalises once.
The arrays on rank 0 must equal a serial run's at rtol 2e-9, as the
reference's MPI suite requires of serial and parallel runs
(tests/mpi/test_transport_mpi.py:56-90).  No kernel of one rank waits on the
other: the ranks only meet in host collectives between device calls.
"""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _config(method, distribution):
    from kubomsd_b200.config import RunConfig
    return RunConfig(energy_eV=np.linspace(-9, 9, 19), time_fs=[0., 1., 2., 3.], axes=("x",),
                     spectral_bounds=(-11.5, 11.5), n_moments=64, nsamples=8, sample_batch=2, statistics_block=2,
                     include_vac=False, stochastic_method=method, seed=515, integration_dt_fs=.05,
                     transport_distribution=distribution)


def _run(method, parallel=None):
    from kubomsd_b200 import lattices
    from kubomsd_b200.operators import build_operators
    from kubomsd_b200.stochastic import iter_stochastic_blocks
    m = lattices.square_lattice(16, seed=99)
    cfg = _config(method, "serial" if parallel is None else "torch")
    ops = build_operators(m, cfg)
    blocks = list(iter_stochastic_blocks(ops, cfg, method, parallel=parallel,
                                         bounds_report={"bounds": cfg.spectral_bounds}))
    if blocks and blocks[0] is None:
        return None
    out = {}
    for blk in blocks:
        for k, v in {**blk.static, **blk.arrays}.items():
            out[k] = np.asarray(v)
    return out


def _worker(rank, world, port, method, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from kubomsd_b200.parallel import ParallelContext
        ctx = ParallelContext(distributed=True)
        out = _run(method, ctx)
        if rank == 0:
            q.put({k: v for k, v in out.items()})
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("method", ["stepwise", "spectral"])
def test_two_ranks_equal_serial(cuda, method):
    import torch.multiprocessing as mp
    serial = _run(method)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, method, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=600)
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    arrays = [k for k in serial if serial[k].dtype.kind == "f"]
    assert arrays and set(arrays) <= set(got)
    assert "numerator_block_sums/msd_A2/" + ("commutator" if method == "stepwise" else "vac_integral") in arrays
    for k in arrays:
        np.testing.assert_allclose(got[k], serial[k], rtol=2e-9, atol=0, equal_nan=True, err_msg=k)
    for k in serial:
        if serial[k].dtype.kind in "biu":
            np.testing.assert_array_equal(got[k], serial[k], err_msg=k)
