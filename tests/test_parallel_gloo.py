"""Sample-parallel host logic over two gloo ranks on the CPU: round-robin block
ownership, ordered gather of float64 block sums to root, and stage failure
agreement (a rank that raises makes every rank raise, none waits)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kubomsd_b200.parallel import ParallelContext, owned_blocks


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ctx = ParallelContext(distributed=True)
        nblocks = 5
        ids = owned_blocks(9 * 2 - 1, 2, ctx.rank, ctx.size)  # 17 samples, blocks of 2 -> 9 blocks
        local = np.stack([np.full((3, 4), float(i)) for i in ids])
        if mode == "gather":
            full = ctx.gather_blocks(local, ids, 9)
            if ctx.root:
                out.put(("gather", full.tolist()))
            b = ctx.broadcast("root-bounds" if ctx.root else None)
            out.put(("bcast", rank, b))
        elif mode == "fail":
            def action():
                if rank == 1:
                    raise ValueError("injected failure on rank 1")
                return "ok"
            try:
                ctx.stage("injected", action)
                out.put(("nofail", rank))
            except Exception as exc:  # noqa: BLE001
                out.put(("failed", rank, str(exc)))
        del nblocks
    finally:
        dist.destroy_process_group()


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    items = []
    while not q.empty():
        items.append(q.get())
    return items


def test_owned_blocks_cover_each_block_once():
    blocks = sorted(b for r in range(3) for b in owned_blocks(20, 3, r, 3))
    assert blocks == list(range(7))
    with pytest.raises(ValueError):
        owned_blocks(0, 1, 0, 1)


def test_gather_orders_blocks_globally_on_root():
    items = _run("gather")
    gathered = [i for i in items if i[0] == "gather"]
    assert len(gathered) == 1
    full = np.array(gathered[0][1])
    assert full.shape == (9, 3, 4)
    np.testing.assert_array_equal(full[:, 0, 0], np.arange(9))
    assert sorted(i[1] for i in items if i[0] == "bcast") == [0, 1]
    assert all(i[2] == "root-bounds" for i in items if i[0] == "bcast")


def test_stage_failure_is_agreed_by_all_ranks():
    items = _run("fail")
    failed = [i for i in items if i[0] == "failed"]
    assert sorted(i[1] for i in failed) == [0, 1]
    assert all("injected failure on rank 1" in i[2] for i in failed)
