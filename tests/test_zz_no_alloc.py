"""The allocation-free moments entry point against the allocating one.

`kmsd_engine_moments_noalloc` exists for callers that cannot allocate device
memory where they need moments: serving loops that must not stall other
streams on cudaMalloc's device synchronisation, frameworks that keep all
device memory in their own pool, code that must not fail with out-of-memory
mid-run.  Its workspace is a static 64 MiB device block inside the library.
Here it is called through the C ABI and compared with `kmsd_engine_moments`
on the same engine and input, in FP64 and in the mixed form, with both moment
methods.  It is called twice in a row: the second call starts from the scratch
contents the first one left behind.  Around those two calls the device's free
memory must not change: the output and the input are allocated, and one
warm-up call made (it may load the library's device code and with it the
static block), before the first reading.  A block too large for the static
scratch must be rejected, never allocated.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu
HALF = 9.2


def _noalloc(lib, eng, B, length, flags, torch, mu=None):
    from kubomsd_b200 import _abi
    if mu is None:
        mu = torch.full((length, B.shape[1]), np.nan, dtype=torch.float64, device="cuda")
    else:
        mu.fill_(np.nan)
    rc = lib.kmsd_engine_moments_noalloc(eng.handle, C.c_void_p(B.data_ptr()),
                                         C.cast(C.c_void_p(mu.data_ptr()), C.POINTER(C.c_double)), B.shape[1],
                                         length, 0., HALF, flags, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _abi.KMSD_OK, _abi.last_error(lib)
    torch.cuda.synchronize()
    return mu.cpu().numpy()


@pytest.mark.parametrize("doubling", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_moments_match_allocating_entry_point(cuda, precision, doubling):
    from kubomsd_b200 import _abi, kpm, lattices
    from tests.gpu_util import engine
    torch = cuda
    m = lattices.honeycomb(64, 32, seed=11)
    B = torch.from_numpy(kpm.random_phases(m.n, 5, range(12))).cuda()
    _, eng, _ = engine(m.H, m.S, velocity=m.velocity, precision=precision)
    # the allocating entry point (kmsd_engine_moments) on the same input
    want = eng.moments(B, 200, 0., HALF, doubling=doubling).cpu().numpy()
    lib = _abi.load()
    flags = _abi.KMSD_MOMENTS_DOUBLING if doubling else _abi.KMSD_MOMENTS_DIRECT
    mu = torch.empty((200, B.shape[1]), dtype=torch.float64, device="cuda")
    _noalloc(lib, eng, B, 200, flags, torch, mu)  # warm-up: may load the device code and the static block
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    got = []
    for call in range(2):
        got.append(_noalloc(lib, eng, B, 200, flags, torch, mu))
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before, f"device free memory changed by {free_before - free_after} bytes"
    for call, g in enumerate(got):
        assert np.isfinite(g).all()
        assert_rel(g, want, 1e-10, f"{precision} doubling={doubling} call {call}")


def test_noalloc_rejects_blocks_beyond_its_scratch(cuda):
    from kubomsd_b200 import _abi, lattices
    from tests.gpu_util import engine
    torch = cuda
    m = lattices.honeycomb(512, 256, seed=3, with_velocity=False)
    _, eng, _ = engine(m.H, m.S)
    B = torch.ones((m.n, 32), dtype=torch.complex128, device="cuda")  # 2 x 134 MB of recurrence buffers
    mu = torch.zeros((8, 32), dtype=torch.float64, device="cuda")
    lib = _abi.load()
    rc = lib.kmsd_engine_moments_noalloc(eng.handle, C.c_void_p(B.data_ptr()),
                                         C.cast(C.c_void_p(mu.data_ptr()), C.POINTER(C.c_double)), 32, 8, 0., HALF,
                                         0, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _abi.KMSD_EINVAL
    assert "scratch" in _abi.last_error(lib) and "64 MiB" in _abi.last_error(lib)
    assert bool((mu == 0).all())
