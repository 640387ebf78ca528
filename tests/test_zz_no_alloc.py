"""The allocation-free moments entry point against the allocating one.

`kmsd_engine_moments_noalloc` exists for callers that cannot allocate device
memory where they need moments: serving loops that must not stall other
streams on cudaMalloc's device synchronisation, frameworks that keep all
device memory in their own pool, code that must not fail with out-of-memory
mid-run.  Its workspace is a static 64 MiB device block inside the library.
Here it is called through the C ABI and compared with `kmsd_engine_moments`
on the same engine and input, in FP64 and in the mixed form, with both moment
methods.  It is called twice in a row: the second call starts from the scratch
contents the first one left behind.  A block too large for the static scratch
must be rejected, never allocated.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import assert_rel

pytestmark = pytest.mark.gpu
HALF = 9.2


def _noalloc(lib, eng, B, length, flags, torch):
    from kubomsd_b200 import _abi
    mu = torch.full((length, B.shape[1]), np.nan, dtype=torch.float64, device="cuda")
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
    for call in range(2):
        got = _noalloc(lib, eng, B, 200, flags, torch)
        assert np.isfinite(got).all()
        assert_rel(got, want, 1e-10, f"{precision} doubling={doubling} call {call}")


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
