"""The C-ABI library loads and exports every function include/kmsd.h declares;
host-side argument validation mirrors the reference (no GPU needed)."""
import ctypes as C

import numpy as np
import pytest

from kubomsd_b200 import _abi


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    declared = _abi.header_functions()
    assert len(declared) >= 20
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing
    assert set(declared) == set(_abi.SIGNATURES), set(declared) ^ set(_abi.SIGNATURES)


def test_build_info_names_the_architecture():
    import json
    info = json.loads(_abi.load().kmsd_build_info().decode())
    assert info["architecture"] == "sm_100a"


@pytest.mark.parametrize("indptr,indices,vals,message", [
    ([1, 1, 2], [0, 1], [1., 2.], "invalid CSR row pointers"),
    ([0, 2, 1], [0, 1], [1., 2.], "nonmonotone CSR row pointers"),
    ([0, 1, 2], [0, 2], [1., 2.], "invalid CSR index or nonfinite entry"),
    ([0, 1, 2], [0, 1], [1., np.nan], "invalid CSR index or nonfinite entry"),
])
def test_csr_validation_matches_reference_messages(indptr, indices, vals, message):
    lib = _abi.load()
    n = len(indptr) - 1
    p = np.asarray(indptr, np.int64)
    i = np.asarray(indices + [0] * 4, np.int64)
    v = np.asarray(vals + [0.] * 4, np.float64)
    h = C.c_void_p()
    rc = lib.kmsd_csr_create(n, p.ctypes.data_as(C.POINTER(C.c_int64)), i.ctypes.data_as(C.POINTER(C.c_int64)),
                             v.ctypes.data_as(C.POINTER(C.c_double)), None, C.byref(h))
    assert rc == _abi.KMSD_EINVAL
    assert message in _abi.last_error(lib)


def test_missing_library_is_actionable(tmp_path):
    from kubomsd_b200.errors import BackendUnavailable
    with pytest.raises(BackendUnavailable, match="build"):
        _abi.load(tmp_path / "absent.so")
