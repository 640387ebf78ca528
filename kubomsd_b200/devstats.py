"""Device-resident statistics and sampling of the stochastic driver.

Block sums of the DOS and of the transport numerators stay in device memory
while the sample batches run; the energy projection of moments and the
paired block bootstrap run as library kernels (kmsd_project_moments,
kmsd_bootstrap_ratio in include/kmsd.h), so the only device-to-host copies of
a transport run are the normalised results at the end.

The bootstrap draws its resampling weights on the host exactly as the
reference does (NumPy default_rng(21491), 256 resamples of the block indices;
src/kubo_msd/observables/statistics.py:5-23), so the resamples are the same
ones; only the sums over blocks and resamples run on the device.
"""
from __future__ import annotations

import numpy as np

from . import _abi, kpm
from .errors import KuboMSDError

_G_CACHE: dict = {}


def _torch():
    import torch
    return torch


def _ptr(t):
    import ctypes as C
    return C.c_void_p(t.data_ptr())


def _stream(torch):
    import ctypes as C
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def reconstruction_matrix(energies, bounds, n_moments):
    """The Jackson reconstruction matrix G (ne, M) on the device, cached."""
    torch = _torch()
    key = (tuple(np.asarray(energies, float).tolist()), tuple(bounds), int(n_moments),
           torch.cuda.current_device())
    G = _G_CACHE.get(key)
    if G is None:
        G = torch.from_numpy(np.ascontiguousarray(kpm.reconstruction_matrix(energies, bounds, n_moments))).cuda()
        if len(_G_CACHE) > 16:
            _G_CACHE.clear()
        _G_CACHE[key] = G
    return G


def project(mu, G):
    """(G mu)^T of device moments mu (M, b) as a device tensor (b, ne)."""
    torch = _torch()
    lib = _abi.require_library()
    mu = mu.contiguous()
    M, b = mu.shape
    ne = G.shape[0]
    if G.shape[1] != M:
        raise KuboMSDError("reconstruction matrix and moments disagree")
    out = torch.empty((b, ne), dtype=torch.float64, device=mu.device)
    rc = lib.kmsd_project_moments(_ptr(mu), M, b, _ptr(G), ne, _ptr(out), _stream(torch))
    if rc != _abi.KMSD_OK:
        raise KuboMSDError(_abi.last_error(lib))
    return out


def bootstrap_weights(nblocks, n_resamples=256, seed=21491):
    """Counts of each block in each resample, drawn as the reference draws them."""
    rng = np.random.default_rng(seed)
    indices = rng.integers(nblocks, size=(n_resamples, nblocks))
    weights = np.zeros((n_resamples, nblocks))
    for j, row in enumerate(indices):
        weights[j] = np.bincount(row, minlength=nblocks)
    return weights


def estimate_ratio(block_numerators, block_dos, counts, n_resamples=256):
    """kpm.estimate_ratio with device block sums: returns device tensors
    (value, stderr or None) and the reference's status dict."""
    torch = _torch()
    lib = _abi.require_library()
    A = block_numerators.to(torch.float64).contiguous()
    D = block_dos.to(torch.float64)
    counts = np.asarray(counts, int)
    nb = len(counts)
    if A.shape[0] != nb or D.shape[0] != nb or np.any(counts <= 0):
        raise KuboMSDError("inconsistent statistical blocks/counts")
    ne = A.shape[-1]
    if D.ndim != 2 or D.shape[-1] != ne:
        if tuple(D.shape) == (nb, 1):
            D = D.expand(nb, ne)
        else:
            raise KuboMSDError("statistical denominator must be (blocks,energy)")
    D = D.contiguous()
    P = int(np.prod(A.shape[1:]))
    value = torch.empty(A.shape[1:], dtype=torch.float64, device=A.device)
    status = {"method": "paired block bootstrap of sums", "n_blocks": nb, "counts": counts.tolist(),
              "reliable_interval": nb >= 8, "bootstrap_seed": 21491, "n_resamples": n_resamples,
              "input_accumulation": "sum; actual unequal counts retained", "device": True}
    if nb < 2:
        rc = lib.kmsd_bootstrap_ratio(_ptr(A), _ptr(D), nb, P, ne, None, 0, _ptr(value), None, _stream(torch))
        if rc != _abi.KMSD_OK:
            raise KuboMSDError(_abi.last_error(lib))
        return value, None, status
    w = torch.from_numpy(bootstrap_weights(nb, n_resamples)).to(A.device)
    stderr = torch.empty_like(value)
    rc = lib.kmsd_bootstrap_ratio(_ptr(A), _ptr(D), nb, P, ne, _ptr(w), n_resamples, _ptr(value), _ptr(stderr),
                                  _stream(torch))
    if rc != _abi.KMSD_OK:
        raise KuboMSDError(_abi.last_error(lib))
    return value, stderr, status


def random_phases(n, seed, sample_ids):
    """The reference sampler's phases exp(2 pi i u), u from NumPy's
    Generator(PCG64(SeedSequence([seed, id]))).random(n) (metric/sampling.py:
    8-9), generated on the device (kmsd_random_phases) as an (n, b)
    complex128 tensor.  The seeding runs here; the draws are bit-identical to
    NumPy's, the phases equal to a few ulp."""
    torch = _torch()
    lib = _abi.require_library()
    ids = list(sample_ids)
    st = np.zeros((len(ids), 4), np.uint64)
    mask = (1 << 64) - 1
    for j, i in enumerate(ids):
        s = np.random.PCG64(np.random.SeedSequence([int(seed), int(i)])).state["state"]
        st[j] = (s["state"] & mask, s["state"] >> 64, s["inc"] & mask, s["inc"] >> 64)
    dst = torch.from_numpy(st.view(np.int64)).cuda()
    out = torch.empty((n, len(ids)), dtype=torch.complex128, device="cuda")
    rc = lib.kmsd_random_phases(int(n), len(ids), _ptr(dst), _ptr(out), _stream(torch))
    if rc != _abi.KMSD_OK:
        raise KuboMSDError(_abi.last_error(lib))
    return out
