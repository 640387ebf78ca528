"""SHA-256 digest of a canonical complex CSR matrix (generator drift check for
the golden fixtures; the same digest make_golden.py stores)."""
import hashlib

import numpy as np
import scipy.sparse as sp


def digest(A):
    A = sp.csr_matrix(A, dtype=np.complex128)
    A.sum_duplicates()
    A.sort_indices()
    h = hashlib.sha256()
    for v in (A.indptr.astype(np.int64), A.indices.astype(np.int64), A.data):
        h.update(np.ascontiguousarray(v).tobytes())
    return h.hexdigest()
