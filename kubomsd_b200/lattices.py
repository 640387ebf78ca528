"""Seeded synthetic tight-binding models for the transport workloads.

Every model is returned as host SciPy CSR matrices in the reference's
`kubomsd-model-v1` conventions (energies in eV, lengths in angstrom,
covariant velocity in angstrom/fs):

* square_lattice  — orthogonal 2D square lattice, nearest-neighbour hopping,
  Anderson on-site disorder (64 x 64, t = -2.7 eV, W = 0.5 eV is the
  CPU-runnable reference case);
* honeycomb       — orthogonal honeycomb lattice (2048 x 1024 cells x 2 =
  4,194,304 sites, t = -2.7 eV, W = 1 eV is the precision-form case);
* diamond_sp3     — nonorthogonal sp3 model on the diamond lattice with 4x4
  atom blocks of H and S on first and second neighbours decaying as
  exp(-r / 1.5 A), S = I + s O scaled to a target condition number.

The velocity of the orthogonal lattices is the explicit covariant matrix
v_ij = i H_ij (x_j - x_i) / hbar with minimum-image bond vectors (the
reference's `velocity_source.type = "matrix"`); the nonorthogonal model uses
the composite bond / xbar / delta form (kind 2).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

HBAR_EV_FS = 0.6582119569509067


@dataclass
class Model:
    H: sp.csr_matrix
    S: sp.csr_matrix
    velocity: dict = field(default_factory=dict)
    position: dict = field(default_factory=dict)
    composite: dict = field(default_factory=dict)
    atom_slices: list = field(default_factory=list)
    description: str = ""

    @property
    def n(self) -> int:
        return self.H.shape[0]


def _csr(rows, cols, vals, n, dtype):
    A = sp.csr_matrix((np.asarray(vals, dtype), (np.asarray(rows), np.asarray(cols))), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A


def _bond_velocity(rows, cols, hop, dx, n):
    """v_ij = i H_ij dx_ij / hbar for the bonds (rows, cols)."""
    return _csr(rows, cols, 1j * hop * dx / HBAR_EV_FS, n, np.complex128)


def square_lattice(L: int = 64, t: float = -2.7, W: float = .5, seed: int = 20261203, a: float = 1.) -> Model:
    """L x L periodic square lattice, site i = x L + y."""
    n = L * L
    rng = np.random.default_rng(seed)
    onsite = rng.uniform(-W, W, n)
    x, y = np.divmod(np.arange(n), L)
    rows, cols, dxs = [], [], []
    for dxc, dyc in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        j = ((x + dxc) % L) * L + (y + dyc) % L
        rows.append(np.arange(n))
        cols.append(j)
        dxs.append(np.full(n, dxc * a))
    rows, cols, dxs = map(np.concatenate, (rows, cols, dxs))
    hop = np.full(rows.shape, t)
    H = _csr(np.r_[np.arange(n), rows], np.r_[np.arange(n), cols], np.r_[onsite, hop], n, np.float64)
    V = _bond_velocity(rows, cols, hop, dxs, n)
    S = sp.identity(n, format="csr", dtype=np.float64)
    return Model(H, S, velocity={"x": V}, description=f"square {L}x{L}, t={t} eV, W={W} eV, seed {seed}")


def honeycomb(Lx: int = 2048, Ly: int = 1024, t: float = -2.7, W: float = 1., seed: int = 20261203,
              acc: float = 1.42, with_velocity: bool = True) -> Model:
    """Periodic honeycomb lattice, site index 2 (x Ly + y) + s (s = 0: A, 1: B).

    Lattice vectors a1 = acc (3/2, sqrt3/2), a2 = acc (3/2, -sqrt3/2); B sits at
    A + (acc, 0).  Each A couples to B of cells (x, y), (x-1, y), (x, y-1).
    """
    cells = Lx * Ly
    n = 2 * cells
    rng = np.random.default_rng(seed)
    onsite = rng.uniform(-W, W, n)
    cx, cy = np.divmod(np.arange(cells, dtype=np.int64), Ly)
    A = 2 * (cx * Ly + cy)
    bonds = (
        (2 * (cx * Ly + cy) + 1, acc),                               # same cell
        (2 * (((cx - 1) % Lx) * Ly + cy) + 1, -acc / 2),             # cell x-1
        (2 * (cx * Ly + (cy - 1) % Ly) + 1, -acc / 2),               # cell y-1
    )
    rows, cols, dxs = [], [], []
    for B, dx in bonds:
        rows += [A, B]
        cols += [B, A]
        dxs += [np.full(cells, dx), np.full(cells, -dx)]
    rows, cols, dxs = map(np.concatenate, (rows, cols, dxs))
    hop = np.full(rows.shape, t)
    diag = np.arange(n, dtype=np.int64)
    H = _csr(np.r_[diag, rows], np.r_[diag, cols], np.r_[onsite, hop], n, np.float64)
    V = _bond_velocity(rows, cols, hop, dxs, n) if with_velocity else None
    S = sp.identity(n, format="csr", dtype=np.float64)
    return Model(H, S, velocity={"x": V} if with_velocity else {},
                 description=f"honeycomb {Lx}x{Ly}x2, t={t} eV, W={W} eV, seed {seed}")


def diamond_sp3(cells: int = 10, a0: float = 3.567, decay: float = 1.5, kappa: float = 50., W: float = 0.,
                seed: int = 20261203, scale_hint: float | None = None) -> Model:
    """Diamond lattice, cells^3 conventional cells x 8 atoms, 4 orbitals/atom.

    H: on-site diag(eps_s, eps_p, eps_p, eps_p) + disorder U[-W/2, W/2]
    (per orbital), random symmetric 4x4 off-site blocks on first (a0 sqrt3/4)
    and second (a0/sqrt2) neighbours, scaled by exp(-r/decay).  S = I + s O,
    O a random symmetric block pattern with the same decay; s is bisected so
    that lambda_max(S) / lambda_min(S) ~ kappa.  Velocity: composite
    bond / xbar / delta per axis with minimum-image bond vectors.
    """
    rng = np.random.default_rng(seed)
    basis = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                      [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    grid = np.stack(np.meshgrid(*(np.arange(cells),) * 3, indexing="ij"), -1).reshape(-1, 3)
    frac = (grid[:, None, :] + basis[None, :, :]).reshape(-1, 3)  # in units of a0
    natoms = len(frac)
    box = cells * a0
    pos = frac * a0
    n = 4 * natoms
    d1, d2 = a0 * np.sqrt(3) / 4, a0 / np.sqrt(2)
    # neighbour search on the fractional grid (periodic): candidate offsets
    from scipy.spatial import cKDTree
    tree = cKDTree(pos, boxsize=box)
    pairs = tree.query_pairs(d2 * 1.05, output_type="ndarray")
    delta = pos[pairs[:, 1]] - pos[pairs[:, 0]]
    delta -= box * np.round(delta / box)
    dist = np.linalg.norm(delta, axis=1)
    first = np.abs(dist - d1) < 1e-6
    second = np.abs(dist - d2) < 1e-6
    keep = first | second
    pairs, delta, dist = pairs[keep], delta[keep], dist[keep]
    npair = len(pairs)
    hblk = rng.normal(size=(npair, 4, 4)) * np.exp(-dist / decay)[:, None, None]
    oblk = rng.normal(size=(npair, 4, 4)) * np.exp(-dist / decay)[:, None, None]
    eps = np.array([-5., 1.5, 1.5, 1.5])
    onsite = np.tile(eps, natoms) + rng.uniform(-W / 2, W / 2, n) if W else np.tile(eps, natoms)
    ii, jj = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
    rows = (4 * pairs[:, 0, None, None] + ii[None]).ravel()
    cols = (4 * pairs[:, 1, None, None] + jj[None]).ravel()
    dvec = np.repeat(delta, 16, axis=0)

    def sym(blocks, diag_vals):
        v = blocks.ravel()
        return _csr(np.r_[np.arange(n), rows, cols], np.r_[np.arange(n), cols, rows], np.r_[diag_vals, v, v],
                    n, np.float64)

    H = sym(hblk, onsite)
    O = sym(oblk, np.zeros(n))

    # lambda(S) = 1 + s lambda(O): kappa (1 + s lmin) = 1 + s lmax fixes s.
    if scale_hint is not None:
        s = scale_hint
    else:
        from scipy.sparse.linalg import eigsh
        v0 = np.random.default_rng(seed + 1).normal(size=n)
        lmax = float(eigsh(O, k=1, which="LA", return_eigenvectors=False, tol=1e-8, v0=v0)[0])
        lmin = float(eigsh(O, k=1, which="SA", return_eigenvectors=False, tol=1e-8, v0=v0)[0])
        s = (kappa - 1.) / (lmax - kappa * lmin)
    S = (sp.identity(n, format="csr") + s * O).tocsr()
    S.sort_indices()
    # composite velocity (kind 2) per axis: bond = H_ij d_ij, xbar = S_ij d_ij / 2,
    # delta = -S_ij d_ij / 2 with d the minimum-image bond vector (zero on site).
    Hc, Sc = H.tocoo(), S.tocoo()
    comp = {}
    for ax, name in enumerate("xyz"):
        def bondvec(M):
            d = pos[M.col // 4, ax] - pos[M.row // 4, ax]
            return d - box * np.round(d / box)
        dh, ds = bondvec(Hc), bondvec(Sc)
        bond = _csr(Hc.row, Hc.col, Hc.data * dh, n, np.complex128)
        xbar = _csr(Sc.row, Sc.col, Sc.data * ds / 2, n, np.complex128)
        dlt = _csr(Sc.row, Sc.col, -Sc.data * ds / 2, n, np.complex128)
        comp[name] = (bond, xbar, dlt)
    slices = [(4 * i, 4 * i + 4) for i in range(natoms)]
    return Model(H, S, composite=comp, atom_slices=slices,
                 description=f"diamond sp3 {cells}^3 cells, {natoms} atoms, s={s:.4g}, seed {seed}")
