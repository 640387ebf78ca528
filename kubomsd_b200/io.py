"""Model input and results output in KuboMSD's formats.

* `load_model` reads `model.json` (`kubomsd-model-v1`) with matrices in NPZ
  (dense or CSR) or HDF5, applying the reference's unit factors and checks
  (src/kubo_msd/io/model.py:11-77).
* `ResultsWriter` stores transport blocks under the reference's dataset names
  and metadata layout (src/kubo_msd/io/results.py:20-112): `results.h5` +
  `metadata.json` when h5py is importable; otherwise the reference's own NPZ
  export schema (`results.npz` with schema_version, run_status,
  primary_estimator and metadata_json beside the datasets), which the
  reference's `read_results` accepts.
* `read_results` reads either form.
"""
from __future__ import annotations

import json
import os
from dataclasses import asdict, is_dataclass
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import scipy.sparse as sp

from .errors import BackendUnavailable, KuboMSDError, NumericalError
from .kpm import HBAR_EV_FS, hermitian
from .lattices import Model

HARTREE_EV = 27.211386245988
RYDBERG_EV = HARTREE_EV / 2
BOHR_A = 0.529177210903
REASONS = {"LOW_DOS": 1, "UNCERTAIN_TRACE": 2, "NO_SELECTED_STATES": 4, "TRUNCATION_UNVERIFIED": 8,
           "INTEGRATION_UNVERIFIED": 16, "INSUFFICIENT_BLOCKS": 32}


def _h5py():
    try:
        import h5py  # noqa: F401
        return h5py
    except ImportError:
        return None


def read_matrix(entry, root, n):
    required = {"path", "shape", "dtype", "storage", "index_base", "representation"}
    if not required <= entry.keys():
        raise KuboMSDError(f"matrix declaration missing {sorted(required - entry.keys())}")
    if (entry["shape"] != [n, n] or entry["index_base"] not in (0, 1) or entry["representation"] != "covariant"
            or entry["dtype"] not in ("float64", "complex128")):
        raise KuboMSDError("invalid matrix shape/index/representation/dtype")
    path = (root / entry["path"]).resolve()
    if not path.is_file():
        raise KuboMSDError(f"missing matrix: {path}")
    storage = entry["storage"]
    if path.suffix == ".npz":
        with np.load(path, allow_pickle=False) as f:
            if storage == "dense":
                A = np.array(f[entry.get("key", "matrix")])
            elif storage == "csr":
                shape = tuple(f["shape"])
                idx, ptr, base = f["indices"], f["indptr"], entry["index_base"]
                if (shape != (n, n) or idx.dtype.kind not in "iu" or ptr.dtype.kind not in "iu" or len(ptr) != n + 1
                        or ptr[0] != base or ptr[-1] - base != len(idx) or len(f["data"]) != len(idx)
                        or np.any(np.diff(ptr) < 0) or np.any(idx < base) or np.any(idx >= n + base)):
                    raise KuboMSDError("malformed CSR arrays")
                A = sp.csr_matrix((f["data"], idx - base, ptr - base), shape=shape)
            else:
                raise KuboMSDError("matrix storage must be dense/csr")
    elif path.suffix in (".h5", ".hdf5"):
        h5py = _h5py()
        if h5py is None:
            raise BackendUnavailable("HDF5 matrix input needs h5py, which is not installed")
        with h5py.File(path, "r") as f:
            if storage == "dense":
                A = np.array(f[entry.get("key", "matrix")])
            elif storage == "csr":
                g = f[entry.get("key", "matrix")]
                base = entry["index_base"]
                A = sp.csr_matrix((g["data"][:], g["indices"][:] - base, g["indptr"][:] - base),
                                  shape=tuple(g["shape"][:]))
                A.check_format(full_check=True)
            else:
                raise KuboMSDError("matrix storage must be dense/csr")
    else:
        raise KuboMSDError("matrix container must be NPZ/HDF5")
    if A.shape != (n, n) or str(A.dtype) != entry["dtype"]:
        raise KuboMSDError("matrix shape/dtype disagrees with declaration")
    return sp.csr_matrix(A, dtype=complex)


def load_model(path) -> Model:
    path = Path(path).resolve()
    if not path.is_file():
        raise KuboMSDError(f"missing model: {path}")
    d = json.loads(path.read_text())
    root = path.parent
    if d.get("format") != "kubomsd-model-v1":
        raise KuboMSDError("unknown input schema")
    for key in ("n_orbitals", "basis", "kpoint", "energy_unit", "length_unit", "orbital_order", "hamiltonian",
                "velocity_source"):
        if key not in d:
            raise KuboMSDError("missing model field " + key)
    n = d["n_orbitals"]
    order = d["orbital_order"]
    if not isinstance(n, int) or n < 1 or len(order) != n or len(set(map(str, order))) != n:
        raise KuboMSDError("invalid orbital count/order")
    if d["kpoint"] != [0, 0, 0]:
        raise KuboMSDError("v1 supports only one Gamma point")
    if d["basis"] not in ("orthogonal", "nonorthogonal"):
        raise KuboMSDError("basis must be explicit")
    ef = {"eV": 1., "hartree": HARTREE_EV, "rydberg": RYDBERG_EV}.get(d["energy_unit"])
    lf = {"angstrom": 1., "bohr": BOHR_A}.get(d["length_unit"])
    if ef is None or lf is None:
        raise KuboMSDError("unsupported energy/length units")
    H = hermitian(read_matrix(d["hamiltonian"], root, n) * ef, "Hamiltonian")
    if "overlap" in d:
        S = hermitian(read_matrix(d["overlap"], root, n), "overlap")
    elif d["basis"] == "orthogonal":
        S = sp.eye(n, dtype=complex, format="csr")
    else:
        raise KuboMSDError("nonorthogonal model requires overlap")
    if d["basis"] == "orthogonal" and sp.linalg.norm(S - sp.eye(n)) > 1e-12:
        raise KuboMSDError("orthogonal model supplied nonidentity S")
    source = d["velocity_source"]
    kind = source.get("type")
    velocity, position, composite = {}, {}, {}
    if kind == "matrix":
        factor = {"angstrom/fs": 1., "eV*angstrom": 1 / HBAR_EV_FS}.get(source.get("unit"))
        if factor is None:
            raise KuboMSDError("explicit physical velocity unit required")
        velocity = {a: hermitian(read_matrix(e, root, n) * factor, "velocity " + a)
                    for a, e in source["matrices"].items()}
    elif kind == "position":
        if "coordinates" in source:
            if d["basis"] != "orthogonal":
                raise KuboMSDError("atomic coordinates cannot replace nonorthogonal dipole matrices")
            r = np.asarray(source["coordinates"], float) * lf
            if r.shape != (n, 3) or not np.isfinite(r).all():
                raise KuboMSDError("invalid orbital positions")
            position = {a: sp.diags(r[:, k], format="csr") for k, a in enumerate("xyz")}
        else:
            position = {a: hermitian(read_matrix(e, root, n) * lf, "position " + a)
                        for a, e in source["matrices"].items()}
    elif kind == "composite":
        for a, parts in source["axes"].items():
            composite[a] = (read_matrix(parts["bond"], root, n) * ef * lf, read_matrix(parts["xbar"], root, n) * lf,
                            read_matrix(parts["delta"], root, n) * lf)
    else:
        raise KuboMSDError("unknown velocity source")
    slices = [tuple(s) for s in d.get("atom_slices", [])]
    return Model(H, S, velocity=velocity, position=position, composite=composite, atom_slices=slices,
                 description=str(path))


def save_model(model: Model, target, basis="orthogonal"):
    """Write model.json + NPZ CSR matrices (the reference's input schema)."""
    target = Path(target)
    target.mkdir(parents=True, exist_ok=True)

    def entry(name, matrix):
        p = target / (name + ".npz")
        A = sp.csr_matrix(matrix, dtype=np.complex128)
        np.savez(p, data=A.data, indices=A.indices.astype(np.int64), indptr=A.indptr.astype(np.int64),
                 shape=np.array(A.shape))
        return dict(path=p.name, shape=list(A.shape), dtype="complex128", storage="csr", index_base=0,
                    representation="covariant")

    doc = dict(format="kubomsd-model-v1", n_orbitals=model.n, basis=basis, kpoint=[0, 0, 0], energy_unit="eV",
               length_unit="angstrom", orbital_order=list(range(model.n)), hamiltonian=entry("H", model.H))
    if basis == "nonorthogonal":
        doc["overlap"] = entry("S", model.S)
    if model.velocity:
        doc["velocity_source"] = dict(type="matrix", unit="angstrom/fs",
                                      matrices={a: entry("V" + a, v) for a, v in model.velocity.items()})
    elif model.composite:
        doc["velocity_source"] = dict(type="composite", axes={a: dict(bond=entry("bond" + a, p[0]),
                                                                      xbar=entry("xbar" + a, p[1]),
                                                                      delta=entry("delta" + a, p[2]))
                                                              for a, p in model.composite.items()})
    if model.atom_slices:
        doc["atom_slices"] = [list(s) for s in model.atom_slices]
    path = target / "model.json"
    path.write_text(json.dumps(doc, indent=2) + "\n")
    return path


def json_safe(v):
    if is_dataclass(v):
        return json_safe(asdict(v))
    if isinstance(v, dict):
        return {str(k): json_safe(x) for k, x in v.items()}
    if isinstance(v, (list, tuple, np.ndarray)):
        return [json_safe(x) for x in v]
    if isinstance(v, np.generic):
        return json_safe(v.item())
    if isinstance(v, float) and not np.isfinite(v):
        return None
    if isinstance(v, Path):
        return str(v)
    if isinstance(v, SimpleNamespace):
        return json_safe(vars(v))
    return v


class ResultsWriter:
    """Time-block result store with explicit completion (io/results.py:20-112)."""

    def __init__(self, path, config):
        self.path = Path(path).resolve()
        self.path.mkdir(parents=True, exist_ok=False)
        self.cfg = config
        self.next = 0
        self.keys = None
        self.done = False
        self.data = {"energy_eV": np.asarray(config.energy_eV), "time_fs": np.asarray(config.time_fs),
                     "axes_vectors": np.asarray(config.axes_vectors)}
        self.h5 = _h5py()
        self.metadata = {"schema_version": "1.0", "run_status": "partial", "resolved_config": config.as_dict(),
                         "axis_order": "axis,time,energy; statistical sums: block,axis,time,energy",
                         "units": {"energy": "eV", "time": "fs", "msd": "angstrom^2", "diffusion": "angstrom^2/fs",
                                   "vac": "angstrom^2/fs^2", "dos": "states/eV/system"},
                         "spin_degeneracy_multiplier": 1, "reason_codes": dict(REASONS), "hbar_eV_fs": HBAR_EV_FS,
                         "container": "hdf5" if self.h5 else "npz (h5py not installed)"}
        self._save_meta()

    def _save_meta(self):
        temp = self.path / "metadata.json.tmp"
        temp.write_text(json.dumps(json_safe(self.metadata), ensure_ascii=False, indent=2, allow_nan=False) + "\n")
        os.replace(temp, self.path / "metadata.json")

    def __enter__(self):
        return self

    def __exit__(self, typ, value, tb):
        if not self.done:
            self.metadata["run_status"] = "failed" if typ else "partial"
            self.metadata["written_time_points"] = self.next
            if typ:
                self.metadata["failure"] = {"type": typ.__name__, "message": str(value)}
                if hasattr(value, "diagnostics"):
                    self.metadata["failure"]["numerics"] = value.diagnostics
            self._save_meta()

    def append(self, block):
        if self.done:
            raise KuboMSDError("cannot append finalized results")
        t = np.asarray(block.time_fs)
        end = block.start + len(t)
        if block.start != self.next or end > len(self.cfg.time_fs) or not np.array_equal(
                t, self.cfg.time_fs[block.start:end]):
            raise KuboMSDError("TransportBlock must contain contiguous configured times")
        if not len(t) or not block.arrays:
            raise KuboMSDError("empty TransportBlock")
        keys = set(block.arrays)
        if self.keys is not None and keys != self.keys:
            raise KuboMSDError("estimator schema changed during append")
        for key, value in block.arrays.items():
            a = np.asarray(value)
            axis = 2 if key.startswith("numerator_block_sums/") else 1
            if key not in self.data:
                shape = list(a.shape)
                shape[axis] = len(self.cfg.time_fs)
                self.data[key] = np.full(shape, np.nan if a.dtype.kind == "f" else 0, dtype=a.dtype)
            index = [slice(None)] * a.ndim
            index[axis] = slice(block.start, end)
            self.data[key][tuple(index)] = a
        if self.next and (block.static or block.metadata):
            raise KuboMSDError("static fields/metadata are allowed only in first block")
        for key, value in block.static.items():
            if key in self.data:
                raise KuboMSDError("duplicate static field " + key)
            self.data[key] = np.asarray(value)
        self.metadata.update(block.metadata)
        self.keys = keys
        self.next = end
        self.metadata["written_time_points"] = self.next
        self._save_meta()

    def _derive(self):
        primary = self.metadata["primary_estimator"]
        nt = len(self.cfg.time_fs)
        key = "diffusion_A2_per_fs/msd_gradient"
        if nt >= 2 and key not in self.data:
            edge = 2 if nt > 2 else 1
            self.data[key] = .5 * np.gradient(self.data["msd_A2/" + primary], self.cfg.time_fs, axis=1,
                                              edge_order=edge)
            num = self.data.get("numerator_msd_A2/" + primary)
            if num is not None:
                self.data["numerator_diffusion_A2_per_fs/msd_gradient"] = .5 * np.gradient(
                    num, self.cfg.time_fs, axis=1, edge_order=edge)
            for prefix in ("valid/", "reason_code/"):
                if prefix + primary in self.data:
                    self.data[prefix + "msd_gradient"] = self.data[prefix + primary].copy()
            self.metadata["msd_gradient"] = {"source": primary, "edge_order": edge,
                                             "time_array": "actual output time_fs"}
        dp = self.metadata.get("primary_diffusion_estimator", primary)
        aliases = {}
        for quantity, unit, est in (("msd", "A2", primary), ("diffusion", "A2_per_fs", dp)):
            k = f"{quantity}_{unit}/{est}"
            if k not in self.data:
                continue
            data = self.data[k]
            for i, axis in enumerate(self.cfg.axes):
                if axis in ("x", "y", "z"):
                    alias = f"{quantity}_{axis}_{unit}"
                    self.data[alias] = data[i].copy()
                    aliases[alias] = k
            self.data[f"{quantity}_direction_average_{unit}"] = np.mean(data, axis=0)
        self.metadata["legacy_aliases"] = aliases
        self.metadata["direction_average"] = ("arithmetic mean over declared orthonormal directions; no volume "
                                              "normalization")

    def finalize(self, summary):
        if self.done or self.next != len(self.cfg.time_fs) or summary.get("run_status") != "complete":
            raise KuboMSDError("cannot mark incomplete computation complete")
        if "dos_states_per_eV" not in self.data or "primary_estimator" not in self.metadata:
            raise KuboMSDError("required result metadata missing")
        self._derive()
        self.metadata["summary"] = json_safe(summary)
        self.metadata["run_status"] = "complete"
        meta = json.dumps(json_safe(self.metadata), allow_nan=False)
        if self.h5 is not None:
            tmp = self.path / "results.partial.h5"
            with self.h5.File(tmp, "w") as f:
                f.attrs["schema_version"] = "1.0"
                for k, v in self.data.items():
                    f.create_dataset(k, data=v)
                f.attrs["run_status"] = "complete"
                f.attrs["metadata_json"] = meta
            os.replace(tmp, self.path / "results.h5")
        if self.h5 is None or getattr(self.cfg, "output_npz", False):
            arrays = dict(self.data)
            arrays["schema_version"] = np.array("1.0")
            arrays["run_status"] = np.array("complete")
            arrays["primary_estimator"] = np.array(self.metadata["primary_estimator"])
            arrays["metadata_json"] = np.array(meta)
            np.savez_compressed(self.path / "results.npz", **arrays)
        self._save_meta()
        self.done = True


def read_results(path, allow_partial=False):
    p = Path(path)
    if p.is_dir():
        metadata = json.loads((p / "metadata.json").read_text())
        p = p / ("results.h5" if (p / "results.h5").exists() else "results.npz")
    else:
        metadata = None
    arrays = {}
    if p.suffix == ".npz":
        with np.load(p, allow_pickle=False) as f:
            if "schema_version" not in f or str(f["schema_version"]) != "1.0" or "metadata_json" not in f:
                raise KuboMSDError("unversioned legacy NPZ cannot establish full spectrum/kernel metadata")
            metadata = json.loads(str(f["metadata_json"]))
            arrays = {k: np.array(f[k]) for k in f.files if k != "metadata_json"}
    else:
        h5py = _h5py()
        if h5py is None:
            raise BackendUnavailable("reading results.h5 needs h5py")
        with h5py.File(p, "r") as f:
            if f.attrs.get("schema_version") != "1.0":
                raise KuboMSDError("unknown result schema")
            if metadata is None:
                metadata = json.loads(f.attrs.get("metadata_json", "{}"))
                metadata["run_status"] = f.attrs["run_status"]
            f.visititems(lambda name, obj: arrays.update({name: obj[()]}) if isinstance(obj, h5py.Dataset) else None)
    if metadata.get("run_status") != "complete" and not allow_partial:
        raise KuboMSDError("result is failed/partial; use allow_partial explicitly")
    return {"metadata": metadata, "arrays": arrays}


__all__ = ["load_model", "save_model", "ResultsWriter", "read_results", "NumericalError"]
