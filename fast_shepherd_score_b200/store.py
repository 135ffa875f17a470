"""ProfileStore: the screening library on disk, in shepherd_score's store format (version 1).

A store is a directory holding ``manifest.json`` and ``shard_NNNNN.npz`` files (five-digit,
zero-padded shard index).  The manifest records ``version`` (1), ``num_surf_points``,
``modes``, ``schema`` (seven booleans, below), ``dtype`` ("float16" or "float32", the on-disk
type of every real-valued column), ``shard_size``, ``pre_centered``, ``n_total`` and
``shards``: a list of ``{"name", "n", "start"}``.  A shard holds the columns of :data:`COLUMNS`
for its ``n`` molecules, concatenated, each ragged column indexed by an int64 offset table of
n + 1 entries.  Stores written here are read by shepherd_score and the other way round
(shepherd_score/screen.py:317-606 is the other implementation of the format).

This implementation is column-oriented: the writer appends each molecule's arrays to one list
per column (no per-molecule objects are kept), a shard is flushed by concatenating the
columns, and the reader hands the columns to the device loader as they are, so a float16 shard
is uploaded in float16 (``layout.CloudSet`` / the server widen it on the device).  The manifest
is replaced atomically after every flushed shard, so an interrupted writer leaves a readable
store of the shards written so far.
"""
from __future__ import annotations

import json
import os
import re
from dataclasses import dataclass
from types import SimpleNamespace
from typing import Callable, Dict, Iterator, List, Optional, Sequence, Tuple

import numpy as np

from .modes import CANONICAL_MODES, canonical

FORMAT_VERSION = 1
MANIFEST_NAME = "manifest.json"
_SHARD_FILE = re.compile(r"shard_\d{5}\.npz")

# schema flag -> the modes that need it (vol needs only atom_pos, which every store keeps;
# vol_pharm -- shape + directional pharmacophores, a mode of this package -- needs "pharm")
SCHEMA_FLAGS: Dict[str, frozenset] = {
    "surf": frozenset({"surf", "surf_esp", "vol_and_surf_esp"}),
    "surf_esp": frozenset({"surf_esp", "vol_and_surf_esp"}),
    "charges": frozenset({"vol_esp", "vol_and_surf_esp"}),
    "with_H": frozenset({"vol_and_surf_esp"}),
    "radii": frozenset({"vol_and_surf_esp"}),
    "centers_w_H": frozenset({"vol_and_surf_esp"}),
    "pharm": frozenset({"pharm", "vol_color", "vol_pharm"}),
}
STORE_MODES = tuple(CANONICAL_MODES) + ("vol_pharm",)


def schema_for(modes: Sequence[str]) -> dict:
    """The schema flags a store needs to serve ``modes`` (legacy names accepted)."""
    wanted = {canonical(m) for m in modes}
    unknown = wanted - set(STORE_MODES)
    if unknown:
        raise ValueError(f"unknown modes {sorted(unknown)}; valid: {list(STORE_MODES)}")
    return {flag: bool(users & wanted) for flag, users in SCHEMA_FLAGS.items()}


def schema_supports(schema: dict, mode: str) -> bool:
    """True when a store with ``schema`` holds every array ``mode`` reads."""
    mode = canonical(mode)
    if mode not in STORE_MODES:
        return False
    return all(schema.get(flag, False) for flag, users in SCHEMA_FLAGS.items() if mode in users)


@dataclass(frozen=True)
class Column:
    """One shard array.  ``index`` names the offset table that splits it per molecule:
    "mol" (one row per molecule), "atom" (``atom_off``), "all" (``all_off``, the atoms with
    hydrogens), "pharm" (``pharm_off``) or "surf" (a dense (n, num_surf_points, ...) block).
    ``kind`` is "real" (stored in the store's dtype), "int32", "int64" or "id"."""
    name: str
    index: str
    kind: str
    width: int                       # trailing dimension (0: scalar per row)
    needed: Callable[[dict], bool]   # from the schema flags


def _charges_index(sch):
    return "all" if sch["with_H"] else "atom"


COLUMNS: Tuple[Column, ...] = (
    Column("ids", "mol", "id", 0, lambda s: True),
    Column("atom_pos", "atom", "real", 3, lambda s: True),
    Column("surf_pos", "surf", "real", 3, lambda s: s["surf"]),
    Column("surf_esp", "surf", "real", 0, lambda s: s["surf_esp"]),
    Column("charges", "?", "real", 0, lambda s: s["charges"]),
    Column("nonH", "atom", "int64", 0, lambda s: s["charges"] and s["with_H"]),
    Column("radii", "all", "real", 0, lambda s: s["charges"] and s["with_H"] and s["radii"]),
    Column("cwh", "all", "real", 3, lambda s: s["charges"] and s["with_H"] and s["centers_w_H"]),
    Column("pharm_types", "pharm", "int32", 0, lambda s: s["pharm"]),
    Column("pharm_ancs", "pharm", "real", 3, lambda s: s["pharm"]),
    Column("pharm_vecs", "pharm", "real", 3, lambda s: s["pharm"]),
)
OFFSETS = {"atom": "atom_off", "all": "all_off", "pharm": "pharm_off", "heavy": "heavy_off"}
# Optional pair of a charged store: when some molecule's heavy-atom Gaussian centres (the
# heavy rows of the all-atom positions, or ``atom_pos_noH``) differ from its ``atom_pos``, the
# shard also keeps ``xyz_noH`` (those centres, one row per heavy charge) with ``heavy_off``.
_HEAVY = Column("xyz_noH", "heavy", "real", 3, lambda s: s["charges"])
# columns that hold positions: shifted with the molecule when the store is pre-centred
_POSITIONS = ("atom_pos", "surf_pos", "cwh", "pharm_ancs", "xyz_noH")

# where each column comes from on a Molecule / MoleculeProfile-like object
_ATTRS = {"atom_pos": "atom_pos", "surf_pos": "surf_pos", "surf_esp": "surf_esp",
          "charges": "partial_charges", "nonH": "_nonH_atoms_idx", "radii": "radii",
          "cwh": "centers_w_H", "pharm_types": "pharm_types", "pharm_ancs": "pharm_ancs",
          "pharm_vecs": "pharm_vecs"}
# keyword names of add_arrays (the profile attribute names) for each column
_KEYWORDS = {"charges": "partial_charges", "nonH": "nonH_atoms_idx", "cwh": "centers_w_H"}


def _resolve_index(col: Column, sch: dict) -> str:
    return _charges_index(sch) if col.index == "?" else col.index


def _offsets(lengths) -> np.ndarray:
    out = np.zeros(len(lengths) + 1, np.int64)
    np.cumsum(lengths, out=out[1:])
    return out


def _write_json_atomic(path: str, obj: dict) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(obj, fh, indent=2)
    os.replace(tmp, path)


class ProfileStore:
    """A store directory opened for writing (:meth:`create`) or reading (:meth:`open`)."""

    MANIFEST = MANIFEST_NAME
    VERSION = FORMAT_VERSION

    def __init__(self, path: str, manifest: dict, writable: bool):
        self.path = path
        self.manifest = manifest
        self.writable = writable
        self._columns = [c for c in COLUMNS if c.needed(manifest["schema"])]
        self._pending: Dict[str, list] = {c.name: [] for c in self._columns + [_HEAVY]}
        self._pending_n = 0

    # ---- creation / writing -------------------------------------------------------------
    @classmethod
    def create(cls, path, *, num_surf_points: int, modes: Sequence[str], dtype: str = "float16",
               shard_size: int = 100_000, pre_centered: bool = True,
               overwrite: bool = False) -> "ProfileStore":
        """Start a new store at ``path`` for ``modes``; only the columns those modes read are
        kept.  ``dtype`` is the on-disk type of the real-valued columns; ``pre_centered``
        shifts every molecule to the mean of its ``atom_pos`` at write time.  An existing
        store in ``path`` raises ``FileExistsError`` unless ``overwrite`` (which deletes only
        the store's own manifest and shard files)."""
        if dtype not in ("float16", "float32"):
            raise ValueError("dtype must be 'float16' or 'float32'")
        if int(shard_size) < 1:
            raise ValueError("shard_size must be >= 1")
        schema = schema_for(modes)
        os.makedirs(path, exist_ok=True)
        manifest_path = os.path.join(path, MANIFEST_NAME)
        if os.path.exists(manifest_path):
            if not overwrite:
                raise FileExistsError(f"{manifest_path} already exists; pass overwrite=True "
                                      "to replace it")
            for name in os.listdir(path):
                if name == MANIFEST_NAME or _SHARD_FILE.fullmatch(name):
                    os.remove(os.path.join(path, name))
        manifest = {"version": FORMAT_VERSION, "num_surf_points": int(num_surf_points),
                    "modes": list(modes), "schema": schema, "dtype": dtype,
                    "shard_size": int(shard_size), "pre_centered": bool(pre_centered),
                    "n_total": 0, "shards": []}
        store = cls(path, manifest, writable=True)
        _write_json_atomic(manifest_path, manifest)
        return store

    def _need_writable(self):
        if not self.writable:
            raise RuntimeError("store is open for reading")

    def add(self, molecule, id=None) -> None:
        """Append one molecule given as an object with the profile attributes (``atom_pos``,
        ``surf_pos``, ``surf_esp``, ``partial_charges``, ``radii``, ``pharm_types`` /
        ``pharm_ancs`` / ``pharm_vecs``, ``_nonH_atoms_idx``, and the all-atom positions as
        ``centers_w_H`` or an RDKit ``mol``), e.g. a shepherd_score ``Molecule`` or
        ``MoleculeProfile``.  ``id`` defaults to the molecule's ``id`` attribute, else its
        position in the store."""
        sch = self.manifest["schema"]
        arrays = {}
        for col in self._columns:
            if col.name == "ids":
                continue
            value = getattr(molecule, _ATTRS[col.name], None)
            if value is None and col.name == "cwh" and getattr(molecule, "mol", None) is not None:
                value = molecule.mol.GetConformer().GetPositions()
            arrays[_KEYWORDS.get(col.name, col.name)] = value
        if sch["charges"]:
            arrays["atom_pos_noH"] = getattr(molecule, "atom_pos_noH", None)
        heavy = getattr(molecule, "_nonH_atoms_idx", None)
        charges = arrays.get("partial_charges")
        if (sch["charges"] and not sch["with_H"] and charges is not None and heavy is not None
                and len(charges) != len(molecule.atom_pos)):
            # a molecule with hydrogens: the store keeps the heavy atoms' charges
            arrays["partial_charges"] = np.asarray(charges)[np.asarray(heavy)]
        if id is None:
            id = getattr(molecule, "id", None)
        self.add_arrays(id=id, **arrays)

    add_profile = add

    def add_arrays(self, *, atom_pos, surf_pos=None, surf_esp=None, partial_charges=None,
                   pharm_types=None, pharm_ancs=None, pharm_vecs=None, centers_w_H=None,
                   radii=None, nonH_atoms_idx=None, atom_pos_noH=None, id=None) -> None:
        """Append one molecule given as arrays.  A store of heavy-atom charges (vol_esp)
        takes ``partial_charges`` per row of ``atom_pos``; a store with hydrogens
        (vol_and_surf_esp) takes ``partial_charges``, ``radii`` and ``centers_w_H`` for all
        atoms, and ``nonH_atoms_idx`` (default: the first len(atom_pos) atoms are the heavy
        ones).  ``atom_pos_noH`` gives the heavy-atom Gaussian centres of a charged store when
        they are not the rows of ``atom_pos`` (kept as ``xyz_noH``)."""
        self._need_writable()
        sch = self.manifest["schema"]
        given = {"atom_pos": atom_pos, "surf_pos": surf_pos, "surf_esp": surf_esp,
                 "charges": partial_charges, "pharm_types": pharm_types,
                 "pharm_ancs": pharm_ancs, "pharm_vecs": pharm_vecs, "cwh": centers_w_H,
                 "radii": radii, "nonH": nonH_atoms_idx}
        rows = {}
        atoms = np.asarray(atom_pos, np.float32).reshape(-1, 3)
        for col in self._columns:
            if col.name == "ids":
                continue
            value = given[col.name]
            if value is None and col.name == "nonH":
                value = np.arange(len(atoms), dtype=np.int64)
            if value is None:
                raise ValueError(f"this store ({', '.join(self.modes)}) needs "
                                 f"{_KEYWORDS.get(col.name, col.name)} for every molecule")
            dt = {"real": np.float32, "int32": np.int32, "int64": np.int64}[col.kind]
            arr = np.asarray(value, dt)
            arr = arr.reshape(-1, col.width) if col.width else arr.reshape(-1)
            rows[col.name] = arr
        rows["atom_pos"] = atoms
        if "surf_pos" in rows and len(rows["surf_pos"]) != self.num_surf_points:
            raise ValueError(f"surf_pos has {len(rows['surf_pos'])} points; the store keeps "
                             f"{self.num_surf_points} per molecule")
        if "surf_esp" in rows and len(rows["surf_esp"]) != self.num_surf_points:
            raise ValueError("surf_esp must have one value per surface point")
        if sch["charges"] and not sch["with_H"] and len(rows["charges"]) != len(atoms):
            raise ValueError("partial_charges must have one value per row of atom_pos")
        if sch["pharm"] and not (len(rows["pharm_types"]) == len(rows["pharm_ancs"])
                                 == len(rows["pharm_vecs"])):
            raise ValueError("pharm_types, pharm_ancs and pharm_vecs differ in length")
        if sch["charges"]:
            # the heavy charges' Gaussian centres: given, or the heavy rows of the all-atom
            # positions; stored only when they are not atom_pos itself
            if atom_pos_noH is not None:
                centres = np.asarray(atom_pos_noH, np.float32).reshape(-1, 3)
            elif sch["with_H"] and "cwh" in rows:
                centres = rows["cwh"][rows["nonH"]]
            else:
                centres = atoms
            if centres.shape != atoms.shape or not np.array_equal(centres, atoms):
                rows["xyz_noH"] = centres
        if self.manifest["pre_centered"]:
            com = atoms.mean(0)
            for name in _POSITIONS:
                if name in rows:
                    rows[name] = rows[name] - com
        if sch["charges"]:
            # one entry per molecule (None: the centres are its atom_pos), resolved at flush
            self._pending["xyz_noH"].append(rows.pop("xyz_noH", None))
        for name, arr in rows.items():
            self._pending[name].append(arr)
        self._pending["ids"].append(len(self) + self._pending_n if id is None else id)
        self._pending_n += 1
        if self._pending_n >= self.manifest["shard_size"]:
            self.flush()

    def flush(self) -> None:
        """Write the buffered molecules as the next shard (no-op when none are buffered)."""
        self._need_writable()
        if not self._pending_n:
            return
        sch = self.manifest["schema"]
        real = np.float16 if self.manifest["dtype"] == "float16" else np.float32
        out = {}
        for col in self._columns:
            parts = self._pending[col.name]
            index = _resolve_index(col, sch)
            if col.name == "ids":
                out["ids"] = np.asarray(parts)
                continue
            if index in OFFSETS and OFFSETS[index] not in out:
                out[OFFSETS[index]] = _offsets([len(a) for a in parts])
            joined = np.stack(parts) if index == "surf" else np.concatenate(parts)
            out[col.name] = joined.astype(real) if col.kind == "real" else joined
        heavy = self._pending["xyz_noH"]
        if any(h is not None for h in heavy):
            n_heavy = self._pending["nonH" if sch["with_H"] else "charges"]
            out["heavy_off"] = _offsets([len(a) for a in n_heavy])
            atoms = self._pending["atom_pos"]
            out["xyz_noH"] = np.concatenate(
                [atoms[i] if h is None else h for i, h in enumerate(heavy)]).astype(real)
        shard_idx = len(self.manifest["shards"])
        name = f"shard_{shard_idx:05d}.npz"
        np.savez(os.path.join(self.path, name), **out)
        start = int(self.manifest["n_total"])
        self.manifest["shards"].append({"name": name, "n": self._pending_n, "start": start})
        self.manifest["n_total"] = start + self._pending_n
        self._pending = {c.name: [] for c in self._columns + [_HEAVY]}
        self._pending_n = 0
        _write_json_atomic(os.path.join(self.path, MANIFEST_NAME), self.manifest)

    def close(self) -> None:
        if self.writable:
            self.flush()
            self.writable = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- reading -------------------------------------------------------------------------
    @classmethod
    def open(cls, path) -> "ProfileStore":
        with open(os.path.join(path, MANIFEST_NAME)) as fh:
            manifest = json.load(fh)
        if manifest.get("version") != FORMAT_VERSION:
            raise ValueError(f"ProfileStore at {path!r} has on-disk format version "
                             f"{manifest.get('version')!r}; this reader reads "
                             f"{FORMAT_VERSION} (rebuild the store)")
        return cls(path, manifest, writable=False)

    def __len__(self) -> int:
        return int(self.manifest["n_total"])

    @property
    def num_surf_points(self) -> int:
        return int(self.manifest["num_surf_points"])

    @property
    def modes(self) -> tuple:
        return tuple(self.manifest["modes"])

    @property
    def schema(self) -> dict:
        return dict(self.manifest["schema"])

    @property
    def dtype(self) -> str:
        return self.manifest["dtype"]

    @property
    def pre_centered(self) -> bool:
        return bool(self.manifest["pre_centered"])

    @property
    def num_shards(self) -> int:
        return len(self.manifest["shards"])

    def supports(self, mode: str) -> bool:
        return schema_supports(self.manifest["schema"], mode)

    def read_shard(self, idx: int, columns: Optional[Sequence[str]] = None) -> tuple:
        """(shard record, {column: array}) of shard ``idx``, every array in its stored dtype.
        ``columns`` limits what is read from the file (offset tables always come along)."""
        meta = self.manifest["shards"][idx]
        with np.load(os.path.join(self.path, meta["name"])) as data:
            keep = data.files if columns is None else [
                k for k in data.files if k in set(columns) or k.endswith("_off")]
            return meta, {k: data[k] for k in keep}

    def iter_shards(self) -> Iterator[List[SimpleNamespace]]:
        """Each shard as a list of per-molecule profiles (attribute access as
        ``MoleculeProfile``: ``atom_pos``, ``surf_pos``, ``partial_charges``, ...)."""
        for i in range(self.num_shards):
            yield self.read_profiles(i)

    def read_profiles(self, idx: int) -> List[SimpleNamespace]:
        meta, cols = self.read_shard(idx)
        sch = self.manifest["schema"]
        n = int(meta["n"])
        per = {name: [None] * n for name in cols if name not in OFFSETS.values()}
        for col in self._columns:
            if col.name not in cols:
                continue
            arr = cols[col.name]
            index = _resolve_index(col, sch)
            if index in ("mol", "surf"):
                for i in range(n):
                    per[col.name][i] = arr[i]
            else:
                off = cols[OFFSETS[index]]
                for i in range(n):
                    per[col.name][i] = arr[off[i]:off[i + 1]]
        profiles = []
        for i in range(n):
            fields = {_ATTRS.get(name, name): per[name][i] for name in per if name != "ids"}
            rid = per["ids"][i]
            fields["id"] = rid.item() if isinstance(rid, np.generic) else rid
            profiles.append(SimpleNamespace(**fields))
        return profiles
