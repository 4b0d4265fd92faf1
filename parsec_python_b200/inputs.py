"""Inputs: element table, pseudopotential tables, input files, unit handling.

Reads the same input formats as PARSEC.py's rsdft_input.py
(``.in``/``.inp`` with ``$system``/``$settings`` sections, ``.json``,
``.txt`` atom lines, ``.dat``; load_atomic_data_from_file :282-468) and
converts coordinates and length overrides to bohr the same way
(convert_units_to_bohr :582-632: files default to angstrom).  The element
table keeps the reference's columns (Element, AtomicNumber, Z, Zvalue, h, r,
R; load_elements :23-31).
"""
from __future__ import annotations

import json
from pathlib import Path
from typing import Any

import numpy as np

from .models import A0_ANG, InputData, SolverSettings

DATA = Path(__file__).resolve().parent / "data"


class ElementTable:
    """Rows of the element table keyed by symbol, in file order."""

    COLUMNS = ("Element", "AtomicNumber", "Z", "Zvalue", "h", "r", "R")

    def __init__(self, path: Path | None = None):
        self.rows: dict[str, dict[str, Any]] = {}
        for order, line in enumerate((path or DATA / "elements.csv").read_text().splitlines()):
            f = line.split(",")
            if len(f) < 7 or not f[0].strip():
                continue
            self.rows[f[0]] = {"Element": f[0], "order": order, "AtomicNumber": int(f[1]), "Z": int(f[2]),
                               "Zvalue": float(f[3]), "h": float(f[4]), "r": float(f[5]), "R": float(f[6])}

    def __contains__(self, sym: str) -> bool:
        return sym in self.rows

    def __getitem__(self, sym: str) -> dict[str, Any]:
        if sym not in self.rows:
            raise KeyError(f"element {sym!r} is not in the element table (first 18 elements only)")
        return self.rows[sym]

    def __len__(self) -> int:
        return len(self.rows)

    def order(self, sym: str) -> int:
        return self.rows[sym]["order"]


def load_elements(base_dir: str | Path | None = None):
    """(element table, number of elements), as rsdft_input.load_elements."""
    table = ElementTable(Path(base_dir) / "elements.csv" if base_dir else None)
    return table, len(table)


_TABLES: dict[str, np.ndarray] | None = None


def pseudo_tables() -> dict[str, np.ndarray]:
    """Radial tables per element: columns radius, charge, hartree, pot_P,
    pot_S, wfn_P, wfn_S (V_ion/splineData.py:35)."""
    global _TABLES
    if _TABLES is None:
        with np.load(DATA / "pseudo_tables.npz") as z:
            _TABLES = {k: np.ascontiguousarray(z[k], dtype=np.float64) for k in z.files}
    return _TABLES


def parse_atom_lines(lines: list[str]):
    """``TYPE x y z`` lines grouped by species in first-appearance order."""
    groups: dict[str, list[list[float]]] = {}
    for raw in lines:
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        parts = line.split()
        if len(parts) != 4:
            raise ValueError("Atom line must be: TYPE x y z")
        try:
            xyz = [float(v) for v in parts[1:]]
        except ValueError as exc:
            raise ValueError("Could not parse coordinates; must be numeric.") from exc
        groups.setdefault(parts[0], []).append(xyz)
    atoms = [{"typ": t, "coord": np.array(c, dtype=float)} for t, c in groups.items()]
    return atoms, [a["coord"].shape[0] for a in atoms]


def _non_empty(d: dict[str, Any]) -> dict[str, Any]:
    return {k: v for k, v in d.items() if v is not None and not (isinstance(v, str) and not v.strip())}


def load_atomic_data_from_file(file_name: str) -> InputData:
    path = Path(file_name).expanduser()
    if not path.exists():
        raise FileNotFoundError(f"File not found: {file_name}")
    ext = path.suffix.lower()
    atoms: list[dict[str, Any]] = []
    z_charge = 0.0
    density_method = "sad"
    ml_file = None
    overrides: dict[str, Any] = {}
    unit = None
    if ext in (".in", ".inp"):
        section = None
        atom_lines, setting_lines = [], []
        for raw in path.read_text().splitlines():
            line = raw.strip()
            if not line or line.startswith("#"):
                continue
            tok = line.lower()
            if tok in ("$system", "$settings"):
                name = tok[1:]
                section = None if section == name else name
                continue
            (atom_lines if section == "system" else setting_lines if section == "settings" else []).append(line)
        atoms, _ = parse_atom_lines(atom_lines)
        for entry in setting_lines:
            if "=" not in entry:
                continue
            key, val = (s.strip() for s in entry.split("=", 1))
            if not val:
                continue
            kl = key.lower()
            if kl in ("z_charge", "charge"):
                try:
                    z_charge = float(val)
                except ValueError:
                    print(f'Warning: could not parse Z_charge "{val}", using default 0.')
            elif kl in ("density_method", "density"):
                density_method = val.lower()
            elif kl in ("ml_file_path", "density_file"):
                ml_file = str((path.parent / Path(val).expanduser()) if not Path(val).is_absolute() else val)
            elif kl == "unit":
                unit = val
            else:
                overrides[key] = val
        overrides = _non_empty(overrides)
    elif ext == ".json":
        data = json.loads(path.read_text())
        block = data.get("atoms") or data.get("Atoms")
        if not block:
            raise ValueError('JSON file missing "atoms" list.')
        if isinstance(block, str):
            atoms, _ = parse_atom_lines(block.strip().splitlines())
        elif isinstance(block[0], str):
            atoms, _ = parse_atom_lines(block)
        else:
            for entry in block:
                typ = entry.get("typ") or entry.get("type") or entry.get("element")
                coords = entry.get("coord") or entry.get("coords") or entry.get("coordinates")
                if typ is None or coords is None:
                    raise ValueError("Each atom entry must have typ and coord/coords.")
                atoms.append({"typ": str(typ), "coord": np.asarray(coords, dtype=float).reshape(-1, 3)})
        try:
            z_charge = float(data.get("Z_charge", data.get("charge", 0.0)))
        except (TypeError, ValueError):
            z_charge = 0.0
        dm = data.get("density_method", density_method)
        density_method = dm.lower() if isinstance(dm, str) else "sad"
        overrides = data.get("settings", data.get("params", {})) or {}
        if not isinstance(overrides, dict):
            overrides = {}
        unit = overrides.get("unit", unit)
        ml = data.get("ml_file_path") or data.get("density_file")
        if ml:
            cand = Path(str(ml)).expanduser()
            ml_file = str(cand if cand.is_absolute() else path.parent / cand)
        for key in ("nev", "grid_spacing", "h", "sphere_radius", "radius", "grid_npy_path", "grid_poscar_path",
                    "recenter_atoms"):
            if key in data and key not in overrides:
                overrides[key] = data[key]
        overrides = _non_empty(overrides)
    elif ext == ".txt":
        atoms, _ = parse_atom_lines(path.read_text().splitlines())
    elif ext == ".dat":
        lines = path.read_text().splitlines()
        count = int(lines[0].strip())
        for i in range(count):
            typ = lines[1 + 2 * i].strip()
            vals = np.array([float(v) for v in lines[2 + 2 * i].split()], dtype=float)
            if vals.size % 3:
                raise ValueError("Coordinate count in .dat must be divisible by 3.")
            atoms.append({"typ": typ, "coord": vals.reshape(-1, 3)})
    else:
        raise ValueError("File extension not recognized (supported: .dat, .json, .txt, .in, .inp).")
    if density_method not in ("sad", "ml", "sad_ml_grid"):
        density_method = "sad"
    if unit:
        overrides["unit"] = unit
    return InputData(atoms=atoms, n_atom=[a["coord"].shape[0] for a in atoms], z_charge=z_charge,
                     density_method=density_method, ml_file_path=ml_file, settings_overrides=overrides,
                     input_file_path=str(path.resolve()))


def convert_units_to_bohr(atoms, overrides, input_file_path):
    """Coordinates and length overrides to bohr; files default to angstrom."""
    ov = dict(overrides or {})
    unit = ov.get("unit") or ("ang" if input_file_path is not None else "bohr")
    unit = str(unit).lower()
    if unit in ("ang", "angstrom", "a"):
        factor = 1.0 / A0_ANG
    elif unit in ("bohr", "au", "a.u."):
        factor = 1.0
    else:
        factor = 1.0 / A0_ANG if input_file_path is not None else 1.0
    out = [{"typ": a["typ"], "coord": np.asarray(a["coord"], dtype=float).copy() * factor} for a in atoms]
    for key in ("grid_spacing", "h", "sphere_radius", "radius"):
        if key in ov:
            try:
                ov[key] = float(ov[key]) * factor
            except (TypeError, ValueError):
                pass
    ov.pop("unit", None)
    return out, ov, unit


def resolve_optional_path(raw_path, label: str, input_file_path: str | None = None) -> str | None:
    """First existing candidate of a possibly relative path: as given
    (absolute), under the working directory, next to the package, next to the
    input file (rsdft_input.py:505-529)."""
    if not raw_path:
        return None
    raw = Path(str(raw_path)).expanduser()
    cands = [raw] if raw.is_absolute() else [Path.cwd() / raw, Path(__file__).resolve().parent / raw]
    if not raw.is_absolute() and input_file_path:
        cands.append(Path(input_file_path).resolve().parent / raw)
    for c in cands:
        if c.exists():
            return str(c.resolve())
    print(f"Warning: {label} {raw_path} not found. Tried: {[str(c) for c in cands]}")
    return None


def read_poscar_cube_length(poscar_path: str) -> float:
    """Mean length (angstrom) of the three scaled lattice vectors of a POSCAR
    file (rsdft_input.py:532-557)."""
    lines = [ln.strip() for ln in Path(poscar_path).read_text().splitlines() if ln.strip()]
    if len(lines) < 5:
        raise ValueError("Incomplete POSCAR file for grid size.")
    scale = float(lines[1].split()[0])
    lengths = []
    for i in range(2, 5):
        parts = lines[i].split()
        if len(parts) < 3:
            raise ValueError(f'Invalid lattice vector line: "{lines[i]}"')
        v = [float(parts[0]) * scale, float(parts[1]) * scale, float(parts[2]) * scale]
        lengths.append(np.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    return sum(lengths) / 3.0


def load_grid_data_from_files(grid_npy: str, grid_poscar: str) -> dict[str, Any]:
    """Grid of an ML density file: shape from the .npy (read without loading
    it), spacing L / nx and radius L / 2 from the POSCAR cell, in bohr
    (rsdft_input.py:560-579)."""
    density = np.load(grid_npy, mmap_mode="r")
    if density.ndim != 3:
        raise ValueError("Grid .npy file must be a 3D array.")
    nx, ny, nz = density.shape
    if nx <= 0 or ny <= 0 or nz <= 0:
        raise ValueError("Invalid grid shape in .npy file.")
    length = read_poscar_cube_length(grid_poscar)
    return {"nx": int(nx), "ny": int(ny), "nz": int(nz), "h": length / float(nx) / A0_ANG,
            "radius": length / 2.0 / A0_ANG}


def prepare_input_data(settings: SolverSettings, input_path: str) -> InputData:
    """Parse an input file, resolve its auxiliary files, convert to bohr and,
    for the ML density modes, read the grid from the density and POSCAR files
    (rsdft_input.py:636-701)."""
    data = load_atomic_data_from_file(input_path)
    if not data.atoms:
        raise SystemExit("No atoms loaded, exiting RSDFT.")
    ov = dict(data.settings_overrides or {})
    data.grid_npy_path = ov.pop("grid_npy_path", None) or ov.pop("grid_npy", None)
    data.grid_poscar_path = ov.pop("grid_poscar_path", None) or ov.pop("grid_poscar", None)
    data.settings_overrides = ov
    data.ml_file_path = resolve_optional_path(data.ml_file_path, "ML density file", data.input_file_path)
    data.grid_npy_path = resolve_optional_path(data.grid_npy_path, "Grid npy file", data.input_file_path)
    data.grid_poscar_path = resolve_optional_path(data.grid_poscar_path, "Grid POSCAR file", data.input_file_path)
    if data.density_method in ("ml", "sad_ml_grid") and data.ml_file_path is None:
        raise SystemExit("Density method requires ML .npy file but no ml_file_path was provided or found. "
                         "Add ml_file_path to the input file.")
    data.atoms, data.settings_overrides, data.unit_used = convert_units_to_bohr(
        data.atoms, data.settings_overrides, data.input_file_path)
    data.grid_mode = "ml" if data.density_method in ("ml", "sad_ml_grid") else "default"
    if data.grid_mode == "ml":
        if data.grid_npy_path is None:
            data.grid_npy_path = data.ml_file_path
        if data.grid_poscar_path is None:
            raise SystemExit("Grid POSCAR file is required to set grid structure.")
        data.grid_data = load_grid_data_from_files(data.grid_npy_path, data.grid_poscar_path)
    return data


def has_diagmeth_override(overrides) -> bool:
    """rsdft_input.py:39-41."""
    return any(str(k).lower() == "diagmeth" for k in (overrides or {}))
