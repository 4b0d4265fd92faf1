"""Problem setup between input parsing and the SCF: grid spacing, number of
states, cube domain, recentring and output paths.

Same rules as PARSEC.py's rsdft_setup.py: h = smallest tabulated spacing
unless overridden, nev = max(16, round(0.7*Z + 0.5)) unless overridden
(calculate_grid_spacing :19-83); nx = 2*ceil((int(2R/h)+1)/2), radius
0.5*h*(nx-1), cube nx = ny = nz (estimate_radius_and_grid :86-150); atoms
recentred on their centroid for SAD runs (recenter_atoms :153-160); outputs
next to the input file (build_output_paths :215-249).
"""
from __future__ import annotations

import os
from copy import deepcopy
from typing import Any

import numpy as np

from .models import A0_ANG, InputData, PreparedSystem, RunPaths, SolverSettings


def calculate_grid_spacing(atoms, elem, n_atom, z_charge, h_override=None, nev_override=None, grid_data=None):
    """With grid_data (an ML grid) h is the file grid's spacing and an h
    override is ignored (rsdft_setup.py:40-63)."""
    zelec = 0.0
    hmin = 100.0 if grid_data is None else grid_data["h"]
    for species, count in zip(atoms, n_atom):
        row = elem[species["typ"]]
        if grid_data is None:
            hmin = min(hmin, row["h"])
        zelec += row["Z"] * count
    ztest = zelec - z_charge
    if ztest < 0:
        raise SystemExit("Problem with charge state. Negative number of electrons.")
    h = hmin
    if grid_data is not None:
        if h_override is not None:
            print("Warning: grid spacing override ignored when using ML grid.")
    elif h_override is not None:
        try:
            h = float(h_override)
        except (TypeError, ValueError):
            print("Warning: invalid grid spacing override, using auto value.")
    nev = max(16, round(0.7 * zelec + 0.5))
    if nev_override is not None:
        try:
            nev = max(1, int(nev_override))
        except (TypeError, ValueError):
            print("Warning: invalid nev override, using auto value.")
    return h, nev, zelec, ztest


def cube_for_radius(radius: float, h: float) -> dict[str, Any]:
    nx = int(2 * radius / h) + 1
    nx = 2 * ((nx + 1) // 2)
    return {"radius": 0.5 * h * (nx - 1), "nx": nx, "ny": nx, "nz": nx, "h": h}


def estimate_radius_and_grid(atoms, elem, h, radius_override=None):
    rmax = 0.0
    for species in atoms:
        rsize = elem[species["typ"]]["r"]
        xyz = np.asarray(species["coord"], dtype=float)
        for a in range(xyz.shape[0]):
            rmax = max(rmax, np.sqrt(xyz[a, 0] ** 2 + xyz[a, 1] ** 2 + xyz[a, 2] ** 2) + rsize)
    domain = cube_for_radius(rmax, h)
    if radius_override is not None:
        try:
            domain = cube_for_radius(float(radius_override), h)
        except (TypeError, ValueError):
            print("Warning: invalid radius override, keeping auto radius.")
    return domain, len(atoms)


def recenter_atoms(atoms):
    out = deepcopy(atoms)
    center = np.mean(np.vstack([a["coord"] for a in out]), axis=0)
    for a in out:
        a["coord"] -= center
    return out


def formula(atoms, n_atom, elem) -> str:
    counts: dict[str, int] = {}
    for a, c in zip(atoms, n_atom):
        counts[a["typ"].strip()] = counts.get(a["typ"].strip(), 0) + int(c)
    if not counts:
        return "system"
    syms = sorted(counts, key=lambda s: (elem.order(s) if s in elem else 10 ** 9, s))
    return "".join(f"{s}{counts[s]}" if counts[s] != 1 else s for s in syms)


def _fmt(v: float) -> str:
    s = f"{v:.6f}".rstrip("0").rstrip(".")
    return (s or "0").replace(".", "p")


def build_output_paths(inp: InputData, settings: SolverSettings, elem, domain) -> RunPaths:
    if inp.input_file_path:
        base = os.path.splitext(os.path.basename(inp.input_file_path))[0]
        out_dir = os.path.dirname(inp.input_file_path) or "."
    else:
        base = (f"{formula(inp.atoms, inp.n_atom, elem)}_{inp.density_method}_diagmeth{settings.diagmeth}_"
                f"{_fmt(domain['radius'] * A0_ANG)}A_{_fmt(domain['h'] * A0_ANG)}A")
        out_dir = os.path.join(".", base)
    stem = os.path.join(out_dir, base)
    return RunPaths(output_file=stem + ".out", wfn_file=stem + "_wfn.dat", initial_density_base=stem + "_init_rho",
                    converged_density_base=stem + "_conv_rho")


def prepare_system(inp: InputData, settings: SolverSettings, elem, n_elements: int | None = None) -> PreparedSystem:
    ov = inp.settings_overrides
    ml_grid = inp.grid_mode == "ml"
    h, nev, zelec, ztest = calculate_grid_spacing(inp.atoms, elem, inp.n_atom, inp.z_charge,
                                                  ov.get("grid_spacing", ov.get("h")), ov.get("nev"),
                                                  inp.grid_data if ml_grid else None)
    atoms = inp.atoms
    if inp.density_method == "sad" and not ml_grid and settings.recenter_atoms:
        atoms = recenter_atoms(inp.atoms)
    if ml_grid:
        # rsdft_setup.py:106-117: the file grid as it is (atoms in its cell frame)
        if ov.get("sphere_radius", ov.get("radius")) is not None:
            print("Warning: radius override ignored when using ML grid.")
        g = inp.grid_data
        domain, n_types = {"radius": g["radius"], "nx": g["nx"], "ny": g["ny"], "nz": g["nz"], "h": h}, len(atoms)
    else:
        domain, n_types = estimate_radius_and_grid(atoms, elem, h, ov.get("sphere_radius", ov.get("radius")))
    prepared = InputData(atoms=atoms, n_atom=list(inp.n_atom), z_charge=inp.z_charge,
                         density_method=inp.density_method, ml_file_path=inp.ml_file_path,
                         settings_overrides=dict(ov), input_file_path=inp.input_file_path,
                         grid_npy_path=inp.grid_npy_path, grid_poscar_path=inp.grid_poscar_path,
                         unit_used=inp.unit_used, grid_mode=inp.grid_mode, grid_data=deepcopy(inp.grid_data))
    paths = build_output_paths(prepared, settings, elem, domain)
    return PreparedSystem(input_data=prepared, settings=settings, domain=domain, h=h, nev=nev, zelec=zelec,
                          ztest=ztest, n_types=n_types, paths=paths)


def system_from_atoms(atoms, *, h: float, radius: float, nev: int, settings: SolverSettings | None = None,
                      elem=None, output_dir: str | None = None, name: str = "run") -> PreparedSystem:
    """A prepared system for atoms already in bohr (no recentring, no files
    read): the entry used by benchmarks, tests and training-data generation."""
    from .inputs import ElementTable

    elem = elem or ElementTable()
    settings = settings or SolverSettings()
    n_atom = [np.asarray(a["coord"]).reshape(-1, 3).shape[0] for a in atoms]
    atoms = [{"typ": a["typ"], "coord": np.asarray(a["coord"], dtype=float).reshape(-1, 3)} for a in atoms]
    zelec = float(sum(elem[a["typ"]]["Z"] * c for a, c in zip(atoms, n_atom)))
    domain = cube_for_radius(radius, h)
    stem = os.path.join(output_dir, name) if output_dir else ""
    paths = RunPaths(output_file=stem + ".out" if stem else "", wfn_file=stem + "_wfn.dat" if stem else "",
                     initial_density_base=stem + "_init_rho" if stem else "",
                     converged_density_base=stem + "_conv_rho" if stem else "")
    inp = InputData(atoms=atoms, n_atom=n_atom, z_charge=0.0)
    return PreparedSystem(input_data=inp, settings=settings, domain=domain, h=h, nev=nev, zelec=zelec,
                          ztest=zelec, n_types=len(atoms), paths=paths)
