"""The run log (``.out``), density snapshots (``.npy``) and ``wfn.dat``.

Formats follow PARSEC.py's rsdft_output.py line for line (header
:39-46, parameter block :86-139, initial-density diagnostics :140-173, SCF
iteration block :176-230, total-energy summary :243-271, three density
variants in F order :49-83, legacy wfn.dat :298-334), so tools that parse
the reference's logs read these too.  An empty path disables writing.
"""
from __future__ import annotations

import os

import numpy as np

from .models import A0_ANG, RY_EV, EnergyComponents


def _append(path: str, text: str) -> None:
    if path:
        with open(path, "a", encoding="utf-8") as fh:
            fh.write(text)


def initialize_output_file(path: str, backend_label: str, density_method: str) -> None:
    if not path:
        return
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "w", encoding="utf-8") as fh:
        fh.write(f"Solver backend: {backend_label}\nDensity initialization: {density_method}\n")


def write_parameters(path, nev, atoms, n_atom, domain, h, poldeg, fd_order) -> None:
    out = [f"\n Number of states: \t{nev}\n\n", "Atom data:\n -------------\n",
           f" Total # of atom types is {len(atoms)}\n"]
    total = 0
    for t, a in enumerate(atoms):
        xyz = np.asarray(a["coord"])
        out.append(f" There are {n_atom[t]} {a['typ']} atoms\n and their coordinates are:\n\n")
        out.append("\t{:<12s}\t{:<12s}\t{:<12s}\n".format("x [a.u.]", "y [a.u.]", "z [a.u.]"))
        total += n_atom[t]
        for i in range(n_atom[t]):
            out.append(f"\t{xyz[i, 0]:12.6f}\t{xyz[i, 1]:12.6f}\t{xyz[i, 2]:12.6f}\n")
        out.append("\n\t{:<12s}\t{:<12s}\t{:<12s}\n".format("x [Ang]", "y [Ang]", "z [Ang]"))
        for i in range(n_atom[t]):
            v = xyz[i] * A0_ANG
            out.append(f"\t{v[0]:12.6f}\t{v[1]:12.6f}\t{v[2]:12.6f}\n")
        out.append("\n")
    n = domain["nx"] * domain["ny"] * domain["nz"]
    out += [" --------------------------------------------------\n",
            f" Total number of atoms :         {total}\n\n",
            f" Number of states:               {nev:10d} \n",
            f" h grid spacing :                {h:10.5f} a.u.   ({h * A0_ANG:10.5f} Ang)\n",
            f" Hamiltonian size :              {n:10d}  \n",
            f" Sphere Radius :                 {domain['radius']:10.5f} a.u.   ({domain['radius'] * A0_ANG:10.5f} Ang)\n",
            f" # grid points in each direction {domain['nx']:10d}  \n",
            f" Polynomial degree used :        {poldeg:10d}  \n",
            f" Finite difference order :       {fd_order:10d}  \n",
            " --------------------------------------------------\n"]
    _append(path, "".join(out))


def write_diag_info(path: str, info: dict | None) -> None:
    if not info:
        return
    s = " --------------------------------------------------\n Initial density electron count\n"
    if info.get("electron_count_initial") is not None:
        s += f" Initial density integrates to :     {info['electron_count_initial']:.6f} e-\n"
    if info.get("electron_count_normalized") is not None:
        s += f" Normalized density integrates to:  {info['electron_count_normalized']:.6f} e-"
        if info.get("electron_target") is not None:
            s += f" (target {info['electron_target']:.6f})"
        s += "\n"
    _append(path, s + " --------------------------------------------------\n")


def write_initial_density_diagnostics(path, rho_max, rho_min, hpsum0_ev, exc_ry) -> None:
    _append(path, f" max and min values of charge density [e/bohr^3]   {rho_max:.5e}   {rho_min:.5e}\n"
                  f" Initial Hartree energy (eV) = {hpsum0_ev:10.5f}  \n"
                  f" Initial Exchange-corr. energy (eV) = {exc_ry * RY_EV:10.5f}  \n")


def write_timings(path: str, entries: list[tuple[str, float]]) -> None:
    if entries:
        _append(path, "\n Setup timings [sec]\n --------------------------------------------------\n" +
                "".join(f" {label:<35} {t:12.6f}\n" for label, t in entries))


def write_density_range(path: str, rho_max: float, rho_min: float) -> None:
    _append(path, f" max and min values of charge density [e/bohr^3]   {rho_max:.5e}   {rho_min:.5e}\n")


def _energy_lines(e: EnergyComponents, n_atoms: int, indent: str) -> str:
    rows = [("Sum of eigenvalues     ", e.eigen_sum_ry), ("Hartree energy         ", e.hartree_ry),
            ("Exchange-corr. energy  ", e.xc_ry), ("Ion-ion repulsion      ", e.ion_ry),
            ("Total electronic energy", e.total_ry)]
    s = "".join(f"{indent}{lab} = {v * RY_EV:10.5f}  eV   = {v:10.5f}  Ry  \n" for lab, v in rows)
    s += (f"{indent}Electronic energy/atom  = {(e.total_ry * RY_EV) / n_atoms:10.5f}  eV   = "
          f"{e.total_ry / n_atoms:10.5f}  Ry  \n")
    return s


def write_scf_iteration(path, it, diag_label, diag_time, nev, lam, occ, hart_tol, hart_label, hart_time, err,
                        energies: EnergyComponents, n_atoms) -> None:
    s = [f"\n\n SCF iter # {it}  ... \n", f"Diagonalization method :\t{diag_label}\n",
         f"Diagonalization time [sec] :\t{diag_time}\n\n", "   State  Eigenvalue [Ry]     Eigenvalue [eV]  Occupation\n\n"]
    for i in range(nev):
        ev = float(lam[i]) * 2 * RY_EV
        s.append(f"{i + 1:5d}   {ev / RY_EV:15.10f}   {ev:18.10f}  {2 * float(occ[i]):5.2f}\n")
    s += [f"Hartree CG tol :\t{hart_tol:.1e} ({hart_label})\n", f"\nHartree potential time [sec]: \t{hart_time}\n\n",
          f"   ... SCF error = {err:10.2e}\n", "   Energy components this iter:\n",
          _energy_lines(energies, n_atoms, "     ")]
    _append(path, "".join(s))


def write_total_energy_summary(path: str, energies: EnergyComponents, n_atoms: int) -> None:
    _append(path, "\n\n Total Energies \n\n" + _energy_lines(energies, n_atoms, " "))


def save_density_variants(density_grid, domain, base_path: str) -> None:
    """<base>_grid.npy (electrons per point), <base>_bohr3.npy, <base>.npy
    (per cubic angstrom); arrays of shape (nx, ny, nz) in Fortran order."""
    if not base_path or density_grid is None:
        return
    flat = np.asarray(density_grid).reshape(-1)
    nx, ny, nz, h = int(domain["nx"]), int(domain["ny"]), int(domain["nz"]), float(domain["h"])
    if flat.size != nx * ny * nz or h <= 0:
        print(f"Warning: density size {flat.size} does not match grid {nx * ny * nz}, skipping {base_path}")
        return
    d = os.path.dirname(base_path)
    if d:
        os.makedirs(d, exist_ok=True)
    g = flat.reshape((nx, ny, nz), order="F")
    b3 = g / (h ** 3)
    np.save(f"{base_path}_grid.npy", g)
    np.save(f"{base_path}_bohr3.npy", b3)
    np.save(f"{base_path}.npy", b3 / (A0_ANG ** 3))


def save_wavefunction(path, domain, potential, rho, W, nev, n_types, atoms) -> None:
    """Legacy binary wfn.dat: magic 26, radius, h, pot, rho, first nev
    columns of W, then atom coordinates per species."""
    u32 = lambda v: np.array(v, dtype=np.uint32).tobytes()  # noqa: E731
    f64 = lambda v: np.asarray(v, dtype=np.float64).tobytes()  # noqa: E731
    with open(path, "wb") as fh:
        fh.write(u32(26) + f64(domain["radius"]) + f64(domain["h"]))
        pot = np.asarray(potential, dtype=np.float64)
        fh.write(u32(len(pot)) + pot.tobytes())
        r = np.asarray(rho, dtype=np.float64)
        fh.write(u32(len(r)) + r.tobytes())
        w = np.asarray(W, dtype=np.float64)
        fh.write(u32(w.shape[0]) + u32(nev))
        for i in range(nev):
            fh.write(f64(w[:, i]))
        fh.write(u32(n_types))
        for a in atoms:
            xyz = np.asarray(a["coord"], dtype=np.float64)
            fh.write(u32(len(xyz)))
            for row in xyz:
                fh.write(f64(row))


def load_wavefunction(path) -> dict:
    """Read the legacy binary wfn.dat that save_wavefunction writes
    (rsdft_output.py:298-334): magic 26, radius, h, the potential, the
    density, n x nev wavefunctions (one column after another), then per
    species its atom coordinates.  Returns a dict with those fields
    (wavefunctions as an n x nev array, atoms as a list of (count, 3) arrays).
    Species symbols are not in the file."""
    raw = open(path, "rb").read()
    pos = 0

    def u32():
        nonlocal pos
        v = int(np.frombuffer(raw, dtype=np.uint32, count=1, offset=pos)[0])
        pos += 4
        return v

    def f64(count):
        nonlocal pos
        v = np.frombuffer(raw, dtype=np.float64, count=count, offset=pos).copy()
        pos += 8 * count
        return v

    magic = u32()
    if magic != 26:
        raise ValueError(f"{path}: not a wfn.dat file (magic {magic}, expected 26)")
    radius, h = f64(1)[0], f64(1)[0]
    pot = f64(u32())
    rho = f64(u32())
    n = u32()
    nev = u32()
    W = np.empty((n, nev))
    for i in range(nev):
        W[:, i] = f64(n)
    atoms = []
    for _ in range(u32()):
        count = u32()
        atoms.append(f64(3 * count).reshape(count, 3))
    if pos != len(raw):
        raise ValueError(f"{path}: {len(raw) - pos} trailing bytes")
    return {"radius": float(radius), "h": float(h), "potential": pot, "rho": rho, "wavefunctions": W,
            "nev": nev, "atoms": atoms}
