"""Synthetic input geometries of the benchmark configurations (angstrom).

No public dataset is involved; every structure is generated:
  h2o()                    O at the origin, H at (+-0.757, 0.586, 0)
  naphthalene()            planar C10H8, two regular hexagons (C-C 1.40)
                           sharing an edge on the y axis, C-H 1.09, centred
  sih_cluster(shells)      Si atoms of the diamond lattice (a = 5.43) in the
                           first `shells` neighbour-distance shells of an
                           atom-centred Si (4 -> Si35H36, 7 -> Si87H76), every
                           dangling bond capped by H at 1.48 along the bond
  sih_random_cluster(seed) Si(n)H(m), n ~ U{5..35}, grown on the same lattice
                           from an atom-centred Si, H-capped, default_rng(seed)
  water_cluster(seed)      (H2O)n, n ~ U{2..8}, rigid O-H 0.957 / 104.5 deg,
                           random positions in a 6 A ball with O-O >= 2.6,
                           random orientations, numpy default_rng(seed)
Species are grouped in the order they first appear.
"""
from __future__ import annotations

import numpy as np

from .models import A0_ANG


def group(symbols, coords):
    """[(sym, xyz)] -> reference atom list [{'typ', 'coord'}] in angstrom."""
    out: dict[str, list] = {}
    for s, c in zip(symbols, coords):
        out.setdefault(s, []).append(np.asarray(c, dtype=float))
    return [{"typ": s, "coord": np.array(v)} for s, v in out.items()]


def to_bohr(atoms):
    f = 1.0 / A0_ANG
    return [{"typ": a["typ"], "coord": np.asarray(a["coord"], dtype=float) * f} for a in atoms]


def h2o():
    return group(["O", "H", "H"], [(0.0, 0.0, 0.0), (0.757, 0.586, 0.0), (-0.757, 0.586, 0.0)])


def naphthalene(cc: float = 1.40, ch: float = 1.09):
    s3 = np.sqrt(3.0)
    syms, xyz = [], []
    shared = [(0.0, cc / 2), (0.0, -cc / 2)]
    for p in shared:
        syms.append("C")
        xyz.append((p[0], p[1], 0.0))
    hs = []
    for side in (1.0, -1.0):
        cx = side * cc * s3 / 2
        for ang in (30.0, 90.0, 270.0, 330.0) if side > 0 else (150.0, 90.0, 270.0, 210.0):
            t = np.deg2rad(ang)
            c = np.array([cx + cc * np.cos(t), cc * np.sin(t), 0.0])
            syms.append("C")
            xyz.append(tuple(c))
            d = c - np.array([cx, 0.0, 0.0])
            hs.append(tuple(c + ch * d / np.linalg.norm(d)))
    syms += ["H"] * len(hs)
    xyz += hs
    xyz = np.array(xyz)
    xyz -= xyz.mean(axis=0)
    return group(syms, xyz)


def sih_cluster(shells: int, a: float = 5.43, sih: float = 1.48):
    """Si atoms of the diamond lattice in the first `shells` neighbour
    (distance) shells around an atom-centred Si, plus H caps on every bond to
    an excluded lattice site.  shells = 4 gives Si35H36, shells = 7 Si87H76."""
    bond = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=float) * (a / 4)
    fcc = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]]) * a
    r = np.arange(-4, 5)
    cells = np.array(np.meshgrid(r, r, r, indexing="ij")).reshape(3, -1).T * a
    site_a = (cells[:, None, :] + fcc[None]).reshape(-1, 3)
    sites = np.vstack([site_a, site_a + bond[0]])
    sub = np.concatenate([np.zeros(len(site_a), int), np.ones(len(site_a), int)])
    dist = np.round(np.linalg.norm(sites, axis=1), 6)
    radii = np.unique(dist)
    keep = dist <= radii[shells]
    si, si_sub = sites[keep], sub[keep]
    si_set = {tuple(np.round(p, 6)) for p in si}
    hs = []
    for p, s in zip(si, si_sub):
        for b in bond * (1.0 if s == 0 else -1.0):
            if tuple(np.round(p + b, 6)) not in si_set:
                hs.append(p + sih * b / np.linalg.norm(b))
    return group(["Si"] * len(si) + ["H"] * len(hs), list(si) + hs)


def sih_random_cluster(seed: int, nmin: int = 5, nmax: int = 35, a: float = 5.43, sih: float = 1.48):
    """Seeded hydrogen-passivated silicon cluster of n ~ U{nmin..nmax} Si
    atoms: the diamond lattice (a = 5.43) grown from an atom-centred Si by
    adding, one at a time, a random lattice site bonded to the cluster (drawn
    with weight bonds^2 exp(-|r| / 0.8 A), so the clusters stay compact),
    then every dangling bond capped by H at 1.48 along the bond.  The
    training set of the learned start for the Si-H configurations."""
    rng = np.random.default_rng(seed)
    n_si = int(rng.integers(nmin, nmax + 1))
    bond = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=float) * (a / 4)
    key = lambda p: tuple(np.round(p, 6))  # noqa: E731
    si = [np.zeros(3)]
    sub = [0]
    have = {key(si[0])}
    while len(si) < n_si:
        cand: dict = {}
        for p, s in zip(si, sub):
            for b in bond * (1.0 if s == 0 else -1.0):
                q = p + b
                kq = key(q)
                if kq not in have:
                    c = cand.setdefault(kq, [q, 1 - s, 0])
                    c[2] += 1
        keys = sorted(cand)
        w = np.array([cand[k][2] ** 2 * np.exp(-np.linalg.norm(cand[k][0]) / 0.8) for k in keys], dtype=float)
        pick = cand[keys[int(rng.choice(len(keys), p=w / w.sum()))]]
        si.append(pick[0])
        sub.append(pick[1])
        have.add(key(pick[0]))
    hs = []
    for p, s in zip(si, sub):
        for b in bond * (1.0 if s == 0 else -1.0):
            if key(p + b) not in have:
                hs.append(p + sih * b / np.linalg.norm(b))
    return group(["Si"] * len(si) + ["H"] * len(hs), list(si) + hs)


def water_cluster(seed: int, nmin: int = 2, nmax: int = 8, ball: float = 6.0, dmin: float = 2.6,
                  roh: float = 0.957, angle_deg: float = 104.5):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(nmin, nmax + 1))
    half = np.deg2rad(angle_deg) / 2
    local = np.array([[0.0, 0.0, 0.0], [roh * np.sin(half), roh * np.cos(half), 0.0],
                      [-roh * np.sin(half), roh * np.cos(half), 0.0]])
    oxy = []
    while len(oxy) < n:
        p = rng.uniform(-ball, ball, 3)
        if np.linalg.norm(p) > ball:
            continue
        if all(np.linalg.norm(p - q) >= dmin for q in oxy):
            oxy.append(p)
    syms, xyz = [], []
    for p in oxy:
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        for s, r in zip(("O", "H", "H"), local @ q.T + p):
            syms.append(s)
            xyz.append(r)
    return group(syms, xyz)


def count(atoms) -> dict[str, int]:
    return {a["typ"]: int(np.asarray(a["coord"]).reshape(-1, 3).shape[0]) for a in atoms}


# Benchmark configurations: geometry builder, sphere radius and spacing (A),
# nev (occupied + extra), Chebyshev degree, SCF tolerance.
CONFIGS = {
    "h2o": dict(atoms=h2o, radius=5.0, h=0.2, nev=12, poldeg=10, tol=1e-6),
    "c10h8": dict(atoms=naphthalene, radius=7.0, h=0.18, nev=40, poldeg=12, tol=1e-6),
    "si35h36": dict(atoms=lambda: sih_cluster(4), radius=9.0, h=0.25, nev=128, poldeg=10, tol=1e-6),
    "si87h76": dict(atoms=lambda: sih_cluster(7), radius=11.0, h=0.25, nev=292, poldeg=16, tol=1e-6),
}


def config_system(name: str) -> dict:
    """Atoms (bohr), spacing and radius (bohr) and solver knobs of a named
    configuration; angstrom values are scaled by 1/a0 as the reference's
    convert_units_to_bohr does (rsdft_input.py:582-632)."""
    cfg = CONFIGS[name]
    f = 1.0 / A0_ANG
    return {"atoms": to_bohr(cfg["atoms"]()), "h": cfg["h"] * f, "radius": cfg["radius"] * f, "nev": cfg["nev"],
            "poldeg": cfg["poldeg"], "tol": cfg["tol"]}
