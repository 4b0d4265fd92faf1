"""Generate the fixture that pins the oracle's preconditioned CG to the
reference's own Eigensolvers/pcg.py (zeyizhang-berkeley/parsec_python).

The reference's preconditioned branch (pcg.py:42-44,67-70) calls
precfun(PRE, r).  Its own driver hands it the string "precLU"
(rsdft_solver.py:339), which cannot be called, so here it is run with a
callable: PRE = the oracle's spectral preconditioner (the one the GPU path
uses for cg_prec = 1) and precfun(PRE, r) = PRE(r).  Writes
tests/golden/ref_pcg_prec.npz.

Usage: python tests/golden/make_golden_pcg_prec.py [reference src dir]
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))
from make_golden import _import_reference  # noqa: E402


def main(src: str) -> None:
    _import_reference(src)
    from Eigensolvers.pcg import pcg
    from Laplacian.fd3d import fd3d

    from oracle import oracle as O

    out = {}
    rng = np.random.default_rng(77)
    for tag, (nx, ny, nz, order, h) in {"a": (16, 14, 12, 8, 0.4), "b": (12, 12, 12, 4, 0.3)}.items():
        dom = {"nx": nx, "ny": ny, "nz": nz, "h": h}
        A = (1.0 / (h * h)) * fd3d(nx, ny, nz, order)
        M = O.spectral_preconditioner(dom, order)
        n = nx * ny * nz
        rhs = rng.standard_normal(n)
        x0 = rng.standard_normal(n) * 0.1
        x, its = pcg(A, rhs, x0.copy(), 200, 1e-5, M, lambda P, r: P(r))
        out.update({f"{tag}_rhs": rhs, f"{tag}_x0": x0, f"{tag}_x": x, f"{tag}_its": np.array(its),
                    f"{tag}_dims": np.array([nx, ny, nz, order]), f"{tag}_h": np.array(h)})
        print(tag, "its", its)
    np.savez_compressed(HERE / "ref_pcg_prec.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("PARSEC_REF_SRC"):
        main(os.environ["PARSEC_REF_SRC"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference src directory> (or set PARSEC_REF_SRC)")
