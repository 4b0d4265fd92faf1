"""Import the pseudopotential tables and the element table into this package.

The reference ships its norm-conserving pseudopotential data as a MATLAB file
(``src/V_ion/splineData.mat``: one ``data<El>`` array per element with the
columns radius, charge, hartree, pot_P, pot_S, wfn_P, wfn_S) and its element
defaults as ``src/elements_new.csv`` (Element, AtomicNumber, Z, Zvalue, h, r,
R).  Both are physical input data, not code.  This script converts them once
into ``pseudo_tables.npz`` (float64, values unchanged) and ``elements.csv``
(same rows, newline line endings) so that neither the product nor its tests
need the reference tree at run time.

Usage: python parsec_python_b200/data/import_tables.py <reference src dir>
"""
import os
import sys
from pathlib import Path

import numpy as np


def main(src_dir: str) -> None:
    import scipy.io

    src = Path(src_dir)
    here = Path(__file__).resolve().parent
    mat = scipy.io.loadmat(src / "V_ion" / "splineData.mat")
    arrays = {k[4:]: np.ascontiguousarray(v, dtype=np.float64)
              for k, v in mat.items() if k.startswith("data")}
    np.savez_compressed(here / "pseudo_tables.npz", **arrays)
    raw = (src / "elements_new.csv").read_bytes().decode("ascii")
    rows = [r for r in raw.replace("\r\n", "\n").replace("\r", "\n").split("\n") if r.strip()]
    (here / "elements.csv").write_text("\n".join(rows) + "\n")
    print(f"wrote {len(arrays)} element tables and {len(rows)} element rows")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("PARSEC_REF_SRC"):
        main(os.environ["PARSEC_REF_SRC"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference src directory> (or set PARSEC_REF_SRC)")
