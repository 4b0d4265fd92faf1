"""Golden vectors of the reference's Type-II multisecant mixer
(Mixer/msecant2.py with the parameters of Mixer/includemix.py), run in this
container on seeded fixed-point problems:

- "anderson": group_size = 0 (all iterates in one group: Anderson mixing);
- "group2": group_size = 2 (full groups orthogonalised against, the last
  group's DF replaced by DF C when it is full).

Step 9 scales the residual by 50, which triggers the restart branch; after a
restart the reference alternates its EN stage (2 -> 1 -> 2 ...), and later
steps cover that too.  Writes tests/golden/ref_mixer2.npz.

Usage: python tests/golden/make_golden_mixer2.py <reference src dir>
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def run(ms2, group_size: int, nmix: int = 64, steps: int = 16, seed: int = 21):
    rng = np.random.default_rng(seed)
    amat = rng.standard_normal((nmix, nmix)) * 0.3 / np.sqrt(nmix)
    bvec = rng.standard_normal(nmix)
    x = rng.standard_normal(nmix)
    mx = ms2.mixer()
    mx.params["group_size"] = group_size
    xs, fs, outs, ms = [], [], [], []
    for step in range(steps):
        f = np.tanh(amat @ x) + bvec - x
        if step == 9:
            f = f * 50.0
        xs.append(x.copy())
        fs.append(f.copy())
        x, m = mx.mixer(x, f)
        outs.append(np.asarray(x).copy())
        ms.append(m)
    return np.array(xs), np.array(fs), np.array(outs), np.array(ms)


def main(src: str) -> None:
    sys.path.insert(0, src)
    from Mixer import msecant2 as ms2

    out = {}
    for name, gs in (("anderson", 0), ("group2", 2)):
        x, f, o, m = run(ms2, gs)
        out[f"{name}_x"], out[f"{name}_f"], out[f"{name}_out"], out[f"{name}_m"] = x, f, o, m
        print(name, "m per step", m.tolist())
    np.savez_compressed(HERE / "ref_mixer2.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden_mixer2.py <reference src dir>")
    main(sys.argv[1])
