"""Learned initial density: a 3-D convolutional encoder-decoder that maps the
SAD density and the local ionic potential on the grid to a correction of the
density, used only as the SCF's starting point.

Contract (the consumer side of the reference, V_ion/pseudoDiag_ML4Den_poisson.py
:448-538, dispatched at rsdft_solver.py:95-108): the predicted density is
clamped at zero, renormalised to the valence charge, and the Hartree potential
of its difference from the SAD density is solved by the same CG (tol 1e-5, 200
iterations) and added to the SAD Hartree potential.  SAD stays the fallback:
with no trained weights the solver runs from SAD.

Network (1.29 M parameters; channels-last BF16 activations, BF16 weights,
FP32 accumulation; all kernels in csrc/unet.cu):

    (leaky ReLU after every layer but the last)
    e0  3^3  8 -> 8           full grid           (input: rho_SAD, V_loc, 6 zero channels)
    d1  3^3  8 -> 32  /2      half
    e1  3^3  32 -> 32         half
    d2  3^3  32 -> 64 /2      quarter
    e2  3^3  64 -> 64         quarter
    d3  3^3  64 -> 128 /2     eighth
    b   3^3  128 -> 128       eighth
    u2  3^3  up(b) + e2 -> 64   quarter
    u1  3^3  up(u2) + e1 -> 32  half
    u0  3^3  up(u1) + e0 -> 8   full
    out 1^3  8 -> 8 (channel 0 = correction), linear

Training data come from this project's own FP64 GPU SCF on seeded systems of
two families (water clusters; hydrogen-capped silicon clusters).  `generate`
writes a training set with one replica per GPU under torchrun (a strided
share of the seeds per rank, no exchange but one host barrier); training
runs on one GPU through psc_conv3d_fwd / psc_conv3d_bwd / psc_adam_step,
from such a set or generating its samples itself.

    torchrun --nproc-per-node 8 -m parsec_python_b200.learned generate --family sih --out DIR
    python -m parsec_python_b200.learned train --family sih --data DIR
"""
from __future__ import annotations

import argparse
import json
import time
from ctypes import byref, c_int
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from . import gpu, workloads
from .models import A0_ANG, SolverSettings

DATA_DIR = Path(__file__).resolve().parent / "data"
DEFAULT_WEIGHTS = DATA_DIR / "learned_init_water.npz"
SIH_WEIGHTS = DATA_DIR / "learned_init_sih.npz"


@dataclass(frozen=True)
class Layer:
    name: str
    src: str          # A input
    up: int           # A is upsampled x2
    skip: str | None  # S input
    ca: int
    cs: int
    cout: int
    stride: int
    ksize: int
    act: int          # 0 identity, 2 leaky ReLU


LAYERS = (
    Layer("e0", "in", 0, None, 8, 0, 8, 1, 3, 2),
    Layer("d1", "e0", 0, None, 8, 0, 32, 2, 3, 2),
    Layer("e1", "d1", 0, None, 32, 0, 32, 1, 3, 2),
    Layer("d2", "e1", 0, None, 32, 0, 64, 2, 3, 2),
    Layer("e2", "d2", 0, None, 64, 0, 64, 1, 3, 2),
    Layer("d3", "e2", 0, None, 64, 0, 128, 2, 3, 2),
    Layer("b", "d3", 0, None, 128, 0, 128, 1, 3, 2),
    Layer("u2", "b", 1, "e2", 128, 64, 64, 1, 3, 2),
    Layer("u1", "u2", 1, "e1", 64, 32, 32, 1, 3, 2),
    Layer("u0", "u1", 1, "e0", 32, 8, 8, 1, 3, 2),
    Layer("out", "u0", 0, None, 8, 0, 8, 1, 1, 0),
)


def n_params() -> int:
    return sum(l.ksize ** 3 * (l.ca + l.cs) * l.cout + l.cout for l in LAYERS)


def _half(d):
    return tuple((x + 1) // 2 for x in d)


class UNet3D:
    """Parameters, activations and gradients of the encoder-decoder on one
    grid, all in device memory of the context's GPU."""

    WORK_FLOATS = 16 * 1024 * 1024

    def __init__(self, ctx: gpu.GridContext, seed: int = 0, params: dict | None = None):
        self.ctx = ctx
        self.dev = ctx.device
        dims = {"in": (ctx.nx, ctx.ny, ctx.nz)}
        level = {"in": dims["in"]}
        for l in LAYERS:
            src = level[l.src]
            if l.up:
                out = level[l.skip]
                if _half(out) != src:
                    raise ValueError(f"layer {l.name}: grid mismatch for upsampling")
            elif l.stride == 2:
                out = _half(src)
            else:
                out = src
            level[l.name] = out
        self.grid = level
        # one flat FP32 master vector for all weights and biases
        self.offsets = {}
        off = 0
        for l in LAYERS:
            nw = l.ksize ** 3 * (l.ca + l.cs) * l.cout
            self.offsets[l.name] = (off, nw, off + nw, l.cout)
            off += nw + l.cout
        self.n = off
        self.w = torch.zeros(self.n, dtype=torch.float32, device=self.dev)
        if params is None:
            rng = np.random.default_rng(seed)
            host = np.zeros(self.n, dtype=np.float32)
            for l in LAYERS:
                o, nw, ob, nb = self.offsets[l.name]
                fan_in = l.ksize ** 3 * (l.ca + l.cs)
                std = np.sqrt(2.0 / fan_in) * (0.1 if l.name == "out" else 1.0)
                host[o:o + nw] = rng.standard_normal(nw).astype(np.float32) * std
            self.w.copy_(torch.from_numpy(host))
            self.scales = {"a0": 1.0, "a1": 1.0, "at": 1.0}
        else:
            self.w.copy_(torch.from_numpy(np.asarray(params["w"], dtype=np.float32)))
            self.scales = {k: float(params[k]) for k in ("a0", "a1", "at")}
        self.wb = torch.empty(self.n, dtype=torch.bfloat16, device=self.dev)
        self.ctx.call("psc_f32_to_bf16", gpu._p(self.w), gpu._p(self.wb), self.n, gpu._stream())
        self.grad = torch.zeros(self.n, dtype=torch.float32, device=self.dev)
        self.m = torch.zeros_like(self.grad)
        self.v = torch.zeros_like(self.grad)
        self.step_count = 0
        self.acts: dict[str, torch.Tensor] = {}
        self.work = None
        self.loss_dev = torch.zeros(1, dtype=torch.float64, device=self.dev)

    # -- helpers -------------------------------------------------------------
    def _nvox(self, name):
        x, y, z = self.grid[name]
        return x * y * z

    def _geom(self, l: Layer):
        gi = self.grid[l.skip] if l.up else self.grid[l.src]
        ga = self.grid[l.src]
        go = self.grid[l.name]
        g = (c_int * 15)(gi[0], gi[1], gi[2], ga[0], ga[1], ga[2], l.up, l.ca, l.cs, go[0], go[1], go[2],
                         l.stride, l.ksize, l.cout)
        return g

    def _wviews(self, l: Layer, t: torch.Tensor):
        o, nw, ob, nb = self.offsets[l.name]
        return t[o:o + nw], t[ob:ob + nb]

    # -- forward / backward --------------------------------------------------
    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: BF16 [n][8] network input; returns FP32 [n][8] (channel 0 is the output)."""
        self.acts = {"in": x}
        out32 = None
        for l in LAYERS:
            a = self.acts[l.src]
            s = self.acts[l.skip] if l.skip else None
            wv, bv = self._wviews(l, self.wb)
            _, bias = self._wviews(l, self.w)
            y = torch.empty(self._nvox(l.name), l.cout, dtype=torch.bfloat16, device=self.dev)
            if l.name == "out":
                out32 = torch.empty(self._nvox(l.name), l.cout, dtype=torch.float32, device=self.dev)
            self.ctx.call("psc_conv3d_fwd", self._geom(l), gpu._p(a), gpu._p(s), gpu._p(wv), gpu._p(bias),
                          l.act, gpu._p(y), gpu._p(out32 if l.name == "out" else None), gpu._stream())
            self.acts[l.name] = y
        return out32

    def backward(self, gout: torch.Tensor) -> None:
        """gout: FP32 [n][8] = dL/d(out); fills self.grad (weights and biases)."""
        if self.work is None:
            self.work = torch.empty(self.WORK_FLOATS, dtype=torch.float32, device=self.dev)
        grads = {"out": gout}
        for l in reversed(LAYERS):
            g = grads.pop(l.name)
            a = self.acts[l.src]
            s = self.acts[l.skip] if l.skip else None
            nvo = self._nvox(l.name)
            gm = torch.empty(nvo, l.cout, dtype=torch.float32, device=self.dev)
            need_in = l.src != "in"
            dvin = dA = dS = None
            acc_a = acc_s = 0
            if need_in:
                nvi = self._nvox(l.skip if l.up else l.src)
                dvin = torch.empty(nvi, l.ca + l.cs, dtype=torch.float32, device=self.dev)
                if l.src in grads:
                    acc_a = 1
                else:
                    grads[l.src] = torch.empty(self._nvox(l.src), l.ca, dtype=torch.float32, device=self.dev)
                dA = grads[l.src]
                if l.skip:
                    if l.skip in grads:
                        acc_s = 1
                    else:
                        grads[l.skip] = torch.empty(self._nvox(l.skip), l.cs, dtype=torch.float32, device=self.dev)
                    dS = grads[l.skip]
            dW, dB = self._wviews(l, self.grad)
            wv, _ = self._wviews(l, self.wb)
            self.ctx.call("psc_conv3d_bwd", self._geom(l), gpu._p(a), gpu._p(s), gpu._p(wv), gpu._p(g),
                          gpu._p(self.acts[l.name] if l.act else None), l.act, gpu._p(gm), gpu._p(dvin), gpu._p(dA),
                          acc_a, gpu._p(dS), acc_s, gpu._p(dW), gpu._p(dB), gpu._p(self.work), self.WORK_FLOATS,
                          gpu._stream())

    def loss_and_grad(self, out32: torch.Tensor, target: torch.Tensor):
        grad = torch.empty_like(out32)
        self.ctx.call("psc_mse_loss", gpu._p(out32), out32.shape[1], gpu._p(target), target.numel(), gpu._p(grad),
                      gpu._p(self.loss_dev), gpu._stream())
        return self.loss_dev, grad

    def adam(self, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.step_count += 1
        self.ctx.call("psc_adam_step", gpu._p(self.w), gpu._p(self.wb), gpu._p(self.grad), gpu._p(self.m),
                      gpu._p(self.v), self.n, float(lr), float(b1), float(b2), float(eps), self.step_count,
                      gpu._stream())

    # -- input / output --------------------------------------------------------
    def pack(self, rho_bohr3: torch.Tensor, vloc: torch.Tensor) -> torch.Tensor:
        x = torch.empty(self.ctx.n, 8, dtype=torch.bfloat16, device=self.dev)
        self.ctx.call("psc_pack_input", gpu._p(rho_bohr3.contiguous()), gpu._p(vloc.contiguous()),
                      self.scales["a0"], self.scales["a1"], gpu._p(x), gpu._stream())
        return x

    def predict_delta(self, rho_bohr3: torch.Tensor, vloc: torch.Tensor) -> torch.Tensor:
        """Density correction (e/bohr^3, FP64) on the context's grid."""
        out = self.forward(self.pack(rho_bohr3, vloc))
        return out[:, 0].double() / self.scales["at"]

    def save(self, path: Path, meta: dict) -> None:
        """Weights as BF16 bit patterns (what the kernels compute with), biases
        as FP32, plus the input / target scales and the training record."""
        w = self.w.cpu().numpy()
        bias_mask = np.zeros(self.n, dtype=bool)
        for l in LAYERS:
            o, nw, ob, nb = self.offsets[l.name]
            bias_mask[ob:ob + nb] = True
        wb = self.wb.cpu().view(torch.int16).numpy().view(np.uint16)
        np.savez_compressed(path, wb16=wb, bias=w[bias_mask], a0=self.scales["a0"], a1=self.scales["a1"],
                            at=self.scales["at"], meta=json.dumps(meta))


def _bias_mask() -> np.ndarray:
    mask, off = [], 0
    for l in LAYERS:
        nw = l.ksize ** 3 * (l.ca + l.cs) * l.cout
        mask.append(np.zeros(nw, dtype=bool))
        mask.append(np.ones(l.cout, dtype=bool))
    return np.concatenate(mask)


_W_CACHE: dict = {}


def load_weights(path: Path | str = DEFAULT_WEIGHTS) -> dict | None:
    """The trained parameters in a file, read once per process (and again if
    the file changes): the same dict for every SCF, so the network built from
    it (cached_net) is reused instead of rebuilt with fresh device buffers
    for every solve."""
    p = Path(path)
    if not p.exists():
        return None
    st = p.stat()
    key = (str(p.resolve()), st.st_mtime_ns, st.st_size)
    hit = _W_CACHE.get(key)
    if hit is not None:
        return hit
    z = np.load(p, allow_pickle=False)
    if "wb16" in z.files:
        # BF16 -> FP32 is exact: the bit pattern is the upper half of the FP32 word
        w = (z["wb16"].astype(np.uint32) << 16).view(np.float32).copy()
        w[_bias_mask()] = z["bias"]
    else:
        w = z["w"]
    params = {"w": w, "a0": float(z["a0"]), "a1": float(z["a1"]), "at": float(z["at"]),
              "meta": json.loads(str(z["meta"]))}
    _W_CACHE[key] = params
    return params


# Networks built for a grid shape, reused by later SCFs on the same grid: the
# weights are uploaded once per process, not once per SCF.  Each entry keeps
# the grid context it was built with alive (kernel calls need a context; the
# network's own buffers do not depend on which SCF is running).
_NET_CACHE: dict = {}


def cached_net(ctx: gpu.GridContext, params: dict) -> "UNet3D":
    key = (ctx.device.index, ctx.nx, ctx.ny, ctx.nz, id(params["w"]))
    hit = _NET_CACHE.get(key)
    if hit is None:
        if len(_NET_CACHE) >= 4:
            _NET_CACHE.pop(next(iter(_NET_CACHE)))
        # the entry keeps the weight array alive, so its id cannot be reused
        hit = (UNet3D(ctx, params=params), params["w"])
        _NET_CACHE[key] = hit
    return hit[0]


class LearnedInit:
    """init_density callback for solver.run_rsdft_calculation: SAD density ->
    network correction -> clamp, renormalise, Hartree potential of the
    difference from SAD (pseudoDiag_ML4Den_poisson.py:448-538).  Returns
    (rho1, dh); the solver uses them for the first potential and as the
    Hartree CG's starting point.  dh is solved with the spectrally
    preconditioned CG (2-3 iterations to tol 1e-5; the reference's plain
    200-iteration CG stops short of its tolerance at these grid sizes).
    `last` records the CUDA-event times of the three stages."""

    def __init__(self, params: dict):
        if params["w"].size != n_params():
            raise ValueError("weights do not match the network")
        self.params = params
        self.last = {}

    def __call__(self, ctx: gpu.GridContext, rho0, hpot0, ppot, A):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record()
        net = cached_net(ctx, self.params)
        ev[1].record()
        h3 = ctx.h ** 3
        rho_b = rho0 / h3
        delta = net.predict_delta(rho_b, ppot)
        ev[2].record()
        if not bool(torch.isfinite(delta).all()):
            self.last = {"fallback": "non-finite prediction"}
            return rho0, torch.zeros_like(rho0)
        rho1 = torch.clamp(rho_b + delta, min=0.0) * h3
        zsum = gpu.numpy_sum(ctx, rho0)
        rho1 = rho1 * (zsum / gpu.numpy_sum(ctx, rho1))
        hrhs = (4 * np.pi / h3) * (rho1 - rho0)
        dh, its = gpu.pcg(A, hrhs, torch.zeros_like(hrhs), 200, 1e-5, "spectral", "precLU")
        ev[3].record()
        torch.cuda.synchronize()
        self.last = {"cg_its": its, "rho_start": rho1, "net_s": ev[0].elapsed_time(ev[1]) / 1e3,
                     "forward_s": ev[1].elapsed_time(ev[2]) / 1e3, "hartree_s": ev[2].elapsed_time(ev[3]) / 1e3}
        return rho1, dh


# ---------------------------------------------------------------------------
# data, training, evaluation
# ---------------------------------------------------------------------------
WATER_H_ANG = 0.2
WATER_RADIUS_ANG = 9.0   # clusters live in a 6 A ball; 3 A margin for the density tails


def _water_nev(counts: dict) -> int:
    return 4 * counts.get("O", 0) + 4


def _sih_nev(counts: dict) -> int:
    occ = (4 * counts.get("Si", 0) + counts.get("H", 0)) // 2
    return occ + max(8, int(round(0.45 * occ)))


# Training families: geometry generator, grid, number of states, weights file.
#   water  (H2O)n, n in 2..8 (workloads.water_cluster), h 0.2 A, 9 A sphere
#   sih    Si(5..35) H-capped clusters (workloads.sih_random_cluster), h 0.25 A
#          (the Si-H configurations' spacing), 10 A sphere (extents up to 8 A)
FAMILIES = {
    "water": {"build": workloads.water_cluster, "h_ang": WATER_H_ANG, "radius_ang": WATER_RADIUS_ANG,
              "nev": _water_nev, "weights": DEFAULT_WEIGHTS},
    "sih": {"build": workloads.sih_random_cluster, "h_ang": 0.25, "radius_ang": 10.0, "nev": _sih_nev,
            "weights": SIH_WEIGHTS},
}


def weights_for(atoms) -> Path:
    """The trained network for a system: the Si-H one when the system holds
    silicon, else the water one."""
    species = {a["typ"] for a in atoms}
    return SIH_WEIGHTS if "Si" in species else DEFAULT_WEIGHTS


def family_system(family: str, seed: int, settings: SolverSettings):
    from .inputs import ElementTable
    from .system import system_from_atoms

    fam = FAMILIES[family]
    atoms = fam["build"](seed)
    f = 1.0 / A0_ANG
    atoms = [{"typ": a["typ"], "coord": np.asarray(a["coord"], dtype=float).reshape(-1, 3) * f} for a in atoms]
    nev = fam["nev"](workloads.count(atoms))
    elem = ElementTable()
    prob = system_from_atoms(atoms, h=fam["h_ang"] * f, radius=fam["radius_ang"] * f, nev=nev, settings=settings,
                             elem=elem)
    return prob, elem


def water_system(seed: int, settings: SolverSettings):
    return family_system("water", seed, settings)


def run_scf(seed: int, init=None, tol: float = 1e-6, scf_seed: int = 0, energy_target=None, family: str = "water",
            cg_prec: int = 0, precision: str = "fp64"):
    from .backend import select_solver_backend
    from .solver import run_rsdft_calculation

    s = SolverSettings(tol=tol, poldeg=10, maxits=80, seed=scf_seed, cg_prec=cg_prec, precision=precision)
    s.normalize()
    prob, elem = family_system(family, seed, s)
    backend = select_solver_backend(s)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = run_rsdft_calculation(prob, elem, len(elem), backend, verbose=False, init_density=init,
                                energy_target=energy_target)
    torch.cuda.synchronize()
    return res, time.perf_counter() - t0, backend


def make_sample(seed: int, family: str = "water"):
    """(SAD density e/bohr^3, V_loc, converged - SAD density) on the family's
    grid; the converged density of the FP64 SCF (preconditioned Hartree solve
    for the Si-H family, whose larger grids leave the plain CG short of its
    tolerance)."""
    res, _, backend = run_scf(seed, family=family, cg_prec=1 if family == "sih" else 0)
    rt = backend.runtime
    prob, elem = family_system(family, seed, rt.settings)
    ctx = rt.context(prob.domain)
    rho0, _, ppot, _ = backend.pseudo_diag(prob.domain, prob.input_data.atoms, elem, len(elem), return_info=True)
    h3 = ctx.h ** 3
    rho_sad = rho0 / h3
    return ctx, rho_sad, ppot.clone(), (res.rho - rho_sad).float(), res


TRAIN_SEEDS = 512        # geometries 0..511 train the network; 512.. are held out


def partition_seeds(seeds, rank: int, world: int) -> list:
    """The geometries one replica generates: every world-th seed from position
    rank.  Cluster sizes are drawn independently per seed, so the strided
    split balances the ranks' work without a schedule; the union over ranks is
    every seed exactly once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(seeds)[rank::world]


def sample_arrays(seed: int, family: str):
    """One training sample as host arrays: SAD density (e/bohr^3), V_loc, the
    converged - SAD density (all FP32, x fastest), the domain and the SCF's
    iteration count."""
    ctx, rs, vl, dt, res = make_sample(seed, family)
    dom = {"nx": ctx.nx, "ny": ctx.ny, "nz": ctx.nz, "h": ctx.h, "radius": ctx.radius}
    return (rs.float().cpu().numpy(), vl.float().cpu().numpy(), dt.float().cpu().numpy(), dom,
            int(res.iterations))


def generate(family: str, seeds, out_dir: Path, rank: int = 0, world: int = 1, sample_fn=None, log=print) -> dict:
    """Training samples of one replica into out_dir/<family>_<seed>.npz.

    Each rank runs its share of the seeds (partition_seeds) on its own GPU,
    one SCF per geometry, with no exchange between ranks; a file already
    present is kept, so an interrupted run resumes.  Seeds whose SCF stops
    with ValueError (the reference's "Bounds are incorrect") are listed as
    skipped.  The rank's record goes to out_dir/manifest_rank<r>.json;
    merge_manifests joins them once every rank is done."""
    sample_fn = sample_fn or sample_arrays
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    done, skipped, t0 = [], [], time.perf_counter()
    for sd in partition_seeds(seeds, rank, world):
        path = out_dir / f"{family}_{sd:05d}.npz"
        if path.exists():
            done.append(sd)
            continue
        try:
            rs, vl, dt, dom, its = sample_fn(sd, family)
        except ValueError as exc:
            skipped.append(sd)
            log(f"  rank {rank}: seed {sd} skipped: {exc}")
            continue
        tmp = path.with_name(path.stem + f".part{rank}.npz")
        np.savez(tmp, rho_sad=rs, vloc=vl, delta=dt, domain=json.dumps(dom), iterations=np.array(its),
                 seed=np.array(sd))
        tmp.replace(path)
        done.append(sd)
    rec = {"rank": rank, "world": world, "family": family, "done": done, "skipped": skipped,
           "seconds": time.perf_counter() - t0}
    (out_dir / f"manifest_rank{rank}.json").write_text(json.dumps(rec))
    return rec


def merge_manifests(out_dir: Path, world: int) -> dict:
    """Join the ranks' records into out_dir/manifest.json (seeds ascending).
    Raises if a rank's record is missing or two ranks claim the same seed."""
    out_dir = Path(out_dir)
    recs = []
    for r in range(world):
        f = out_dir / f"manifest_rank{r}.json"
        if not f.exists():
            raise FileNotFoundError(f"rank {r} left no record in {out_dir}")
        recs.append(json.loads(f.read_text()))
    done = [sd for rec in recs for sd in rec["done"]]
    if len(done) != len(set(done)):
        raise ValueError("two ranks generated the same seed")
    man = {"family": recs[0]["family"], "world": world, "seeds": sorted(done),
           "skipped": sorted(sd for rec in recs for sd in rec["skipped"]),
           "rank_seconds": [rec["seconds"] for rec in recs]}
    (out_dir / "manifest.json").write_text(json.dumps(man))
    return man


def load_samples(data_dir: Path, n_train: int, device=None):
    """The first n_train samples (ascending seed) of a generated set as
    (domain, [(rho_sad, vloc, delta)], seeds): inputs FP64, targets FP32, on
    device (host when None)."""
    data_dir = Path(data_dir)
    man = json.loads((data_dir / "manifest.json").read_text())
    seeds = man["seeds"][:n_train]
    out, dom = [], None
    for sd in seeds:
        with np.load(data_dir / f"{man['family']}_{sd:05d}.npz") as z:
            d = json.loads(str(z["domain"]))
            if dom is None:
                dom = d
            elif (d["nx"], d["ny"], d["nz"]) != (dom["nx"], dom["ny"], dom["nz"]):
                raise ValueError(f"seed {sd}: grid {d} differs from {dom}")
            out.append(tuple(torch.from_numpy(z[k]).to(device, dt) for k, dt in
                             (("rho_sad", torch.float64), ("vloc", torch.float64), ("delta", torch.float32))))
    return dom, out, seeds


def train(n_train: int, epochs: int, out: Path, lr: float = 2e-4, seed: int = 0, log=print,
          family: str = "water", data_dir: Path | None = None) -> dict:
    """Train the network on n_train geometries of the family: generated here
    one after another, or read from data_dir (a set written by generate on
    any number of replicas)."""
    t_data = time.perf_counter()
    samples = []
    ctx0 = None
    skipped = []
    sd = 0
    if data_dir is not None:
        dom, samples, used = load_samples(data_dir, n_train, torch.device("cuda", torch.cuda.current_device()))
        ctx0 = gpu.GridContext(dom, 8)
        skipped = json.loads((Path(data_dir) / "manifest.json").read_text())["skipped"]
        sd = used[-1] + 1 if used else 0
    while len(samples) < n_train and sd < TRAIN_SEEDS:
        try:
            ctx, rs, vl, dt, res = make_sample(sd, family)
        except ValueError as exc:   # e.g. the reference's "Bounds are incorrect" stop in chefsi1
            skipped.append(sd)
            log(f"  seed {sd} skipped: {exc}")
            sd += 1
            continue
        if ctx0 is None:
            ctx0 = ctx
        samples.append((rs, vl, dt))
        if len(samples) % 32 == 1:
            log(f"  sample {len(samples) - 1} (seed {sd}): {res.iterations} SCF iterations")
        sd += 1
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t_data
    n_train = len(samples)
    # fixed input / target scales from the training set
    a0 = 1.0 / float(torch.stack([s[0].std() for s in samples]).mean())
    a1 = 1.0 / float(torch.stack([s[1].std() for s in samples]).mean())
    at = 1.0 / float(torch.stack([s[2].std() for s in samples]).mean())
    net = UNet3D(ctx0, seed=seed)
    net.scales = {"a0": a0, "a1": a1, "at": at}
    xs = [net.pack(s[0], s[1]) for s in samples]
    ts = [(s[2] * at).contiguous() for s in samples]
    del samples
    rng = np.random.default_rng(seed)
    t_train = time.perf_counter()
    steps = epochs * n_train
    losses = []
    for ep in range(epochs):
        order = rng.permutation(n_train)
        ep_loss = torch.zeros(1, dtype=torch.float64, device=net.dev)
        for i in order:
            out32 = net.forward(xs[i])
            loss, g = net.loss_and_grad(out32, ts[i])
            ep_loss += loss
            net.backward(g)
            # linear warm-up over the first 10 % of the steps, then cosine decay
            st = net.step_count
            warm = max(1, steps // 10)
            lr_t = lr * (st + 1) / warm if st < warm else lr * 0.5 * (1 + np.cos(np.pi * (st - warm) / (steps - warm)))
            net.adam(lr_t)
        losses.append(float(ep_loss.item()) / n_train)
        log(f"  epoch {ep}: mean loss {losses[-1]:.4e} (relative to the target variance)")
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t_train
    meta = {"n_train": n_train, "epochs": epochs, "lr": lr, "seed": seed, "losses": losses,
            "seeds_used": [0, sd], "seeds_skipped": skipped,
            "data_seconds": t_data, "train_seconds": t_train, "grid": list(net.grid["in"]), "family": family,
            "h_ang": FAMILIES[family]["h_ang"], "radius_ang": FAMILIES[family]["radius_ang"], "params": n_params()}
    net.save(out, meta)
    return meta


def evaluate(seeds, weights: Path, log=print, family: str = "water") -> dict:
    """SCF time-to-1e-5 Ha from SAD and from the learned density on each
    geometry: E* is the SAD-initialised run driven to tol 1e-8; both timed
    runs stop at the reference test (err <= 1e-6) once their energy is within
    1e-5 Ha of E*.  Iterations, wall times and |E - E*| are reported."""
    params = load_weights(weights)
    if params is None:
        raise FileNotFoundError(weights)
    rows = []
    skipped = []
    for sd in seeds:
        try:
            r_ref, _, _ = run_scf(sd, tol=1e-8, family=family)
            if not r_ref.converged:
                skipped.append(sd)
                log(f"  seed {sd} skipped: the tol-1e-8 SCF did not converge")
                continue
            e_star = r_ref.history[-1]["total_ry"]
            target = (e_star, 2e-5)   # 1e-5 Ha
            r_sad, t_sad, _ = run_scf(sd, energy_target=target, family=family)
            init = LearnedInit(params)
            r_ml, t_ml, backend = run_scf(sd, init=init, energy_target=target, family=family)
        except ValueError as exc:
            skipped.append(sd)
            log(f"  seed {sd} skipped: {exc}")
            continue
        e_sad, e_ml = r_sad.history[-1]["total_ry"], r_ml.history[-1]["total_ry"]
        # distance of each starting density from the converged one, in electrons: h^3 sum |rho_start - rho|
        rt = backend.runtime
        prob, elem = family_system(family, sd, rt.settings)
        ctx = rt.context(prob.domain)
        rho0, _, _, _ = backend.pseudo_diag(prob.domain, prob.input_data.atoms, elem, len(elem), return_info=True)
        h3 = ctx.h ** 3
        conv_pt = r_ref.rho * h3
        d_sad = float((rho0 - conv_pt).abs().sum())
        d_ml = float((init.last.get("rho_start", rho0) - conv_pt).abs().sum())
        rows.append({"seed": sd, "its_sad": r_sad.iterations, "its_learned": r_ml.iterations, "t_sad": t_sad,
                     "t_learned": t_ml, "e_star_ry": e_star, "de_sad_ha": abs(e_sad - e_star) / 2,
                     "de_learned_ha": abs(e_ml - e_star) / 2, "start_drho_sad_e": d_sad,
                     "start_drho_learned_e": d_ml, "start_e_err_sad_ha": abs(r_sad.history[0]["total_ry"] - e_star) / 2,
                     "start_e_err_learned_ha": abs(r_ml.history[0]["total_ry"] - e_star) / 2,
                     "converged": bool(r_sad.converged and r_ml.converged)})
        log(f"  seed {sd}: SAD {r_sad.iterations} its {t_sad:.3f}s, learned {r_ml.iterations} its {t_ml:.3f}s, "
            f"|dE| SAD {rows[-1]['de_sad_ha']:.1e} learned {rows[-1]['de_learned_ha']:.1e} Ha, "
            f"start |drho| SAD {d_sad:.3f} learned {d_ml:.3f} e")
    conv = [r for r in rows if r["converged"]]
    its_s = np.array([r["its_sad"] for r in conv])
    its_l = np.array([r["its_learned"] for r in conv])
    summary = {"n": len(conv), "mean_its_sad": float(its_s.mean()), "mean_its_learned": float(its_l.mean()),
               "mean_t_sad": float(np.mean([r["t_sad"] for r in conv])),
               "mean_t_learned": float(np.mean([r["t_learned"] for r in conv])),
               "max_de_sad_ha": float(max(r["de_sad_ha"] for r in conv)),
               "mean_start_drho_sad_e": float(np.mean([r["start_drho_sad_e"] for r in conv])),
               "mean_start_drho_learned_e": float(np.mean([r["start_drho_learned_e"] for r in conv])),
               "mean_first_iter_e_err_sad_ha": float(np.mean([r["start_e_err_sad_ha"] for r in conv])),
               "mean_first_iter_e_err_learned_ha": float(np.mean([r["start_e_err_learned_ha"] for r in conv])),
               "max_de_learned_ha": float(max(r["de_learned_ha"] for r in conv)),
               "not_converged": [r["seed"] for r in rows if not r["converged"]], "skipped": skipped, "rows": rows}
    return summary


def generate_distributed(family: str, seeds, out_dir: Path, sample_fn=None, timeout_s: float = 3600.0) -> dict:
    """generate() on every rank of a torchrun launch (RANK / LOCAL_RANK /
    WORLD_SIZE from the environment; one process per GPU, LOCAL_RANK picks
    the device), then rank 0 merges the records.  The only exchange is one
    host barrier on a gloo group (no data crosses it); without torchrun
    variables it runs as a single replica."""
    import os

    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("gloo", timeout=timedelta(seconds=timeout_s))
    if torch.cuda.is_available():
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    try:
        rec = generate(family, seeds, out_dir, rank, world, sample_fn=sample_fn)
        if world > 1:
            dist.barrier()
        return merge_manifests(out_dir, world) if rank == 0 else rec
    finally:
        if world > 1:
            dist.destroy_process_group()


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m parsec_python_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--family", choices=sorted(FAMILIES), default="water")
    t.add_argument("--n-train", type=int, default=512)
    t.add_argument("--epochs", type=int, default=12)
    t.add_argument("--lr", type=float, default=2e-4)
    t.add_argument("--out", type=Path, default=None)
    t.add_argument("--data", type=Path, default=None, help="a set written by `generate` (else generated here)")
    g = sub.add_parser("generate", help="training samples, one replica per GPU under torchrun")
    g.add_argument("--family", choices=sorted(FAMILIES), default="water")
    g.add_argument("--first", type=int, default=0)
    g.add_argument("--count", type=int, default=TRAIN_SEEDS)
    g.add_argument("--out", type=Path, required=True)
    e = sub.add_parser("eval")
    e.add_argument("--family", choices=sorted(FAMILIES), default="water")
    e.add_argument("--first", type=int, default=512)
    e.add_argument("--count", type=int, default=64)
    e.add_argument("--weights", type=Path, default=None)
    e.add_argument("--json", type=Path, default=None)
    a = ap.parse_args(argv)
    if a.cmd == "train":
        meta = train(a.n_train, a.epochs, a.out or FAMILIES[a.family]["weights"], lr=a.lr, family=a.family,
                     data_dir=a.data)
        print(json.dumps({k: v for k, v in meta.items() if k != "losses"} | {"final_loss": meta["losses"][-1]}))
    elif a.cmd == "generate":
        print(json.dumps(generate_distributed(a.family, range(a.first, a.first + a.count), a.out)))
    else:
        summ = evaluate(range(a.first, a.first + a.count), a.weights or FAMILIES[a.family]["weights"],
                        family=a.family)
        if a.json:
            a.json.write_text(json.dumps(summ, indent=1))
        print(json.dumps({k: v for k, v in summ.items() if k != "rows"}))


if __name__ == "__main__":
    main()
