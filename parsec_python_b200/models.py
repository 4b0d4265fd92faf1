"""Run settings and the records passed between the stages of a run.

Same fields, defaults and override keys as PARSEC.py's rsdft_models.py
(SolverSettings :18-124, InputData :127-148, RunPaths :151-157,
PreparedSystem :160-176, EnergyComponents :220-227, SCFResult :230-246), so
that an input that configures the reference configures this code the same
way.  Keys the reference ignores (``precision``, ``init``, ``seed``) select
options of this implementation.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Callable

A0_ANG = 0.529177210903   # bohr radius in angstrom
RY_EV = 13.605698066      # Rydberg in eV


def _parse_tol(value: Any) -> float:
    """Integers >= 1 mean 10**-value (rsdft_models.py:39-47)."""
    v = float(value)
    if v >= 1 and abs(v - round(v)) < 1e-12:
        return 10 ** (-int(round(v)))
    return v


def _parse_bool(value: Any) -> int:
    if isinstance(value, bool):
        return int(value)
    if isinstance(value, (int, float)):
        return 1 if value else 0
    if isinstance(value, str):
        s = value.strip().lower()
        if s in {"1", "true", "yes", "y", "on"}:
            return 1
        if s in {"0", "false", "no", "n", "off"}:
            return 0
    raise ValueError("invalid boolean value")


@dataclass
class SolverSettings:
    fd_order: int = 8
    maxits: int = 40
    tol: float = 2.0e-4
    fermi_temp: float = 500.0
    save_wfn: int = 0
    cg_prec: int = 0
    poldeg: int = 10
    diagmeth: int = 3
    adaptive_scheme: int = 0
    use_gpu: int = 1
    recenter_atoms: int = 1
    precision: str = "fp64"      # fp64 | mixed
    init: str = "sad"            # sad | learned
    seed: int = 0
    mixed_switch: float = 1e-4   # mixed precision: below this SCF error the block product W T leaves the tensor cores
    mixed_finish: str = "fp64"   # fp64: the last iterations run on FP64 blocks | fp32: the run may end in FP32
    mixed_fp64_at: float = 1e-6  # mixed_finish = fp64: FP64 blocks once the SCF error is below this (or stalls)
    mask: str = "cube"           # cube (the reference's domain) | sphere (H zero outside the inscribed sphere)
    first_tol: float = 0.08      # first_filt: stop when the Ritz trace moves by <= this fraction (first_filt.py:14)
    first_rounds: int = 0        # first_filt: most filter rounds; 0 = the reference's max(min(60 / polm, 5), 3)
    mixer: str = "msecant1"      # msecant1 (the reference's default) | msecant2 (Type-II) | anderson (msecant2, groups of all iterates)
    mix_group_size: int = 0      # msecant2: iterates per group (0 = all of them: Anderson mixing)

    _KEYS = {
        "fd_order": ("fd_order", int), "maxits": ("maxits", int), "tol": ("tol", _parse_tol),
        "fermi_temp": ("fermi_temp", float), "save_wfn": ("save_wfn", _parse_bool),
        "write_wfn": ("save_wfn", _parse_bool), "cg_prec": ("cg_prec", int), "poldeg": ("poldeg", int),
        "diagmeth": ("diagmeth", int), "adaptivescheme": ("adaptive_scheme", int),
        "adaptive_scheme": ("adaptive_scheme", int), "use_gpu": ("use_gpu", _parse_bool),
        "gpu": ("use_gpu", _parse_bool), "recenter_atoms": ("recenter_atoms", _parse_bool),
        "recenter": ("recenter_atoms", _parse_bool), "precision": ("precision", str),
        "init": ("init", str), "seed": ("seed", int), "mixed_switch": ("mixed_switch", float),
        "mixed_finish": ("mixed_finish", str), "mixed_fp64_at": ("mixed_fp64_at", float),
        "mask": ("mask", str), "first_tol": ("first_tol", float), "first_rounds": ("first_rounds", int),
        "mixer": ("mixer", str), "mix_group_size": ("mix_group_size", int),
    }

    def normalize(self) -> None:
        self.fd_order = int(self.fd_order)
        self.maxits = max(1, int(self.maxits))
        self.tol = float(self.tol)
        self.fermi_temp = float(self.fermi_temp)
        self.save_wfn = 1 if int(self.save_wfn) else 0
        self.cg_prec = 1 if int(self.cg_prec) else 0
        self.poldeg = max(1, int(self.poldeg))
        self.diagmeth = int(self.diagmeth)
        self.adaptive_scheme = 1 if int(self.adaptive_scheme) else 0
        self.use_gpu = 1 if int(self.use_gpu) else 0
        self.recenter_atoms = 1 if int(self.recenter_atoms) else 0
        if not 0 <= self.diagmeth <= 3:
            self.diagmeth = 3
        self.precision = str(self.precision).lower()
        if self.precision not in ("fp64", "mixed"):
            self.precision = "fp64"
        self.init = str(self.init).lower()
        if self.init not in ("sad", "learned"):
            self.init = "sad"
        self.mixed_switch = float(self.mixed_switch)
        self.mixer = str(self.mixer).lower()
        if self.mixer == "anderson":
            self.mixer, self.mix_group_size = "msecant2", 0
        if self.mixer not in ("msecant1", "msecant2"):
            self.mixer = "msecant1"
        self.mix_group_size = max(0, int(self.mix_group_size))
        self.mixed_finish = str(self.mixed_finish).lower()
        if self.mixed_finish not in ("fp32", "fp64"):
            self.mixed_finish = "fp64"
        self.mixed_fp64_at = float(self.mixed_fp64_at)
        self.first_tol = float(self.first_tol)
        self.first_rounds = max(0, int(self.first_rounds))
        self.mask = str(self.mask).lower()
        if self.mask not in ("cube", "sphere"):
            self.mask = "cube"

    def apply_overrides(self, overrides: dict[str, Any] | None) -> dict[str, Any]:
        """Apply known keys (case-insensitive), drop unknown ones, return what changed."""
        applied: dict[str, Any] = {}
        for raw_key, raw_value in (overrides or {}).items():
            if raw_value is None:
                continue
            key = str(raw_key).strip()
            target = self._KEYS.get(key) or self._KEYS.get(key.lower())
            if target is None:
                continue
            name, cast = target
            try:
                value = cast(raw_value)
            except (TypeError, ValueError):
                print(f"Warning: Could not parse value for {raw_key}, keeping current setting.")
                continue
            setattr(self, name, value)
            applied[name] = value
        self.normalize()
        return applied


@dataclass
class InputData:
    atoms: list[dict[str, Any]]
    n_atom: list[int]
    z_charge: float
    density_method: str = "sad"
    ml_file_path: str | None = None
    settings_overrides: dict[str, Any] = field(default_factory=dict)
    input_file_path: str | None = None
    grid_npy_path: str | None = None
    grid_poscar_path: str | None = None
    unit_used: str = "bohr"
    grid_mode: str = "default"
    grid_data: dict[str, Any] | None = None


@dataclass
class RunPaths:
    output_file: str
    wfn_file: str
    initial_density_base: str
    converged_density_base: str


@dataclass
class PreparedSystem:
    input_data: InputData
    settings: SolverSettings
    domain: dict[str, Any]
    h: float
    nev: int
    zelec: float
    ztest: float
    n_types: int
    paths: RunPaths


@dataclass
class SolverBackend:
    """GPU implementation bundle with the reference's entry-point names
    (rsdft_models.py:179-217) plus the stages the reference imports directly
    (XC, mixer, Laplacian, density, potential update)."""
    label: str
    pseudo_diag: Callable[..., Any]
    pseudo_nl: Callable[..., Any]
    first_filt: Callable[..., Any]
    chefsi1: Callable[..., Any]
    lanczos: Callable[..., Any]
    chsubsp: Callable[..., Any]
    occupations: Callable[..., Any]
    pcg: Callable[..., Any]
    array_module: Any
    cupy_module: Any | None = None
    runtime: Any = None

    def to_numpy_array(self, value: Any) -> Any:
        import numpy as np
        import torch

        if isinstance(value, torch.Tensor):
            return value.detach().cpu().numpy()
        if hasattr(value, "to_numpy"):
            return value.to_numpy()
        return np.asarray(value) if value is not None else value

    def to_host_scalar(self, value: Any) -> Any:
        import numpy as np
        import torch

        if isinstance(value, torch.Tensor):
            return value.item()
        if isinstance(value, np.ndarray) and value.ndim == 0:
            return value.item()
        if isinstance(value, np.generic):
            return value.item()
        return value


@dataclass
class EnergyComponents:
    eigen_sum_ry: float
    hartree_ry: float
    xc_ry: float
    ion_ry: float
    total_ry: float


@dataclass
class SCFResult:
    rho: Any
    hpot: Any
    xc_potential: Any
    exc: float
    potential: Any
    wavefunctions: Any
    eigenvalues: Any
    occupations: Any
    iterations: int
    error: float
    converged: bool
    e_nuc0: float
    hpot0: Any
    n_atoms: int
    timings: dict[str, float] = field(default_factory=dict)
    history: list[dict[str, Any]] = field(default_factory=list)
