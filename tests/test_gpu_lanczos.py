"""GPU parity of the Lanczos-based eigensolvers (diagmeth 0/1/2) against the
oracle, which tests/test_oracle_golden.py pins to the reference's own
lanczosForChsubsp.py, chsubsp.py and lanczos.py.

The Lanczos recurrence from the same start vector is compared step by step
(FP64, until loss of orthogonality lets the last bits wander); the
tridiagonal eigensolver against LAPACK on tridiagonals with Lanczos ghosts,
exact ties and wide spreads; the drivers by the Ritz values they return;
whole SCFs with diagmeth 2, 0 and 1 by their converged energies against the
reference's diagmeth-2 SCF (1e-5 Ha bar)."""
import json

import numpy as np
import pytest
import scipy.linalg
import scipy.sparse as sp

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parsec_python_b200 import gpu  # noqa: E402
from parsec_python_b200._lib import F64  # noqa: E402
from parsec_python_b200.backend import select_solver_backend  # noqa: E402
from parsec_python_b200.inputs import ElementTable, pseudo_tables  # noqa: E402
from parsec_python_b200.models import A0_ANG, SolverSettings  # noqa: E402
from parsec_python_b200.solver import run_rsdft_calculation  # noqa: E402
from parsec_python_b200.system import system_from_atoms  # noqa: E402

DEV = torch.device("cuda", 0)
H2O = [{"typ": "O", "coord": np.array([[0.0, 0.0, 0.0]]) / A0_ANG},
       {"typ": "H", "coord": np.array([[0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]) / A0_ANG}]


@pytest.fixture(scope="module")
def lz(golden_dir):
    return np.load(golden_dir / "ref_lanczos.npz"), json.loads((golden_dir / "ref_lanczos.json").read_text())


def _systems(dom, g, tag):
    """The same H2O Hamiltonian on the GPU and as the oracle's CSR matrix."""
    ctx = gpu.GridContext(dom, 8)
    rho0, hpot0, ppot, _ = gpu.sad_setup(ctx, H2O, ElementTable(), pseudo_tables())
    gpu.projector_setup(ctx, H2O, ElementTable(), pseudo_tables())
    pot = ppot + hpot0
    np.testing.assert_array_equal(pot.cpu().numpy(), g[f"{tag}_pot"])
    H = gpu.Hamiltonian(ctx, pot)
    n = ctx.n
    elements, tab = O.load_elements(), O.load_tables()
    vnl = O.nonlocal_csr(O.projectors(dom, H2O, elements, tab), n)
    B = (0.5 * O.laplacian(dom, 8) + vnl + sp.diags(g[f"{tag}_pot"], 0, shape=(n, n))).tocsr()
    return ctx, H, B


@pytest.fixture(scope="module")
def small(lz):
    g, meta = lz
    return _systems(meta["small"]["domain"], g, "small")


def test_lanczos_recurrence_matches_oracle(small, lz):
    g, _ = lz
    ctx, H, B = small
    m = 60
    VV, ab, k, rr = gpu.lanczos_krylov(H, 27, m, 0, v=g["small_v"])
    a = ab.cpu().numpy()
    _, alpha, beta, _, rr_o, _ = O.lanczos_krylov(B, g["small_v"], m, 27, 0)
    scale = np.abs(alpha).max()
    # identical recurrence: agreement to rounding while the basis is still
    # nearly orthogonal, then the two runs drift apart at the rounding level
    assert np.abs(a[0:40:2] - alpha[:20]).max() < 1e-11 * scale
    assert np.abs(a[1:40:2] - beta[:20]).max() < 1e-11 * scale
    assert np.abs(a[0::2] - alpha).max() < 1e-6 * scale
    # the extreme Ritz values of T_60 agree to far below the 1e-5 Ha bar
    assert np.abs(rr[:4] - rr_o[:4]).max() < 1e-8
    assert abs(rr[-1] - rr_o[-1]) < 1e-8 * abs(rr_o[-1])
    # the stored basis is the normalised recurrence
    v = VV[:k].cpu().numpy()
    np.testing.assert_allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-13)
    assert ctx.status()[0] == 0


def _tridiag(alpha, beta):
    return np.diag(alpha) + np.diag(beta, 1) + np.diag(beta, -1)


def _ghosted(m, seed):
    """Lanczos tridiagonal of a matrix with a few well-separated extreme
    eigenvalues and no reorthogonalisation: the converged ones reappear as
    ghosts (near-identical eigenvalues of T)."""
    rng = np.random.default_rng(seed)
    d = np.concatenate([[-3.0, -2.0, -1.99999], np.linspace(0.0, 1.0, 400), [5.0]])
    n = d.size
    v = rng.standard_normal(n)
    v /= np.linalg.norm(v)
    v0 = np.zeros(n)
    bet = 0.0
    al, be = np.zeros(m), np.zeros(m)
    for j in range(m):
        w = d * v - bet * v0
        al[j] = v @ w
        w -= al[j] * v
        bet = np.linalg.norm(w)
        be[j] = bet
        v0, v = v, w / bet
    return al, be


CASES = {
    "random": lambda: (np.random.default_rng(1).standard_normal(300), np.random.default_rng(2).standard_normal(300)),
    "ghosts": lambda: _ghosted(350, 3),
    "wide": lambda: (np.concatenate([np.linspace(-1, 1, 100), [1e4]]), np.full(101, 1e-3)),
    "tiny_offdiag": lambda: (np.repeat([1.0, 2.0, 3.0], 40), np.full(120, 1e-12)),
    "one": lambda: (np.array([0.7]), np.array([0.3])),
    "two": lambda: (np.array([1.0, 1.0]), np.array([1e-9, 0.0])),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tridiagonal_eigensolver_vs_lapack(name):
    alpha, beta = CASES[name]()
    k = alpha.size
    ab = np.zeros(2 * k)
    ab[0::2], ab[1::2] = alpha, beta[:k]
    T = _tridiag(alpha, beta[:k - 1])
    w_ref, z_ref = scipy.linalg.eigh(T)
    ctx = gpu.GridContext({"nx": 4, "ny": 4, "nz": 4, "h": 1.0, "radius": 1.0}, 8)
    nvec = min(k, 150)
    abd = torch.from_numpy(ab).to(DEV)
    ev = torch.empty(k, dtype=torch.float64, device=DEV)
    Z = torch.empty(nvec, k, dtype=torch.float64, device=DEV)
    ctx.call("psc_tridiag_eig", gpu._p(abd), k, nvec, gpu._p(ev), gpu._p(Z), k, gpu._stream())
    w = ev.cpu().numpy()
    z = Z.cpu().numpy().T
    tn = max(np.abs(w_ref).max(), 1e-300)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - w_ref).max() <= 8e-15 * k * tn
    # eigenvectors: small residuals, orthonormal, and for well-separated
    # eigenvalues the LAPACK vector up to sign
    res = np.abs(T @ z - z * w[:nvec]).max()
    assert res <= 1e-12 * tn
    assert np.abs(z.T @ z - np.eye(nvec)).max() < 1e-9
    gaps = np.minimum(np.diff(np.r_[-np.inf, w_ref]), np.diff(np.r_[w_ref, np.inf]))[:nvec]
    sep = gaps > 1e-3 * tn
    dots = np.abs(np.sum(z[:, sep] * z_ref[:, :nvec][:, sep], axis=0))
    np.testing.assert_allclose(dots, 1.0, atol=1e-9)


def test_orthonormalize_rank_drops_copies():
    """Columns that repeat (up to 1e-12) earlier ones are dropped; the kept
    block is orthonormal and spans the original columns."""
    ctx = gpu.GridContext({"nx": 20, "ny": 20, "nz": 20, "h": 0.5, "radius": 4.75}, 8)
    n = ctx.n
    rng = np.random.default_rng(4)
    base = rng.standard_normal((n, 10))
    cols = [base[:, i] for i in range(10)]
    cols.insert(3, base[:, 1] * 2.0 + 1e-12 * rng.standard_normal(n))   # near copy
    cols.insert(7, base[:, 0] - base[:, 2])                               # exact combination
    X = np.stack(cols, axis=1)
    W = torch.from_numpy(np.ascontiguousarray(X.T)).to(DEV)
    T = torch.empty_like(W)
    rank, which = gpu.c_int(), gpu.c_int()
    ctx.call("psc_orthonormalize_rank", F64, gpu._p(W), gpu._p(T), n, X.shape[1], 1e-10, gpu.byref(rank),
             gpu.byref(which), gpu._stream())
    assert rank.value == 10
    Q = (T if which.value else W)[:10].cpu().numpy().T
    assert np.abs(Q.T @ Q - np.eye(10)).max() < 1e-13
    # the span of the original columns
    resid = X - Q @ (Q.T @ X)
    assert np.abs(resid).max() < 1e-9 * np.abs(X).max()


@pytest.mark.parametrize("tag", ["small", "big"])
def test_lanczos_for_chsubsp_matches_reference(lz, tag):
    """Same start vector as the reference run; both branches (convergence
    test on for n = 13824, off for n = 39304).  The occupied Ritz values
    (4 for H2O) match the reference's to 1e-8 Ha, the bound to 1e-8."""
    g, meta = lz
    ctx, H, B = _systems(meta[tag]["domain"], g, tag)
    W, lam, bound = gpu.lanczos_for_chsubsp(H, 27, 450, v=g[f"{tag}_v"])
    lam_ref = g[f"{tag}_lfc_lam"]
    lam_h = lam.cpu().numpy()
    assert np.abs(lam_h[:4] - lam_ref[:4]).max() < 1e-8
    # bound = max|theta| + beta_k.  The top Ritz value is converged and agrees
    # with the oracle's to rounding; beta_k after 450 steps without
    # reorthogonalisation is chaotic (a 1e-15 change of the start vector moves
    # it by 2 %), so the bound itself agrees with the reference's only to that
    _, ab, k, rr = gpu.lanczos_krylov(H, 27, 450, 0 if ctx.n > 35000 else 1, v=g[f"{tag}_v"])
    _, _, _, k_o, rr_o, _ = O.lanczos_krylov(B, g[f"{tag}_v"], 450, 27, 0 if ctx.n > 35000 else 1)
    assert k == k_o
    assert abs(np.abs(rr).max() - np.abs(rr_o).max()) < 1e-10 * np.abs(rr_o).max()
    assert np.abs(rr).max() < bound < 1.5 * np.abs(rr).max()
    assert abs(bound - float(g[f"{tag}_lfc_bound"])) < 0.05 * abs(bound)
    # orthonormal block whose Rayleigh quotients are the returned Ritz values
    w = W.cpu().numpy()
    assert np.abs(w @ w.T - np.eye(27)).max() < 1e-12
    HW = (H @ W).cpu().numpy()
    np.testing.assert_allclose(np.sum(w * HW, axis=1), lam_h, atol=1e-10)
    rho4 = (w[:4] ** 2).sum(0)
    assert np.abs(rho4 - g[f"{tag}_lfc_rho4"]).sum() < 1e-6 * rho4.sum()
    assert ctx.status()[0] == 0


def test_chsubsp_and_lanczos_drivers(lz, small):
    g, meta = lz
    ctx, H, B = small
    W, ritz = gpu.chsubsp(10, 27, H)
    r = ritz.cpu().numpy()
    ref = g["small_ch_ritz"]
    # chsubsp stops at a 5 % trace change, so only the occupied values are
    # converged tightly (the reference run drew a different start vector)
    assert np.abs(r[:4] - ref[:4]).max() < 1e-6
    w = W.cpu().numpy()
    assert np.abs(w @ w.T - np.eye(27)).max() < 1e-12
    big_ctx, Hb, _ = _systems(meta["big"]["domain"], g, "big")
    Wl, laml = gpu.lanczos(Hb, 27, g["big_lz_v"], 512, 1e-5)
    assert np.abs(laml.cpu().numpy()[:4] - g["big_lz_lam"][:4]).max() < 1e-8
    rho4 = (Wl.cpu().numpy()[:4] ** 2).sum(0)
    assert np.abs(rho4 - g["big_lz_rho4"]).sum() < 1e-6 * rho4.sum()


def _scf(diagmeth, tol=1e-6, precision="fp64"):
    dom = {"h": 0.3 / A0_ANG}
    s = SolverSettings(tol=tol, poldeg=10, maxits=60, diagmeth=diagmeth, precision=precision)
    s.normalize()
    elem = ElementTable()
    prob = system_from_atoms(H2O, h=dom["h"], radius=4.0 / A0_ANG, nev=12, settings=s, elem=elem)
    return prob, run_rsdft_calculation(prob, elem, len(elem), select_solver_backend(s), verbose=False)


@pytest.mark.parametrize("diagmeth", [2, 0, 1])
def test_scf_diagmeth_matches_reference(lz, diagmeth):
    """The reference's diagmeth-2 SCF on the 28^3 H2O box converges to
    E = -37.5921138 Ry; every Lanczos-started path reaches it within 1e-5 Ha."""
    g, meta = lz
    ms = meta["scf_diagmeth2"]
    prob, res = _scf(diagmeth)
    assert prob.domain == ms["domain"]
    assert res.converged
    e = res.history[-1]["total_ry"]
    assert abs(e - ms["total_ry"]) < 2e-5, (e, ms["total_ry"])
    assert np.abs(res.eigenvalues[:4] - g["scf2_eigenvalues"][:4]).max() < 1e-5
    h = prob.domain["h"]
    drho = np.abs(res.rho.cpu().numpy() - g["scf2_rho"]).sum() * h ** 3
    assert drho < 1e-4, drho
    assert res.history[0]["lam"].shape[0] == 27
