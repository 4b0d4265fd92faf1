"""GPU parity of the libpsc kernels against the oracle and the reference's own
outputs (tests/golden).  Integer/index work and the SAD setup must be
bit-exact; FP64 operator applications within 1e-12 relative."""
import hashlib
import json

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected on CPU runs
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parsec_python_b200 import _lib, gpu, workloads  # noqa: E402
from parsec_python_b200._lib import F32, F64  # noqa: E402
from parsec_python_b200.inputs import ElementTable, pseudo_tables  # noqa: E402

DEV = torch.device("cuda", 0)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def block(x):
    """(n, k) host array -> (k, n) device block (n x k column-major)."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x).T)).to(DEV)


def host(t):
    return t.cpu().numpy().T


@pytest.fixture(scope="module")
def meta(golden_dir):
    return json.loads((golden_dir / "ref_meta.json").read_text())


@pytest.fixture(scope="module")
def h2o_box(meta):
    mi = meta["ion_h2o"]
    atoms = [{"typ": t, "coord": np.array(c)} for t, c in mi["atoms"]]
    ctx = gpu.GridContext(mi["domain"], 8)
    return ctx, atoms, mi


def test_laplacian_matches_reference_fd3d(golden_dir):
    fd = np.load(golden_dir / "ref_fd3d.npz")
    for key in fd.files:
        if not key.startswith("x_"):
            continue
        nx, ny, nz, order = map(int, key[2:].split("_"))
        dom = {"nx": nx, "ny": ny, "nz": nz, "h": 1.0, "radius": 1.0}
        ctx = gpu.GridContext(dom, order)
        y = host(gpu.Laplacian(ctx) @ block(fd[key]))
        assert rel(y, fd["y_" + key[2:]]) < 1e-14, key


def test_sad_setup_bit_exact_vs_reference(h2o_box):
    ctx, atoms, mi = h2o_box
    rho0, hpot0, ppot, info = gpu.sad_setup(ctx, atoms, ElementTable(), pseudo_tables())
    assert sha(rho0.cpu().numpy()) == mi["rho0"]
    assert sha(hpot0.cpu().numpy()) == mi["hpot0"]
    assert sha(ppot.cpu().numpy()) == mi["ppot"]
    assert info["electron_count_initial"] == mi["info"]["electron_count_initial"]


def test_sad_density_of_shipped_sample_bit_exact(meta):
    f = 1.0 / O.A0_ANG
    o = np.array([[-3.56626, 1.77639, 0.0]]) * f
    hh = np.array([[-2.59626, 1.77639, 0.0], [-3.88959, 1.36040, -0.81444]]) * f
    c = np.mean(np.vstack([o, hh]), axis=0)
    atoms = [{"typ": "O", "coord": o - c}, {"typ": "H", "coord": hh - c}]
    dom = O.build_system(atoms, h=0.2 * f, radius=5.0 * f)
    ctx = gpu.GridContext(dom, 8)
    rho0 = gpu.sad_setup(ctx, atoms, ElementTable(), pseudo_tables())[0].cpu().numpy()
    grid = rho0.reshape((dom["nx"],) * 3, order="F")
    assert sha(grid) == meta["sample_h2o_init_rho_grid"]["sha256"]


def test_projector_tables_bit_exact_vs_oracle(h2o_box):
    ctx, atoms, mi = h2o_box
    nl = gpu.projector_setup(ctx, atoms, ElementTable(), pseudo_tables())
    ref = O.projectors(mi["domain"], atoms, O.load_elements(), O.load_tables())
    off, idx, u, w = nl.tables()
    assert nl.n_atoms == len(ref)
    for a, pr in enumerate(ref):
        np.testing.assert_array_equal(idx[off[a]:off[a + 1]], pr["idx"])
        np.testing.assert_array_equal(u[:, off[a]:off[a + 1]], pr["u"])


def _csr_h(mi, pot, elements=None):
    dom = mi["domain"]
    n = dom["nx"] ** 3
    atoms = [{"typ": t, "coord": np.array(c)} for t, c in mi["atoms"]]
    projs = O.projectors(dom, atoms, O.load_elements(), O.load_tables())
    return (0.5 * O.laplacian(dom, 8) + O.nonlocal_csr(projs, n) + sp.diags(pot, 0, shape=(n, n))).tocsr()


def test_hamiltonian_fp64_matches_reference_operator(h2o_box, golden_dir):
    ctx, atoms, mi = h2o_box
    gpu.projector_setup(ctx, atoms, ElementTable(), pseudo_tables())
    ev = np.load(golden_dir / "ref_eigs.npz")
    pot = ev["pot"]
    H = gpu.Hamiltonian(ctx, torch.from_numpy(pot).to(DEV))
    B = _csr_h(mi, pot)
    rng = np.random.default_rng(3)
    for k in (1, 7, 27):
        X = rng.standard_normal((ctx.n, k))
        Y = host(H @ block(X))
        assert rel(Y, B @ X) < 1e-12, k
    # the reference's own V_nl (the pseudoNL_original matrix times vnl_x)
    # against the projector apply alone
    ion = np.load(golden_dir / "ref_ion_h2o.npz")
    X, ref = ion["vnl_x"], ion["vnl_y"]
    Xd = block(X)
    Yd = torch.full_like(Xd, float("nan"))
    k = Xd.shape[0]
    ctx.call("psc_apply_nonlocal", F64, gpu._p(Xd), ctx.n, gpu._p(Yd), ctx.n, k, gpu._stream())
    vnl = host(Yd)
    assert np.abs(vnl - ref).max() <= 1e-12 * np.abs(ref).max()


def test_hamiltonian_matches_reference_csr_on_h2o_grid(golden_dir):
    """H X on the H2O configuration's own grid (52^3, 0.2 A, O-H projectors)
    against the reference's assembled CSR B = 0.5 A + V_nl + diag(pot)
    (rsdft_solver.py:263,285) applied to the same seeded columns, FP64, to
    1e-12 of the largest entry; FP32 blocks to FP32 rounding."""
    ref = np.load(golden_dir / "ref_hx_h2o.npz")
    cfg = workloads.config_system("h2o")
    dom = O.build_system(cfg["atoms"], h=cfg["h"], radius=cfg["radius"])
    assert dom["nx"] == int(ref["nx"]) == 52 and abs(dom["h"] - float(ref["h"])) < 1e-15
    ctx = gpu.GridContext(dom, 8)
    gpu.projector_setup(ctx, cfg["atoms"], ElementTable(), pseudo_tables())
    H = gpu.Hamiltonian(ctx, torch.from_numpy(ref["pot"]).to(DEV))
    X = np.random.default_rng(11).standard_normal((ctx.n, 2))
    y = ref["y"]
    for impl in (0, 1):
        ctx.call("psc_set_stencil_impl", impl)
        got = host(H @ block(X))
        assert np.abs(got - y).max() <= 1e-12 * np.abs(y).max(), impl
        got32 = host(H @ block(X).float()).astype(np.float64)
        assert np.abs(got32 - y).max() <= 2e-6 * np.abs(y).max(), impl
    ctx.check_status()


def test_hamiltonian_fp32(h2o_box, golden_dir):
    ctx, atoms, mi = h2o_box
    gpu.projector_setup(ctx, atoms, ElementTable(), pseudo_tables())
    pot = np.load(golden_dir / "ref_eigs.npz")["pot"]
    H = gpu.Hamiltonian(ctx, torch.from_numpy(pot).to(DEV))
    X = np.random.default_rng(4).standard_normal((ctx.n, 9))
    y64 = host(H @ block(X))
    y32 = host(H @ block(X).float()).astype(np.float64)
    assert rel(y32, y64) < 2e-5


@pytest.mark.parametrize("mode", [0, 1])
def test_chebyshev_filter_matches_oracle(h2o_box, golden_dir, mode):
    ctx, atoms, mi = h2o_box
    gpu.projector_setup(ctx, atoms, ElementTable(), pseudo_tables())
    pot = np.load(golden_dir / "ref_eigs.npz")["pot"]
    H = gpu.Hamiltonian(ctx, torch.from_numpy(pot).to(DEV))
    B = _csr_h(mi, pot)
    X = np.random.default_rng(5).standard_normal((ctx.n, 11))
    lam1, lo, hi = -1.2, 0.4, 60.0
    bounds = torch.tensor([lam1, lo, hi], dtype=torch.float64, device=DEV)
    for deg in (1, 2, 10):
        W = block(X)
        R, _ = gpu.cheb_filter(H, W, torch.empty_like(W), deg, bounds, mode)
        ref = O.ch_filter(B, X, deg, lam1, lo, hi) if mode == 0 else O.cheb_filter_slim(B, X, deg, lo, hi)
        assert rel(host(R), ref) < 1e-11, (mode, deg)


def test_dense_building_blocks():
    dom = {"nx": 20, "ny": 20, "nz": 20, "h": 0.5, "radius": 4.75}
    ctx = gpu.GridContext(dom, 8)
    rng = np.random.default_rng(6)
    for k in (6, 27, 55, 130, 151, 200, 307):  # Cholesky + inverse on chip up to 151, blocked beyond
        W = rng.standard_normal((ctx.n, k))
        V = rng.standard_normal((ctx.n, k))
        g = ctx.empty(k, k)
        Vd, Wd = block(V), block(W)  # keep the device buffers alive across the call
        ctx.call("psc_gram", F64, gpu._p(Vd), ctx.n, gpu._p(Wd), ctx.n, k, 0, gpu._p(g), gpu._stream())
        G = g.cpu().numpy().T
        assert rel(G, V.T @ W) < 1e-13
        # symmetric eigensolver (k x k FP64)
        S = rng.standard_normal((k, k))
        S = S + S.T
        A = torch.from_numpy(np.asfortranarray(S).ravel(order="F").copy()).to(DEV)
        ev, vec = ctx.empty(k), ctx.empty(k * k)
        ctx.call("psc_syev", gpu._p(A), k, gpu._p(ev), gpu._p(vec), gpu._stream())
        lam = ev.cpu().numpy()
        Q = vec.cpu().numpy().reshape(k, k).T
        ref = np.linalg.eigvalsh(S)
        assert np.abs(lam - ref).max() < 1e-12 * np.abs(ref).max()
        assert np.abs(S @ Q - Q * lam).max() < 1e-11 * np.abs(ref).max()
        assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-12
        # CholeskyQR2 keeps the span and gives orthonormal columns
        Wb = block(W)
        R, _ = gpu.orthonormalize(ctx, Wb, torch.empty_like(Wb))
        Qw = host(R)
        assert np.abs(Qw.T @ Qw - np.eye(k)).max() < 1e-13
        P = Qw @ (Qw.T @ W)
        assert rel(P, W) < 1e-12
        # W Q
        Qm = rng.standard_normal((k, k))
        out = ctx.empty(k, ctx.n)
        Qd = torch.from_numpy(Qm.ravel(order="F").copy()).to(DEV)
        ctx.call("psc_gemm_nn", F64, gpu._p(Wd), ctx.n, k, gpu._p(Qd), k, gpu._p(out), ctx.n, gpu._stream())
        assert rel(host(out), W @ Qm) < 1e-13


@pytest.mark.parametrize("k", [8, 160])
def test_cholesky_flags_rank_deficient_block(k):
    """A zero column makes its Cholesky pivot exactly 0: status word 1 names
    it (column 3 -> 4), on chip (k = 8) and in the blocked form (k = 160)."""
    dom = {"nx": 20, "ny": 20, "nz": 20, "h": 0.5, "radius": 4.75}
    ctx = gpu.GridContext(dom, 8)
    W = np.random.default_rng(k).standard_normal((ctx.n, k))
    W[:, 3] = 0.0
    Wd = block(W)
    ctx.status(clear=True)
    gpu.orthonormalize(ctx, Wd, torch.empty_like(Wd), passes=1)
    assert ctx.status()[1] == 4


@pytest.mark.parametrize("k,kind", [(1, "rand"), (2, "rand"), (3, "rand"), (7, "rand"), (55, "diag"),
                                    (56, "degenerate"), (64, "zero"), (111, "rand"), (143, "neardiag"),
                                    (200, "neardiag"), (307, "rand"), (1024, "neardiag")])
def test_syev_edge_cases(k, kind):
    """Householder + bisection + inverse iteration eigensolver: orders with
    no reflector (1, 2) and one (3), the four reductions (one CTA of 256
    threads up to k = 96, of 512 up to 153 with the matrix on chip, a cluster
    of 8 CTAs holding it in their shared memory up to about k = 420 (200,
    307), one CTA with it in global scratch beyond), the widest block (1024), an input that is already
    diagonal (every reflector the identity), eigenvalues of multiplicity 14
    and 28 (one inverse-iteration cluster each), the zero matrix, nearly
    diagonal RR matrices."""
    ctx = gpu.GridContext({"nx": 8, "ny": 8, "nz": 8, "h": 0.5, "radius": 1.75}, 8)
    rng = np.random.default_rng(k)
    if kind == "rand":
        S = rng.standard_normal((k, k))
        S = S + S.T
    elif kind == "diag":
        S = np.diag(rng.standard_normal(k))
    elif kind == "degenerate":
        Q, _ = np.linalg.qr(rng.standard_normal((k, k)))
        S = (Q * np.repeat([1.0, 2.0, -3.0, 2.0], k // 4)) @ Q.T
    elif kind == "zero":
        S = np.zeros((k, k))
    else:
        S = np.diag(np.sort(rng.standard_normal(k))) + 1e-4 * rng.standard_normal((k, k))
        S = 0.5 * (S + S.T)
    A = torch.from_numpy(np.asfortranarray(S).ravel(order="F").copy()).to(DEV)
    ev, vec = ctx.empty(k), ctx.empty(k * k)
    ctx.call("psc_syev", gpu._p(A), k, gpu._p(ev), gpu._p(vec), gpu._stream())
    assert not any(ctx.status())
    lam = ev.cpu().numpy()
    Q = vec.cpu().numpy().reshape(k, k).T
    ref = np.linalg.eigvalsh(S)
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(lam - ref).max() < 1e-12 * scale
    assert np.abs(S @ Q - Q * lam).max() < 1e-11 * scale
    assert np.abs(Q.T @ Q - np.eye(k)).max() < 1e-12


@pytest.mark.parametrize("shape,k", [((30, 28, 26), 27), ((40, 40, 40), 55), ((33, 31, 29), 128),
                                     ((24, 24, 24), 143), ((21, 20, 19), 300)])
def test_gram_pair_tensor_cores_match_fp64(shape, k):
    """FP32 Gram pair on tcgen05 (3xTF32, FP32 accumulation in tensor memory
    per chunk of rows, FP64 across chunks) and on the FP64 tensor cores
    (exact products, FP64 sums), against FP64 products of the same FP32
    values; odd n
    exercises the scalar-load edge.  The tensor-core bound 2e-5 (relative to
    the largest entry) is the FP32 accumulation over a chunk of a few hundred
    rows; the products themselves are exact."""
    nx, ny, nz = shape
    ctx = gpu.GridContext({"nx": nx, "ny": ny, "nz": nz, "h": 0.4, "radius": 0.2 * (nx - 1)}, 8)
    n = ctx.n
    rng = np.random.default_rng(k)
    W = rng.standard_normal((k, n)).astype(np.float32)
    V = (W * 0.3 + rng.standard_normal((k, n)).astype(np.float32)).astype(np.float32)
    Wd, Vd = torch.from_numpy(W).to(DEV), torch.from_numpy(V).to(DEV)
    W64, V64 = W.astype(np.float64), V.astype(np.float64)
    S_ref, K_ref = W64 @ W64.T, W64 @ V64.T
    out = {}
    for impl in (1, 0):
        ctx.call("psc_set_gram_impl", impl)
        S, K = ctx.empty(k, k), ctx.empty(k, k)
        ctx.call("psc_gram_pair", F32, gpu._p(Wd), gpu._p(Vd), n, k, gpu._p(S), gpu._p(K), gpu._stream())
        out[impl] = (S.cpu().numpy().T, K.cpu().numpy().T)
    assert ctx.status()[5] == 0
    # both paths return symmetric matrices: K = 0.5 (K + K^T) inside the
    # diagonal tiles, and the off-diagonal tiles formed above the diagonal
    # only and mirrored (128-column tiles on tcgen05, 64-column tiles on the
    # FP64 tensor cores); V here is not H W, so K itself is not symmetric
    def tiled(width):
        K_t = 0.5 * (K_ref + K_ref.T)
        t = np.arange(k) // width
        off = t[:, None] < t[None, :]
        K_t[off] = K_ref[off]
        K_t.T[off] = K_ref[off]
        return K_t
    for impl, (S, K) in out.items():
        tol = 2e-5 if impl == 1 else 1e-12
        assert np.abs(S - S_ref).max() <= tol * np.abs(S_ref).max(), impl
        assert np.abs(K - tiled(128 if impl == 1 else 64)).max() <= tol * np.abs(K_ref).max(), impl
        assert np.array_equal(S, S.T) and np.array_equal(K, K.T)
        # the diagonals (column norms, Rayleigh quotients) are FP64 sums on
        # both paths: no bias from the tensor cores' FP32 accumulation
        assert rel(np.diag(S), np.diag(S_ref)) < 1e-13, impl
        assert np.abs(np.diag(K) - np.diag(K_ref)).max() < 1e-13 * np.abs(K_ref).max(), impl


@pytest.mark.parametrize("shape,k,kout", [((30, 28, 26), 27, 27), ((40, 40, 40), 55, 55), ((24, 24, 24), 143, 143),
                                          ((40, 40, 40), 307, 307), ((21, 20, 19), 300, 260),
                                          ((16, 16, 16), 64, 30), ((12, 12, 12), 5, 3), ((33, 31, 29), 55, 40)])
def test_block_product_tensor_cores_match_fp64(shape, k, kout):
    """FP32 block product Out = W T (the Rayleigh-Ritz W R^{-1} Y) on tcgen05
    (3xTF32, FP32 accumulation over k) and on the FP64 tensor cores (exact
    products, FP64 sums, one rounding), against the FP64 product of the same
    FP32 W and FP64 T.  kout > 256 uses the second accumulator; an odd n
    (33 x 31 x 29) takes the FP64 tensor-core path.  Bound 2e-5 of the
    largest entry for tcgen05 (the FP32 accumulation over k terms), FP32
    rounding of the result for the FP64 tensor cores."""
    nx, ny, nz = shape
    ctx = gpu.GridContext({"nx": nx, "ny": ny, "nz": nz, "h": 0.4, "radius": 0.2 * (nx - 1)}, 8)
    n = ctx.n
    rng = np.random.default_rng(k + kout)
    W = rng.standard_normal((k, n)).astype(np.float32)
    T = rng.standard_normal((k, kout)) / np.sqrt(k)
    Wd = torch.from_numpy(W).to(DEV)
    Td = torch.from_numpy(np.ascontiguousarray(T.T)).to(DEV)        # column-major k x kout, ld k
    ref = W.astype(np.float64).T @ T                                # n x kout
    for impl, tol in ((1, 2e-5), (0, 1.2e-7)):
        ctx.call("psc_set_gemm_impl", impl)
        out = torch.full((kout, n), np.nan, dtype=torch.float32, device=DEV)
        for _ in range(2):   # twice: the second call reuses the split T buffer
            ctx.call("psc_gemm_nn", F32, gpu._p(Wd), n, k, gpu._p(Td), kout, gpu._p(out), n, gpu._stream())
        got = out.cpu().numpy().T.astype(np.float64)
        assert np.isfinite(got).all(), impl
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (impl, np.abs(got - ref).max() / np.abs(ref).max())
    assert ctx.status()[6] == 0


def test_occupations_match_reference(golden_dir):
    oc = np.load(golden_dir / "ref_occupations.npz")
    ctx = gpu.GridContext({"nx": 8, "ny": 8, "nz": 8, "h": 0.5, "radius": 1.75}, 8)
    for i in range(4):
        lam = torch.from_numpy(oc[f"lam_{i}"].copy()).to(DEV)
        ef, occ = gpu.occupations(ctx, lam, 500.0, float(oc[f"ne_{i}"]), 1e-6)
        assert abs(ef.item() - float(oc[f"ef_{i}"])) < 1e-12
        assert np.abs(occ.cpu().numpy() - oc[f"occ_{i}"]).max() < 1e-12


def test_xc_matches_reference(golden_dir):
    xc = np.load(golden_dir / "ref_xc.npz")
    n = xc["rho"].size
    ctx = gpu.GridContext({"nx": n, "ny": 1, "nz": 1, "h": 0.37, "radius": 1.0}, 8)
    vxc, out = gpu.lda_xc(ctx, torch.from_numpy(xc["rho"]).to(DEV))
    assert rel(vxc.cpu().numpy(), xc["vxc"]) < 1e-13
    o = out.cpu().numpy()
    assert abs(o[0] - float(xc["exc"])) < 1e-12 * abs(float(xc["exc"]))
    assert o[1] == xc["rho"].max() and o[2] == xc["rho"].min()


def test_mixer_matches_reference_including_restart(golden_dir):
    mx = np.load(golden_dir / "ref_mixer.npz")
    n = mx["x"].shape[1]
    ctx = gpu.GridContext({"nx": n, "ny": 1, "nz": 1, "h": 1.0, "radius": 1.0}, 8)
    m = gpu.Mixer(ctx, capacity=20)
    for i in range(len(mx["x"])):
        out, _ = m(torch.from_numpy(mx["x"][i]).to(DEV), torch.from_numpy(mx["f"][i]).to(DEV))
        assert rel(out.cpu().numpy(), mx["out"][i]) < 1e-11, i


@pytest.mark.parametrize("name,group_size", [("anderson", 0), ("group2", 2)])
def test_mixer2_matches_reference_including_restart(golden_dir, name, group_size):
    """Type-II multisecant mixer on the device (history in HBM, libpsc
    kernels; Anderson for group size 0) against the reference's msecant2
    outputs, through the restart and the alternating EN stages after it."""
    g = np.load(golden_dir / "ref_mixer2.npz")
    n = g[f"{name}_x"].shape[1]
    ctx = gpu.GridContext({"nx": n, "ny": 1, "nz": 1, "h": 1.0, "radius": 1.0}, 8)
    m = gpu.Mixer2(ctx, capacity=20, group_size=group_size)
    for i in range(len(g[f"{name}_x"])):
        out, used = m(torch.from_numpy(g[f"{name}_x"][i]).to(DEV), torch.from_numpy(g[f"{name}_f"][i]).to(DEV))
        assert used == int(g[f"{name}_m"][i]), i
        assert rel(out.cpu().numpy(), g[f"{name}_out"][i]) < 1e-10, i
    ctx.check_status()


@pytest.mark.parametrize("group_size", [0, 3])
def test_mixer2_long_history_matches_oracle(group_size):
    """The device Type-II mixer against the oracle's msecant2 (pinned to the
    reference) over 30 steps of a contracting fixed-point map on 5,000
    points: histories past 16 columns (the dot products run in chunks of 16),
    slowly shrinking residual differences, groups of 3."""
    n = 5000
    rng = np.random.default_rng(40 + group_size)
    q = np.linalg.qr(rng.standard_normal((n, 24)))[0]
    lam = np.linspace(0.2, 0.97, 24)
    b = rng.standard_normal(n)

    def g(x):   # x -> b + Q diag(lam) Q^T x + 0.05 tanh(x): residual f = g(x) - x
        return b + q @ (lam * (q.T @ x)) + 0.05 * np.tanh(x)

    ctx = gpu.GridContext({"nx": n, "ny": 1, "nz": 1, "h": 1.0, "radius": 1.0}, 8)
    dev = gpu.Mixer2(ctx, capacity=40, group_size=group_size)
    ora = O.MSecant2(group_size=group_size)
    x = rng.standard_normal(n)
    for i in range(30):
        f = g(x) - x
        xo, mo = ora(x, f)
        xd, md = dev(torch.from_numpy(x).to(DEV), torch.from_numpy(f).to(DEV))
        assert md == mo, i
        assert rel(xd.cpu().numpy(), xo) < 1e-8, i
        x = xo
    ctx.check_status()


def test_pcg_matches_reference(golden_dir):
    pc = np.load(golden_dir / "ref_pcg.npz")
    ctx = gpu.GridContext({"nx": 10, "ny": 10, "nz": 10, "h": 0.4, "radius": 1.8}, 8)
    x, its = gpu.pcg(gpu.Laplacian(ctx), torch.from_numpy(pc["rhs"]).to(DEV), torch.from_numpy(pc["x0"]).to(DEV),
                     200, 1e-5)
    assert abs(its - int(pc["its"])) <= 1
    assert rel(x.cpu().numpy(), pc["x"]) < 1e-9


def test_lanczos_bounds_with_reference_start_vectors(h2o_box, golden_dir):
    """The reference's bounds came from lancz_uppbnd after np.random.seed(7)
    (its start vector is np.random.rand(n, 1), lancz_uppbnd.py:22) and from
    lanczosForChefsi1 on np.random.randn(n, 1) after np.random.seed(8): the
    same start vectors passed in give the same bound and Ritz values to
    1e-12 (the recurrence is a handful of H products and dot products)."""
    ctx, atoms, mi = h2o_box
    gpu.projector_setup(ctx, atoms, ElementTable(), pseudo_tables())
    ev = np.load(golden_dir / "ref_eigs.npz")
    gpu.Hamiltonian(ctx, torch.from_numpy(ev["pot"]).to(DEV))
    np.random.seed(7)
    v0 = torch.from_numpy(np.random.rand(ctx.n)).to(DEV)
    np.random.seed(8)
    v1 = torch.from_numpy(np.random.randn(ctx.n)).to(DEV)
    out = ctx.empty(8)
    ctx.call("psc_lanczos_bound_v", 0, gpu._p(v0), gpu._p(out), gpu._stream())
    b0 = out.cpu().numpy().copy()
    ctx.call("psc_lanczos_bound_v", 1, gpu._p(v1), gpu._p(out), gpu._stream())
    b1 = out.cpu().numpy().copy()
    assert abs(b0[0] - float(ev["uppbnd"])) <= 1e-12 * abs(float(ev["uppbnd"]))
    assert np.abs(b0[1:7] - ev["ritz"]).max() <= 1e-12 * np.abs(ev["ritz"]).max()
    assert abs(b1[0] - float(ev["bound"])) <= 1e-12 * abs(float(ev["bound"]))
    ctx.check_status()


def test_lanczos_bounds_bracket_the_spectrum(h2o_box, golden_dir):
    ctx, atoms, mi = h2o_box
    gpu.projector_setup(ctx, atoms, ElementTable(), pseudo_tables())
    pot = np.load(golden_dir / "ref_eigs.npz")["pot"]
    H = gpu.Hamiltonian(ctx, torch.from_numpy(pot).to(DEV))
    ev = np.load(golden_dir / "ref_eigs.npz")
    b0 = gpu.lanczos_bound(ctx, 0).cpu().numpy()
    b1 = gpu.lanczos_bound(ctx, 1).cpu().numpy()
    # same algorithms as the reference with their own random starts: compare
    # with the reference's estimates on the same operator
    assert abs(b0[0] - float(ev["uppbnd"])) < 0.05 * abs(float(ev["uppbnd"]))
    assert abs(b1[0] - float(ev["bound"])) < 0.05 * abs(float(ev["bound"]))
    assert np.all(np.diff(b0[1:7]) >= 0)


def _smooth_block(nx, ny, nz):
    """Three smooth fields vanishing at the faces (the low end of the
    spectrum, where the occupied states live), as an (n, 3) array."""
    i = (np.arange(nx) + 1.0) / (nx + 1)
    j = (np.arange(ny) + 1.0) / (ny + 1)
    l = (np.arange(nz) + 1.0) / (nz + 1)
    cols = []
    for a, b, c in ((1, 1, 1), (2, 1, 3), (3, 2, 2)):
        f = np.sin(np.pi * a * l)[:, None, None] * np.sin(np.pi * b * j)[None, :, None] * \
            np.sin(np.pi * c * i)[None, None, :]
        cols.append(f.ravel())
    return np.stack(cols, axis=1)


@pytest.mark.parametrize("impl", [0, 2, 3, 4])
def test_fp32_stencil_has_no_eigenvalue_offset(impl, capsys):
    """Rayleigh quotients of smooth fields (the low spectrum, where the
    occupied states live) under the FP32 operator against the FP64 one,
    Si87H76 grid (90^3, h = 0.4724 bohr), zero local potential.  Plain FP32
    weights move them by the sum-rule offset dc0 + 6 sum_d dc_d of the
    weights' FP32 rounding errors (-6.1e-8 Ha here, a constant that the band
    energy multiplies by the electron count); the sum-rule correction removes
    exactly that part (within 5 %).  What remains is the FP32 rounding of the
    accumulation, which for the smoothest field cancels 2400-fold: 3e-8 Ha,
    the value a CPU emulation of the kernel's operation order gives too.  Every
    implementation computes the same operation order, so all four agree; the
    bar of 4e-8 catches a weight-rounding offset or an accumulation whose
    small terms are folded into a large sum (+2.3e-7).  "compensated" below
    is weights mode 1 (the correction as a kernel term); mode 2 (the default)
    carries it in the FP32 potential and must agree with mode 1, also under a
    smooth nonzero potential, where fl(pot + correction) and fl(pot) +
    correction round differently at every point but alike on average."""
    cfg = workloads.config_system("si87h76")
    dom = O.build_system(cfg["atoms"], h=cfg["h"], radius=cfg["radius"])
    ctx = gpu.GridContext(dom, 8)
    gpu.Hamiltonian(ctx, torch.zeros(ctx.n, dtype=torch.float64, device=DEV))
    W = _smooth_block(ctx.nx, ctx.ny, ctx.nz).astype(np.float32).astype(np.float64)
    k = W.shape[1]
    Wd = block(W)
    ctx.call("psc_set_stencil_impl", impl)
    W32 = Wd.float()

    def offsets(modes):
        y64 = torch.empty_like(Wd)
        ctx.call("psc_apply_h", F64, gpu._p(Wd), ctx.n, gpu._p(y64), ctx.n, k, gpu._stream())
        r64 = np.einsum("nk,nk->k", W, host(y64)) / np.einsum("nk,nk->k", W, W)
        res = {}
        for comp in modes:
            ctx.call("psc_set_stencil_weights", comp)
            Y32 = torch.empty_like(W32)
            ctx.call("psc_apply_h", F32, gpu._p(W32), ctx.n, gpu._p(Y32), ctx.n, k, gpu._stream())
            res[comp] = np.einsum("nk,nk->k", W, host(Y32).astype(np.float64)) / np.einsum("nk,nk->k", W, W) - r64
        return res

    out = offsets((2, 1, 0))
    # a smooth well of a few Ha (the scale of the local potential)
    x = (np.arange(ctx.nx) - 0.5 * (ctx.nx - 1)) * dom["h"]
    r2 = x[None, None, :] ** 2 + x[None, :, None] ** 2 + x[:, None, None] ** 2
    gpu.Hamiltonian(ctx, torch.from_numpy((-3.0 * np.exp(-r2 / 40.0)).ravel()).to(DEV))
    well = offsets((2, 1))
    ctx.call("psc_set_stencil_weights", 2)
    ctx.call("psc_set_stencil_impl", 0)
    h = dom["h"]
    c0, c = 205.0 / 24.0, np.array([-8.0 / 5.0, 1.0 / 5.0, -8.0 / 315.0, 1.0 / 560.0])
    w0, wd = 0.5 * (c0 / h ** 2), 0.5 * (c / h ** 2)
    pred = (float(np.float32(w0)) - w0) + 6.0 * sum(float(np.float32(x)) - x for x in wd)
    with capsys.disabled():
        print(f"\nimpl {impl}: FP32 - FP64 Rayleigh quotients, in the potential {out[2]}, compensated {out[1]}, "
              f"plain {out[0]} (predicted plain offset {pred:.3e} Ha); under a well: in the potential "
              f"{well[2]}, compensated {well[1]}")
    assert np.abs(out[1]).max() < 4e-8 and np.abs(out[2]).max() < 4e-8
    assert np.abs((out[0] - out[1]) - pred).max() < 0.05 * abs(pred)
    assert np.abs((out[0] - out[2]) - pred).max() < 0.05 * abs(pred)
    assert np.abs(well[2] - well[1]).max() < 5e-9 and np.abs(well[2]).max() < 6e-8
    ctx.check_status()


@pytest.mark.parametrize("shape,order", [((78, 78, 78), 8), ((24, 24, 24), 8), ((20, 16, 12), 6), ((12, 10, 8), 4),
                                         ((10, 12, 14), 2), ((90, 90, 90), 8)])
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_tma_stencil_matches_register_kernel(shape, order, dt):
    nx, ny, nz = shape
    dom = {"nx": nx, "ny": ny, "nz": nz, "h": 0.34, "radius": 0.17 * (nx - 1)}
    ctx = gpu.GridContext(dom, order)
    n = ctx.n
    k = 55 if nx >= 78 else 5
    tdt = torch.float64 if dt == "f64" else torch.float32
    code = F64 if dt == "f64" else F32
    g = torch.Generator(device="cuda").manual_seed(7)
    gpu.Hamiltonian(ctx, torch.randn(n, dtype=torch.float64, device=DEV, generator=g))
    X = torch.randn(k, n, dtype=tdt, device=DEV, generator=g)
    P = torch.randn(k, n, dtype=tdt, device=DEV, generator=g)
    outs = []
    # 1: register-queue kernel; 0, 2: TMA pipeline (4- or 2-point FP32 runs,
    # packed-pair arithmetic); 3, 4: 2- / 4-point runs, scalar arithmetic
    impls = (1, 0, 2, 3, 4) if dt == "f32" else (1, 0)
    for impl in impls:
        ctx.call("psc_set_stencil_impl", impl)
        Y = P.clone()
        ctx.call("psc_apply_h_axpby", code, gpu._p(X), n, gpu._p(Y), n, gpu._p(Y), n, k, 0.7, -0.2, -0.9,
                 gpu._stream())
        outs.append(Y.double().cpu().numpy())
    ctx.call("psc_set_stencil_impl", 0)
    tol = 1e-14 if dt == "f64" else 2e-6
    for impl, o in zip(impls[1:], outs[1:]):
        assert rel(o, outs[0]) < tol, impl
    ctx.check_status()


def test_pcg_graph_equals_direct_launches():
    dom = {"nx": 40, "ny": 40, "nz": 40, "h": 0.4, "radius": 7.8}
    ctx = gpu.GridContext(dom, 8)
    g = torch.Generator(device="cuda").manual_seed(3)
    rhs = torch.randn(ctx.n, dtype=torch.float64, device=DEV, generator=g)
    x0 = torch.randn(ctx.n, dtype=torch.float64, device=DEV, generator=g) * 0.1
    A = gpu.Laplacian(ctx)
    res = []
    for mode in (1, 0):
        ctx.call("psc_set_use_graphs", mode)
        res.append(gpu.pcg(A, rhs, x0, 200, 1e-5))
    assert res[0][1] == res[1][1]
    assert torch.equal(res[0][0], res[1][0])
    # the oracle's CG on the same system
    xo, its = O.pcg(O.laplacian(dom, 8), rhs.cpu().numpy(), x0.cpu().numpy(), 200, 1e-5)
    assert abs(its - res[0][1]) <= 1
    assert rel(res[0][0].cpu().numpy(), xo) < 1e-8


@pytest.mark.parametrize("shape,order,maxit", [((40, 40, 40), 8, 200), ((78, 78, 78), 8, 200),
                                               ((21, 17, 13), 6, 200), ((16, 12, 20), 4, 7),
                                               ((9, 11, 10), 2, 200)])
def test_pcg_persistent_matches_graph_and_oracle(shape, order, maxit):
    """The one-launch persistent CG against the graph-replayed kernels and the
    oracle.  Partial sums are grouped differently, so iterates agree to
    rounding, not bit for bit."""
    nx, ny, nz = shape
    dom = {"nx": nx, "ny": ny, "nz": nz, "h": 0.4, "radius": 0.2 * (nx - 1)}
    ctx = gpu.GridContext(dom, order)
    g = torch.Generator(device="cuda").manual_seed(5)
    rhs = torch.randn(ctx.n, dtype=torch.float64, device=DEV, generator=g)
    x0 = torch.randn(ctx.n, dtype=torch.float64, device=DEV, generator=g) * 0.1
    A = gpu.Laplacian(ctx)
    res, launches = [], []
    for mode in (2, 1):
        ctx.call("psc_set_use_graphs", mode)
        before = _lib.load().psc_launch_count()
        res.append(gpu.pcg(A, rhs, x0, maxit, 1e-5))
        launches.append(_lib.load().psc_launch_count() - before)
    assert launches[0] == 1                      # the persistent kernel ran
    assert abs(res[0][1] - res[1][1]) <= 1
    assert rel(res[0][0].cpu().numpy(), res[1][0].cpu().numpy()) < 1e-9
    xo, its = O.pcg(O.laplacian(dom, order), rhs.cpu().numpy(), x0.cpu().numpy(), maxit, 1e-5)
    assert abs(its - res[0][1]) <= 1
    assert rel(res[0][0].cpu().numpy(), xo) < 1e-8
    assert int(ctx.status()[4]) == 0


def test_pcg_persistent_falls_back_when_vectors_do_not_fit():
    dom = {"nx": 132, "ny": 132, "nz": 132, "h": 0.4, "radius": 26.2}   # 4 x 2.3M doubles > shared memory
    ctx = gpu.GridContext(dom, 8)
    g = torch.Generator(device="cuda").manual_seed(6)
    rhs = torch.randn(ctx.n, dtype=torch.float64, device=DEV, generator=g)
    x0 = torch.zeros(ctx.n, dtype=torch.float64, device=DEV)
    before = _lib.load().psc_launch_count()
    x, its = gpu.pcg(gpu.Laplacian(ctx), rhs, x0, 12, 1e-5)
    assert _lib.load().psc_launch_count() - before > 1
    assert its == 12


@pytest.mark.parametrize("k", [27, 55, 70])
def test_subspace_rr_matches_qr_rayleigh_ritz(h2o_box, golden_dir, k):
    """One-pass Rayleigh-Ritz of a filtered block vs the reference's route
    (Householder QR, then G = Q^T H Q, eigh) done by the oracle on the same W."""
    ctx, atoms, mi = h2o_box
    gpu.projector_setup(ctx, atoms, ElementTable(), pseudo_tables())
    pot = np.load(golden_dir / "ref_eigs.npz")["pot"]
    H = gpu.Hamiltonian(ctx, torch.from_numpy(pot).to(DEV))
    B = _csr_h(mi, pot)
    rng = np.random.default_rng(11)
    X = rng.random((ctx.n, k))
    Xf = O.cheb_filter_slim(B, X, 10, 5.0, 60.0)          # an ill-conditioned filtered block
    W = block(Xf)
    V = torch.empty_like(W)
    ritz = ctx.empty(k)
    R, _ = gpu.subspace_rr(ctx, W, V, ritz)
    import scipy.linalg
    Q, _ = scipy.linalg.qr(Xf, mode="economic")
    G = O._gram_upper(B @ Q, Q)
    lam, Y = scipy.linalg.eigh(G)
    got = ritz.cpu().numpy()
    assert np.abs(got - lam).max() < 1e-10 * np.abs(lam).max()
    Wr = host(R)
    assert np.abs(Wr.T @ Wr - np.eye(k)).max() < 1e-9
    # Ritz vectors of well-separated Ritz values agree up to sign
    gap = np.minimum(np.diff(lam, prepend=-np.inf), np.diff(lam, append=np.inf))
    good = gap > 1e-3 * np.abs(lam).max()
    ref_vec = Q @ Y
    dots = np.abs(np.sum(Wr[:, good] * ref_vec[:, good], axis=0))
    assert np.all(dots > 1 - 1e-8)
