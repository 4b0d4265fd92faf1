"""Failure detection on the GPU path, in forms that fault, trap or hang no GPU.

Device side: every bounded wait (stencil bulk-copy pipeline, tensor-core Gram,
block-product and convolution pipelines, the persistent CG's grid barrier) takes its poll
limit from the context.  With the limit set to 0 each wait runs out at its
first unsatisfied poll; the kernels must then record their status word,
drain what they issued and return, and the context must stay usable: the
same calls with the default limit give correct results afterwards.

Host side: the errors the reference raises or reports on bad input
(inverted filter bounds, Eigensolvers/chefsi1.py:37-38; an SCF that reaches
maxits, rsdft_solver.py:397-413), a NaN potential, and the learned start's
fallback to SAD on a non-finite prediction.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - collected on CPU runs
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from parsec_python_b200 import gpu  # noqa: E402
from parsec_python_b200._lib import F32, F64, PscError  # noqa: E402

DEV = torch.device("cuda", 0)


def _ctx(nx=24):
    return gpu.GridContext({"nx": nx, "ny": nx, "nz": nx, "h": 0.4, "radius": 0.2 * (nx - 1)}, 8)


def test_wait_limit_zero_reports_every_pipeline_and_context_recovers():
    ctx = _ctx(24)
    n = ctx.n
    rng = np.random.default_rng(3)
    pot = torch.from_numpy(rng.standard_normal(n)).to(DEV)
    H = gpu.Hamiltonian(ctx, pot)
    X64 = torch.from_numpy(rng.standard_normal((4, n))).to(DEV)
    W32 = torch.from_numpy(rng.standard_normal((40, n)).astype(np.float32)).to(DEV)
    T = torch.from_numpy(rng.standard_normal((40, 40))).to(DEV)
    rhs = torch.from_numpy(rng.standard_normal(n)).to(DEV)
    zero = torch.zeros(n, dtype=torch.float64, device=DEV)
    A = gpu.Laplacian(ctx)
    st = gpu._stream()
    # one 3x3x3 convolution of the learned start: 8 -> 16 channels on an 8^3 grid
    geom = (ctypes.c_int * 15)(8, 8, 8, 8, 8, 8, 0, 8, 0, 8, 8, 8, 1, 3, 16)
    cx = torch.from_numpy(rng.standard_normal((512, 8)).astype(np.float32)).to(torch.bfloat16).to(DEV)
    cw = torch.from_numpy((rng.standard_normal(27 * 8 * 16) / 15).astype(np.float32)).to(torch.bfloat16).to(DEV)
    cb = torch.zeros(16, dtype=torch.float32, device=DEV)
    ctx.status(clear=True)

    def conv(impl):
        ctx.call("psc_set_conv_impl", impl)
        y = torch.empty(512, 16, dtype=torch.bfloat16, device=DEV)
        y32 = torch.full((512, 16), float("nan"), dtype=torch.float32, device=DEV)
        ctx.call("psc_conv3d_fwd", geom, gpu._p(cx), None, gpu._p(cw), gpu._p(cb), 0, gpu._p(y), gpu._p(y32), st)
        return y32

    def run_all():
        Y = H @ X64
        S, K = ctx.empty(40, 40), ctx.empty(40, 40)
        ctx.call("psc_gram_pair", F32, gpu._p(W32), gpu._p(W32), n, 40, gpu._p(S), gpu._p(K), st)
        O32 = torch.empty_like(W32)
        ctx.call("psc_gemm_nn", F32, gpu._p(W32), n, 40, gpu._p(T), 40, gpu._p(O32), n, st)
        C = conv(2)
        torch.cuda.synchronize()
        return Y, S, O32, C

    ctx.call("psc_set_wait_limit", 0)
    run_all()
    flags = ctx.status(clear=False)
    assert flags[3] == 1, "stencil pipeline wait did not report"
    assert flags[5] == 1, "tensor-core Gram wait did not report"
    assert flags[6] == 1, "tensor-core block product wait did not report"
    assert flags[7] == 1, "tensor-core convolution wait did not report"
    with pytest.raises(PscError, match="grid barrier timed out"):
        gpu.pcg(A, rhs, zero, 20, 1e-5)
    assert ctx.status(clear=True)[4] == 1
    with pytest.raises(PscError, match="TMA stencil pipeline wait timed out"):
        (H @ X64, torch.cuda.synchronize(), ctx.check_status())

    # default limit: the same calls are correct and report nothing
    ctx.call("psc_set_wait_limit", -1)
    ctx.status(clear=True)
    Y, S, O32, C = run_all()
    x, its = gpu.pcg(A, rhs, zero, 20, 1e-5)
    assert ctx.status(clear=True) == [0] * 8
    dom = {"nx": 24, "ny": 24, "nz": 24, "h": 0.4, "radius": 0.2 * 23}
    Xh = X64.cpu().numpy().T
    ref = O.fd_apply(dom, 8, np.asfortranarray(Xh), 0.5 / 0.4 ** 2, pot.cpu().numpy())
    assert np.abs(Y.cpu().numpy().T - ref).max() < 1e-12 * np.abs(ref).max()
    W64 = W32.double().cpu().numpy()
    assert np.abs(S.cpu().numpy().T - W64 @ W64.T).max() < 2e-5 * np.abs(W64 @ W64.T).max()
    Oref = W64.T @ T.cpu().numpy().T
    assert np.abs(O32.double().cpu().numpy().T - Oref).max() < 2e-5 * np.abs(Oref).max()
    C0 = conv(0)
    assert ctx.status(clear=True) == [0] * 8
    assert (C - C0).abs().max().item() < 2e-5 * max(1.0, C0.abs().max().item())
    xo, its_o = O.pcg(O.laplacian(dom, 8), rhs.cpu().numpy(), np.zeros(n), 20, 1e-5)
    assert its == its_o and np.abs(x.cpu().numpy() - xo).max() < 1e-8 * np.abs(xo).max()


def test_inverted_filter_bounds_raise_value_error():
    """chefsi1.py:37-38: lowerb = max(ritzv) above the Lanczos upper bound."""
    ctx = _ctx(20)
    pot = torch.zeros(ctx.n, dtype=torch.float64, device=DEV)
    H = gpu.Hamiltonian(ctx, pot)
    W = torch.from_numpy(np.random.default_rng(1).standard_normal((8, ctx.n))).to(DEV)
    ritz = torch.full((8,), 1e6, dtype=torch.float64, device=DEV)
    with pytest.raises(ValueError, match="Bounds are incorrect"):
        gpu.chefsi1(W, ritz, 4, 5, H)
        torch.cuda.synchronize()
        ctx.check_status()
    assert ctx.status(clear=True)[0] == 0   # check_status cleared it


def test_nan_potential_is_reported_not_propagated_silently():
    """A NaN in the potential makes the Lanczos bound NaN.  The reference's
    test `lowerb > upperb` is False for NaN and it carries on with NaN
    blocks; here the filter's bound check !(hi > lo) catches it and the
    subspace step raises instead of returning NaN eigenpairs."""
    ctx = _ctx(20)
    p = np.zeros(ctx.n)
    p[ctx.n // 2] = np.nan
    H = gpu.Hamiltonian(ctx, torch.from_numpy(p).to(DEV))
    W = torch.from_numpy(np.random.default_rng(2).standard_normal((8, ctx.n))).to(DEV)
    ritz = torch.linspace(-1.0, 0.5, 8, dtype=torch.float64, device=DEV)
    with pytest.raises((ValueError, PscError)):
        gpu.chefsi1(W, ritz, 4, 5, H)
        torch.cuda.synchronize()
        ctx.check_status()


def test_scf_reaching_maxits_reports_not_converged(capsys):
    """rsdft_solver.py:397-413: the loop stops at maxits and reports the
    last iteration's values as not converged."""
    from parsec_python_b200.backend import select_solver_backend
    from parsec_python_b200.inputs import ElementTable
    from parsec_python_b200.models import SolverSettings
    from parsec_python_b200.solver import run_rsdft_calculation
    from parsec_python_b200.system import system_from_atoms

    a0 = O.A0_ANG
    atoms = [{"typ": "O", "coord": np.array([[0.0, 0.0, 0.0]]) / a0},
             {"typ": "H", "coord": np.array([[0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]) / a0}]
    s = SolverSettings(tol=1e-10, maxits=2, poldeg=6)
    s.normalize()
    elem = ElementTable()
    prob = system_from_atoms(atoms, h=0.45, radius=4.0, nev=8, settings=s, elem=elem)
    res = run_rsdft_calculation(prob, elem, len(elem), select_solver_backend(s), verbose=True)
    out = capsys.readouterr().out
    assert res.iterations == 2 and not res.converged and res.error > 1e-10
    assert "DID NOT CONVERGE" in out
    assert np.isfinite(res.history[-1]["total_ry"])


def test_learned_start_falls_back_to_sad_on_non_finite_prediction():
    from parsec_python_b200 import learned

    params = learned.load_weights()
    if params is None:
        pytest.skip("no trained weights in the package")
    bad = dict(params)
    bad["w"] = params["w"].copy()
    bad["w"][:64] = np.float32("nan") if bad["w"].dtype != np.uint16 else np.uint16(0x7FC0)
    init = learned.LearnedInit(bad)
    ctx = _ctx(24)
    rng = np.random.default_rng(4)
    rho0 = torch.from_numpy(np.abs(rng.standard_normal(ctx.n)) * 1e-3).to(DEV)
    ppot = torch.from_numpy(-np.abs(rng.standard_normal(ctx.n))).to(DEV)
    rho1, dh = init(ctx, rho0, torch.zeros_like(rho0), ppot, gpu.Laplacian(ctx))
    assert init.last.get("fallback") == "non-finite prediction"
    assert torch.equal(rho1, rho0) and float(dh.abs().max()) == 0.0
