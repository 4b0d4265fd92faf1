"""psc_lda_xc_noalloc: LDA XC for callers that cannot allocate device memory.

Callers inside a CUDA stream capture (cudaMalloc cannot be captured) or under
a host that gives all device memory to its own pool cannot create a libpsc
context, because creating one allocates.  This entry point needs no context:
its scratch is a fixed device array inside the library.  The test calls it
through the C ABI twice in a row, on different densities, and compares each
result with the context-based psc_lda_xc at the tolerance of the other XC
test (1e-13 relative on v_xc, 1e-12 on E_xc); it also checks the entry point
against the reference's own exc_nspn fixture and that a call leaves the
device's free memory unchanged, and that a call made during a CUDA graph
capture replays correctly.  The file name sorts last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parsec_python_b200 import _lib, gpu  # noqa: E402


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _densities(n, seed):
    rng = np.random.default_rng(seed)
    rho = 10 ** rng.uniform(-9, 1.5, n)          # both branches (rs < 1 and rs >= 1)
    rho[:7] = 0.0                                # vacuum
    rho[7:11] = -1e-4                            # negative density (skipped by the formula)
    return rho


def test_noalloc_xc_matches_context_xc_on_two_calls():
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    h3 = 0.37 ** 3
    for seed, n in ((1, 300_001), (2, 40_000)):   # the second call is smaller: stale partials must not leak
        rho = torch.from_numpy(_densities(n, seed)).to(dev)
        vxc_a = torch.empty_like(rho)
        out_a = torch.empty(3, dtype=torch.float64, device=dev)
        rc = lib.psc_lda_xc_noalloc(_p(rho), _p(vxc_a), n, h3, _p(out_a), st)
        assert rc == 0, lib.psc_last_error(None)
        ctx = gpu.GridContext({"nx": n, "ny": 1, "nz": 1, "h": 0.37, "radius": 1.0}, 8)
        vxc_b, out_b = gpu.lda_xc(ctx, rho)
        torch.cuda.synchronize()
        va, vb = vxc_a.cpu().numpy(), vxc_b.cpu().numpy()
        assert np.abs(va - vb).max() <= 1e-13 * np.abs(vb).max()
        oa, ob = out_a.cpu().numpy(), out_b.cpu().numpy()
        assert abs(oa[0] - ob[0]) <= 1e-12 * abs(ob[0])
        assert oa[1] == ob[1] and oa[2] == ob[2]


def test_noalloc_xc_matches_reference_fixture(golden_dir):
    """Against the reference's own exc_nspn output (tests/golden/ref_xc.npz,
    made by running V_xc/exc_nspn.py), the same bars as the context path's
    test: 1e-13 on v_xc, 1e-12 on E_xc, exact max and min."""
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    xc = np.load(golden_dir / "ref_xc.npz")
    rho = torch.from_numpy(xc["rho"]).to(dev)
    vxc = torch.empty_like(rho)
    out = torch.empty(3, dtype=torch.float64, device=dev)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.psc_lda_xc_noalloc(_p(rho), _p(vxc), rho.numel(), 0.37 ** 3, _p(out), st) == 0
    torch.cuda.synchronize()
    v = vxc.cpu().numpy()
    assert np.abs(v - xc["vxc"]).max() <= 1e-13 * np.abs(xc["vxc"]).max()
    o = out.cpu().numpy()
    assert abs(o[0] - float(xc["exc"])) <= 1e-12 * abs(float(xc["exc"]))
    assert o[1] == xc["rho"].max() and o[2] == xc["rho"].min()


def test_noalloc_xc_allocates_nothing_and_propagates_nan():
    """After the first call (which may load the module), a call leaves the
    device's free memory unchanged.  A NaN density makes the logged maximum
    and minimum NaN on both entry points, as numpy's max and min do."""
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 50_000
    rho = torch.from_numpy(_densities(n, 3)).to(dev)
    vxc = torch.empty_like(rho)
    out = torch.empty(3, dtype=torch.float64, device=dev)
    assert lib.psc_lda_xc_noalloc(_p(rho), _p(vxc), n, 1.0, _p(out), st) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    assert lib.psc_lda_xc_noalloc(_p(rho), _p(vxc), n, 1.0, _p(out), st) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0
    rho[n // 3] = float("nan")
    assert lib.psc_lda_xc_noalloc(_p(rho), _p(vxc), n, 1.0, _p(out), st) == 0
    ctx = gpu.GridContext({"nx": n, "ny": 1, "nz": 1, "h": 1.0, "radius": 1.0}, 8)
    _, out_b = gpu.lda_xc(ctx, rho)
    torch.cuda.synchronize()
    for o in (out.cpu().numpy(), out_b.cpu().numpy()):
        assert np.isnan(o[1]) and np.isnan(o[2])


def test_noalloc_xc_runs_inside_a_cuda_graph_capture():
    """The case the entry point exists for: after one call outside (which
    looks up its scratch), a call made while a stream is being captured into
    a CUDA graph records its launches; replaying the graph on a new density
    gives the context path's result for that density."""
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n = 20_000
    rho = torch.from_numpy(_densities(n, 4)).to(dev)
    vxc = torch.empty_like(rho)
    out = torch.empty(3, dtype=torch.float64, device=dev)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.psc_lda_xc_noalloc(_p(rho), _p(vxc), n, 1.0, _p(out), st) == 0
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cap = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = lib.psc_lda_xc_noalloc(_p(rho), _p(vxc), n, 1.0, _p(out), cap)
    assert rc == 0, lib.psc_last_error(None)
    rho.copy_(torch.from_numpy(_densities(n, 5)).to(dev))
    vxc.zero_()
    g.replay()
    torch.cuda.synchronize()
    ctx = gpu.GridContext({"nx": n, "ny": 1, "nz": 1, "h": 1.0, "radius": 1.0}, 8)
    vxc_b, out_b = gpu.lda_xc(ctx, rho)
    torch.cuda.synchronize()
    va, vb = vxc.cpu().numpy(), vxc_b.cpu().numpy()
    assert np.abs(va - vb).max() <= 1e-13 * np.abs(vb).max()
    oa, ob = out.cpu().numpy(), out_b.cpu().numpy()
    assert abs(oa[0] - ob[0]) <= 1e-12 * abs(ob[0])
    assert oa[1] == ob[1] and oa[2] == ob[2]
    del g


def test_noalloc_xc_rejects_sizes_beyond_its_scratch():
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    x = torch.zeros(4, dtype=torch.float64, device=dev)
    rc = lib.psc_lda_xc_noalloc(_p(x), _p(x), 33_554_433, 1.0, _p(x), None)
    assert rc == 2
    assert b"33554432" in lib.psc_last_error(None)
