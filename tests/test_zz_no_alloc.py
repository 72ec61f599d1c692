"""pw_apply_vloc_noalloc against pw_apply, through the C ABI.

The allocation-free entry point serves callers that cannot allocate device
memory on the operator path (a host whose pooling allocator owns the GPU's
memory, or a solver loop that must not stall on cudaMalloc's implicit device
synchronisation).  Its intermediate is a fixed 32 MiB device array inside
the library, shared by every call.  This file is collected last so that a
run stopping at the first failure has already run every other test; it also
passes when run alone in a fresh process.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-11, "c64": 2e-5}


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def si64():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    H = systems.Ham_Si64(Nstates=160)
    rng = np.random.default_rng(42)
    pw = H.pw
    V = H.V_Ps_loc + 0.01 * rng.standard_normal(pw.Npoints)
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    ctx.set_vloc(V)
    ngw = pw.gvecw.Ngw[0]
    psis = [(rng.standard_normal((ngw, 64)) + 1j * rng.standard_normal((ngw, 64))) / np.sqrt(ngw) for _ in range(2)]
    yield ctx, psis
    ctx.close()


@pytest.mark.parametrize("prec", ["c128", "c64"])
@pytest.mark.parametrize("acc", [False, True])
def test_noalloc_matches_apply_twice(si64, prec, acc):
    import torch
    import pwb200
    ctx, psis = si64
    dt = torch.complex128 if prec == "c128" else torch.complex64
    ops = pwb200.PW_OP_VLOC | pwb200.PW_OP_K | (pwb200.PW_ACCUMULATE if acc else 0)
    for psi in psis:                      # two calls in a row, different inputs
        x = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda().to(dt)
        base = torch.full_like(x, 0.25 - 0.5j)
        y_ref = base.clone()
        y_new = base.clone()
        ctx.apply(0, 0, x, y_ref, ops)
        ctx.apply_vloc_noalloc(0, 0, x, y_new, ops)
        torch.cuda.synchronize()
        ref = y_ref.cpu().numpy().astype(np.complex128)
        got = y_new.cpu().numpy().astype(np.complex128)
        assert rel_err(got, ref) < TOL[prec]


def test_noalloc_rejects_oversized_grid_and_ops(si64):
    import torch
    import pwb200
    ctx, psis = si64
    x = torch.from_numpy(np.ascontiguousarray(psis[0].T)).cuda()
    with pytest.raises(pwb200.PWError) as e:
        ctx.apply_vloc_noalloc(0, 0, x, torch.empty_like(x), pwb200.PW_OP_H)   # V_nl needs scratch: not offered
    assert e.value.status == pwb200._lib.PW_ERR_ARG
    # a dense 160^3 "sphere": one FP64 band needs 160^3 * 16 B = 64 MiB > 32 MiB
    n = 160
    idx = np.arange(n ** 3, dtype=np.int64)
    big = pwb200.Context((n, n, n), 1000.0, [idx], [np.zeros(n ** 3)])
    big.set_vloc(np.zeros(n ** 3))
    xb = torch.zeros((1, n ** 3), dtype=torch.complex128, device="cuda")
    with pytest.raises(pwb200.PWError) as e:
        big.apply_vloc_noalloc(0, 0, xb, torch.empty_like(xb), pwb200.PW_OP_VLOC)
    assert e.value.status == pwb200._lib.PW_ERR_UNSUPPORTED
    assert int(pwb200.lib().pw_noalloc_scratch_bytes()) == 32 << 20
    big.close()


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_noalloc_leaves_free_memory_unchanged(prec):
    """The property the entry point exists for: after one warm-up call (which
    loads its kernels), calls with growing band counts take no device
    memory.  A fresh context that never ran pw_apply; every tensor is
    allocated before the free memory is read."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from oracle import systems
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1), extra_states=4)
    pw = H.pw
    rng = np.random.default_rng(7)
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    ctx.set_vloc(H.V_Ps_loc + 0.01 * rng.standard_normal(pw.Npoints))
    ngw = pw.gvecw.Ngw[0]
    dt = torch.complex128 if prec == "c128" else torch.complex64
    nmax = 96
    psi = (rng.standard_normal((ngw, nmax)) + 1j * rng.standard_normal((ngw, nmax))) / np.sqrt(ngw)
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda().to(dt)
    y = torch.zeros_like(x)
    ops = pwb200.PW_OP_VLOC | pwb200.PW_OP_K
    ctx.apply_vloc_noalloc(0, 0, x[:1], y[:1], ops)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for nb in (1, 2, 8, 33, nmax):
        ctx.apply_vloc_noalloc(0, 0, x[:nb], y[:nb], ops)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    ctx.close()
