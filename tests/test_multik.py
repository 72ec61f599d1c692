"""Batched op_H over k-points (pw_apply_multi): the BlochWavefunc form of
op_H! (op_H.jl:4-35) for every k-point in one launch per stage.

Al4 conventional fcc cell (config C3's system), 4x4x4 k-mesh reduced by
time reversal (36 k-points, Ngw 1208-1250 per k), 10 bands:
  - against the oracle's op_H per k-point (FP64 1e-11, FP32 2e-5 relative)
  - against pw_apply per k-point (the FFT stages run the same band bodies:
    FP64 1e-13, FP32 1e-6 relative, the nonlocal sums differ in order)
  - accumulate flag, a subset of k-points, and CUDA-graph replay (a second
    call replays the captured graph and follows a new V_loc)
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def al4():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    Ho = systems.Ham_Al4(meshk=(4, 4, 4))
    pw = Ho.pw
    rng = np.random.default_rng(8)
    Ho.V_Total = Ho.V_Ps_loc + 0.05 * np.cos(np.arange(pw.Npoints) * 0.21)
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(k) for k in range(pw.kpoints.Nkpt)])
    ctx.set_vloc(Ho.V_Total)
    for ik in range(pw.kpoints.Nkpt):
        ctx.set_nonlocal(ik, Ho.betaNL[ik])
    ctx.set_nonlocal_coef(Ho.nl_triplets)
    psis = [rng.standard_normal((pw.gvecw.Ngw[ik], 10)) + 1j * rng.standard_normal((pw.gvecw.Ngw[ik], 10))
            for ik in range(pw.kpoints.Nkpt)]
    yield Ho, ctx, psis
    ctx.close()


def _dev(psis, dt):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(p.T)).cuda().to(dt).contiguous() for p in psis]


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_apply_multi_matches_oracle_and_per_k(al4, prec):
    import torch
    from oracle import ops
    Ho, ctx, psis = al4
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = _dev(psis, dt)
    HX = [torch.empty_like(x) for x in X]
    nk = len(X)
    ctx.apply_multi(list(range(nk)), 0, X, HX)
    tol_o = 1e-11 if prec == "c128" else 2e-5
    tol_k = 1e-13 if prec == "c128" else 1e-6
    for ik in range(nk):
        got = HX[ik].cpu().numpy().T.astype(np.complex128)
        assert _rel(got, ops.op_H(Ho, psis[ik], ik)) < tol_o, ik
        one = torch.empty_like(X[ik])
        ctx.apply(ik, 0, X[ik], one)
        assert _rel(got, one.cpu().numpy().T.astype(np.complex128)) < tol_k, ik
    ctx.check_device()


def test_apply_multi_accumulate_subset_and_graph(al4):
    import torch
    import pwb200
    from oracle import ops
    Ho, ctx, psis = al4
    sel = [3, 0, 17, 35, 9]
    X = _dev([psis[i] for i in sel], torch.complex64)
    HX = [torch.ones_like(x) for x in X]
    ctx.apply_multi(sel, 0, X, HX, ops=pwb200.PW_OP_H | pwb200.PW_ACCUMULATE)
    for j, ik in enumerate(sel):
        ref = ops.op_H(Ho, psis[ik], ik) + 1.0
        assert _rel(HX[j].cpu().numpy().T.astype(np.complex128), ref) < 2e-5
    # graph: first call captures, second replays; a new V_loc is picked up
    HY = [torch.empty_like(x) for x in X]
    n0 = ctx.launch_count()
    ctx.apply_multi(sel, 0, X, HY, graph=True)
    ctx.apply_multi(sel, 0, X, HY, graph=True)
    assert ctx.launch_count() - n0 == 8
    V2 = Ho.V_Total + 0.3 * np.sin(np.arange(Ho.pw.Npoints) * 0.05)
    ctx.set_vloc(V2)
    ctx.apply_multi(sel, 0, X, HY, graph=True)
    Ho.V_Total, V_old = V2, Ho.V_Total
    try:
        for j, ik in enumerate(sel):
            assert _rel(HY[j].cpu().numpy().T.astype(np.complex128), ops.op_H(Ho, psis[ik], ik)) < 2e-5
    finally:
        Ho.V_Total = V_old
        ctx.set_vloc(V_old)
    ctx.check_device()


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_apply_multi_persistent_matches_oracle(al4, prec):
    """PW_PERSISTENT: every stage in one cooperative launch (bounded grid
    barriers between the stages): the oracle's op_H per k-point, one launch
    per call, and a CUDA-graph capture of it replays."""
    import torch
    from oracle import ops
    Ho, ctx, psis = al4
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = _dev(psis, dt)
    HX = [torch.empty_like(x) for x in X]
    nk = len(X)
    n0 = ctx.launch_count()
    ctx.apply_multi(list(range(nk)), 0, X, HX, persistent=True)
    assert ctx.launch_count() - n0 == 1
    tol = 1e-11 if prec == "c128" else 2e-5
    for ik in range(nk):
        assert _rel(HX[ik].cpu().numpy().T.astype(np.complex128), ops.op_H(Ho, psis[ik], ik)) < tol, ik
    HY = [torch.zeros_like(x) for x in X]
    ctx.apply_multi(list(range(nk)), 0, X, HY, graph=True, persistent=True)
    ctx.apply_multi(list(range(nk)), 0, X, HY, graph=True, persistent=True)
    for ik in range(nk):
        assert _rel(HY[ik].cpu().numpy().T.astype(np.complex128), HX[ik].cpu().numpy().T.astype(np.complex128)) < 1e-12
    ctx.check_device()


def test_apply_multi_errors(al4):
    import torch
    import pwb200
    Ho, ctx, psis = al4
    X = _dev(psis[:2], torch.complex128)
    with pytest.raises(pwb200.PWError) as e:
        ctx.apply_multi([0, 1], 0, X, [torch.empty_like(x) for x in X], ops=pwb200.PW_OP_K)
    assert e.value.status == pwb200._lib.PW_ERR_UNSUPPORTED
    with pytest.raises(pwb200.PWError):
        ctx.apply_multi([0, 99], 0, X, [torch.empty_like(x) for x in X])
    with pytest.raises(pwb200.PWError):
        ctx.apply_multi([0, 1], 0, X, X)          # aliasing
    ctx.check_device()
