"""Parity of the CUDA operators with the FP64 oracle (op_H.jl, op_K.jl,
op_V_loc.jl, op_V_Ps_nloc.jl, Kprec.jl, calc_rhoe.jl), called through the C ABI.

Tolerances (max-abs error relative to the max-abs of the oracle result):
  FP64 path (complex128):            1e-11
  mixed path (complex64, FP32 FFTs): 2e-5
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-11, "c64": 2e-5}


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module", params=["si_fcc", "si64"])
def system(request):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    if request.param == "si_fcc":
        H = systems.Ham_Si_fcc(meshk=(3, 3, 3), extra_states=4)
        nb = 8
    else:
        H = systems.Ham_Si64(Nstates=160)
        nb = 48
    rng = np.random.default_rng(11)
    N = H.pw.Npoints
    # V_loc: the pseudopotential plus a smooth random perturbation (0.01 Ha)
    dV = rng.standard_normal(N)
    H.V_Total = H.V_Ps_loc + 0.01 * dV / np.abs(dV).max()
    pw = H.pw
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(k) for k in range(pw.kpoints.Nkpt)])
    ctx.set_vloc(H.V_Total)
    for ik in range(pw.kpoints.Nkpt):
        ctx.set_nonlocal(ik, H.betaNL[ik])
    ctx.set_nonlocal_coef(H.nl_triplets)
    psis = []
    for ik in range(pw.kpoints.Nkpt):
        ngw = pw.gvecw.Ngw[ik]
        psis.append((rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb))) / np.sqrt(ngw))
    yield H, ctx, psis
    ctx.close()


def to_dev(psi, dt):
    import torch
    return torch.from_numpy(np.ascontiguousarray(psi.T)).to("cuda").to(dt).contiguous()


def to_host(t):
    return t.to(dtype=t.dtype).cpu().numpy().T.astype(np.complex128)


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_op_H(system, prec):
    import torch
    import pwb200
    from oracle import ops
    H, ctx, psis = system
    dt = torch.complex128 if prec == "c128" else torch.complex64
    for ik in [0, len(psis) - 1]:
        ref = ops.op_H(H, psis[ik], ik)
        x = to_dev(psis[ik], dt)
        y = torch.empty_like(x)
        ctx.apply(ik, 0, x, y, pwb200.PW_OP_H)
        assert rel_err(to_host(y), ref) < TOL[prec]


@pytest.fixture(scope="module")
def si216():
    """Si216 (3x3x3 diamond cells, 120^3 grid, Ngw 80797): the 120-point
    plane kernels (one band per CTA, rows padded one word per 24 elements)
    and z passes (cp.async tiles); five bands; the oracle set-up takes
    about 30 s."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    H = systems.Hamiltonian(systems.diamond_supercell(3, 10.2631), [systems.psp("Si-q4.gth")], 15.0, Nstates=432)
    rng = np.random.default_rng(12)
    N = H.pw.Npoints
    dV = rng.standard_normal(N)
    H.V_Total = H.V_Ps_loc + 0.01 * dV / np.abs(dV).max()
    pw = H.pw
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    ctx.set_vloc(H.V_Total)
    ctx.set_nonlocal(0, H.betaNL[0])
    ctx.set_nonlocal_coef(H.nl_triplets)
    ngw = pw.gvecw.Ngw[0]
    psi = (rng.standard_normal((ngw, 5)) + 1j * rng.standard_normal((ngw, 5))) / np.sqrt(ngw)
    yield H, ctx, psi
    ctx.close()


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_op_H_120_grid(si216, prec):
    import torch
    import pwb200
    from oracle import ops
    H, ctx, psi = si216
    dt = torch.complex128 if prec == "c128" else torch.complex64
    ref = ops.op_H(H, psi, 0)
    x = to_dev(psi, dt)
    y = torch.empty_like(x)
    ctx.apply(0, 0, x, y, pwb200.PW_OP_H)
    assert rel_err(to_host(y), ref) < TOL[prec]
    rho = torch.zeros(H.pw.Npoints, dtype=torch.float64, device="cuda")
    w = np.array([2.0, 2.0, 1.5, 0.5, 0.25])
    ctx.calc_rhoe(0, x, w, rho)
    assert rel_err(rho.cpu().numpy(), ops.calc_rhoe(H, [psi], Focc=w[:, None])) < TOL[prec]


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_op_H_120_grid_band_batch_boundary(si216, prec):
    """Band batches of 5 MiB on the 120-point grid (2 FP32 bands or 1 FP64
    band per batch), so that 5 bands cross 2-4 batch boundaries, with 1 and 2
    sub-planes per plane-kernel CTA."""
    import torch
    import pwb200
    from oracle import ops
    H, ctx, psi = si216
    dt = torch.complex128 if prec == "c128" else torch.complex64
    ref = ops.op_H(H, psi, 0)
    w = np.array([2.0, 2.0, 1.5, 0.5, 0.25])
    ref_rho = ops.calc_rhoe(H, [psi], Focc=w[:, None])
    saved = ctx.get_tuning()
    try:
        for pb in (1, 2):
            ctx.set_tuning(band_chunk_bytes=5 << 20, plane_bands=pb)
            x = to_dev(psi, dt)
            y = torch.empty_like(x)
            ctx.apply(0, 0, x, y, pwb200.PW_OP_H)
            assert rel_err(to_host(y), ref) < TOL[prec], pb
            rho = torch.zeros(H.pw.Npoints, dtype=torch.float64, device="cuda")
            ctx.calc_rhoe(0, x, w, rho)
            assert rel_err(rho.cpu().numpy(), ref_rho) < TOL[prec], pb
    finally:
        ctx.set_tuning(**saved)


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_tuning_candidates(system, prec):
    """Every launch-parameter set the autotuner tries (plane bands per CTA,
    band batch, z-pass columns) gives the oracle's op_H."""
    import torch
    import pwb200
    from oracle import ops
    H, ctx, psis = system
    dt = torch.complex128 if prec == "c128" else torch.complex64
    ik = len(psis) - 1
    ref = ops.op_H(H, psis[ik], ik)
    x = to_dev(psis[ik], dt)
    y = torch.empty_like(x)
    saved = ctx.get_tuning()
    try:
        for pb in (1, 2, 3):
            for ch in (1, 16, 96):
                for zc in (16, 32, 48, 64, 96, 128):
                    ctx.set_tuning(plane_bands=pb, band_chunk_bytes=ch << 20, z_columns=zc)
                    ctx.apply(ik, 0, x, y, pwb200.PW_OP_H)
                    assert rel_err(to_host(y), ref) < TOL[prec], (pb, ch, zc)
    finally:
        ctx.set_tuning(**saved)


@pytest.mark.parametrize("prec", ["c128", "c64"])
@pytest.mark.parametrize("term", ["K", "VLOC", "VNL"])
def test_op_terms_accumulate(system, prec, term):
    """op_K!/op_V_loc!/op_V_Ps_nloc! accumulate into Hpsi."""
    import torch
    import pwb200
    from oracle import ops
    H, ctx, psis = system
    dt = torch.complex128 if prec == "c128" else torch.complex64
    ik = 0
    psi = psis[ik]
    base = 0.3 * psi[:, ::-1].copy()
    ref = base.copy()
    {"K": ops.op_K, "VLOC": ops.op_V_loc, "VNL": ops.op_V_Ps_nloc}[term](H, psi, ref, ik)
    x = to_dev(psi, dt)
    y = to_dev(base, dt)
    flag = {"K": pwb200.PW_OP_K, "VLOC": pwb200.PW_OP_VLOC, "VNL": pwb200.PW_OP_VNL}[term]
    ctx.apply(ik, 0, x, y, flag | pwb200.PW_ACCUMULATE)
    assert rel_err(to_host(y), ref) < TOL[prec]


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_kprec(system, prec):
    """Kprec in FP64 and in the FP32 form the mixed-precision eigensolvers use
    (FP32 result: one rounding of the scaled value)."""
    import torch
    from oracle import ops
    H, ctx, psis = system
    dt = torch.complex128 if prec == "c128" else torch.complex64
    x = to_dev(psis[0], dt)
    y = torch.empty_like(x)
    ctx.kprec(0, x, y)
    ref = ops.Kprec(H, to_host(x), 0)
    assert rel_err(to_host(y), ref) < (1e-14 if prec == "c128" else 2e-7)


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_calc_rhoe(system, prec):
    import torch
    from oracle import ops
    H, ctx, psis = system
    nb = psis[0].shape[1]
    Focc = np.linspace(2.0, 0.0, nb)[:, None] * np.ones((1, len(psis)))
    ref = ops.calc_rhoe(H, psis, Focc=Focc)
    dt = torch.complex128 if prec == "c128" else torch.complex64
    rho = torch.zeros(H.pw.Npoints, dtype=torch.float64, device="cuda")
    for ik, psi in enumerate(psis):
        ctx.calc_rhoe(ik, to_dev(psi, dt), H.pw.kpoints.wk[ik] * Focc[:, ik], rho, accumulate=(ik > 0))
    got = rho.cpu().numpy()
    assert rel_err(got, ref) < TOL[prec]
    # charge: sum(rho) dVol = sum_k wk sum_b Focc |psi_b|^2
    q = sum(H.pw.kpoints.wk[ik] * np.sum(Focc[:, ik] * np.sum(np.abs(p) ** 2, axis=0)) for ik, p in enumerate(psis))
    assert abs(got.sum() * H.pw.CellVolume / H.pw.Npoints - q) < (1e-10 if prec == "c128" else 1e-5) * q


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_gram_and_rotate(system, prec):
    import torch
    H, ctx, psis = system
    dt = torch.complex128 if prec == "c128" else torch.complex64
    A = psis[0]
    B = psis[0][:, ::-1].copy() * (1 + 0.5j)
    G = torch.zeros((B.shape[1], A.shape[1]), dtype=torch.complex128, device="cuda")
    ctx.gram(to_dev(A, dt), to_dev(B, dt), G)
    ref = A.conj().T @ B
    assert rel_err(G.cpu().numpy().T, ref) < TOL[prec]
    rng = np.random.default_rng(3)
    U = rng.standard_normal((A.shape[1], 5)) + 1j * rng.standard_normal((A.shape[1], 5))
    out = torch.zeros((5, A.shape[0]), dtype=dt, device="cuda")
    ctx.rotate(to_dev(A, dt), torch.from_numpy(np.ascontiguousarray(U.T)).cuda(), out)
    assert rel_err(to_host(out), A @ U) < TOL[prec]
    ctx.check_device()   # no bounded device-side wait expired


@pytest.mark.parametrize("m", [480, 1440])
def test_gram_long_k_accuracy(system, m):
    """Overlap of an orthonormal FP32 block at the Si216 size (K = 80797
    plane waves): the split-BF16x3 Gram stays at its per-term error, with no
    drift from long tensor-core accumulation chains (the 480-band Gram was
    off by 1e-4 when all of K went through one chain)."""
    import torch
    H, ctx, psis = system
    if psis[0].shape[0] < 10000:
        pytest.skip("one size suffices")
    K = 80797
    g = torch.Generator(device="cuda").manual_seed(11)
    X = torch.randn((K, m), dtype=torch.complex128, device="cuda", generator=g)
    Q, _ = torch.linalg.qr(X)
    X32 = Q.T.contiguous().to(torch.complex64)
    G = torch.zeros((m, m), dtype=torch.complex128, device="cuda")
    ctx.gram(X32, X32, G)
    Xd = X32.to(torch.complex128)
    exact = Xd.conj() @ Xd.T
    assert (G - exact).abs().max().item() < 2e-5
    ctx.check_device()


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_host_dropin(system, prec):
    import pwb200
    from oracle import ops
    H, ctx, psis = system
    ik = len(psis) // 2
    code = pwb200.PW_C128 if prec == "c128" else pwb200.PW_C64
    got = ctx.op_H_host(ik, 0, psis[ik], dtype=code)
    assert rel_err(got, ops.op_H(H, psis[ik], ik)) < TOL[prec]
    w = np.full(psis[ik].shape[1], 0.5)
    rho = ctx.calc_rhoe_host(ik, psis[ik], w, dtype=code)
    from oracle.ham import G_to_R
    ct = np.zeros((psis[ik].shape[1], H.pw.Npoints), dtype=np.complex128)
    ct[:, H.pw.gvecw.idx_gw2r[ik]] = psis[ik].T
    ct = G_to_R(H.pw.Ns, ct) * (H.pw.Npoints / np.sqrt(H.pw.CellVolume))
    ref = (w[:, None] * np.abs(ct) ** 2).sum(axis=0)
    assert rel_err(rho, ref) < TOL[prec]


def test_errors_are_status_codes(system):
    import torch
    import pwb200
    H, ctx, psis = system
    x = to_dev(psis[0], torch.complex128)
    with pytest.raises(pwb200.PWError) as e:
        ctx.apply(len(psis), 0, x, torch.empty_like(x))
    assert e.value.status == 1
    with pytest.raises(pwb200.PWError):
        ctx.apply(0, 0, x, x)                       # aliasing
    with pytest.raises(pwb200.PWError):
        ctx.apply(0, 3, x, torch.empty_like(x))     # spin channel not set
    fresh = pwb200.Context(H.pw.Ns, H.pw.CellVolume, H.pw.gvecw.idx_gw2r[:1], [H.pw.Gk2(0)])
    with pytest.raises(pwb200.PWError) as e:
        fresh.apply(0, 0, x, torch.empty_like(x), pwb200.PW_OP_VLOC)
    assert e.value.status == 6
    fresh.close()
