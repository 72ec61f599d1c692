"""Adjoint of op_V_loc with respect to the potential (pw_vloc_vjp): dE/dV_loc(r).

  - lam = psi, w = wk*Focc: dE/dV_loc(r) of the band energy, equal to the
    oracle's calc_rhoe (calc_rhoe.jl:51-78) times dVol (FP64 1e-11, FP32 2e-5
    relative);
  - general cotangent lam != psi against the oracle's
    N Re(conj(G_to_R lam) G_to_R psi);
  - central differences of the device energy in V: the band energy
    sum_b w_b <psi_b|H(V + h dV)|psi_b> and L = sum_b w_b Re<lam_b|V psi_b>
    (linear in V, so the difference quotient is exact up to rounding);
  - Hellmann-Feynman: the derivative of the self-consistent total energy of
    Si fcc under an external smooth dV (two device SCFs at +-h) equals
    sum_r dE/dV_loc(r) dV(r) from the converged wavefunctions;
  - the autograd wrappers (pwb200.adjoint) return the same gradients.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


def smooth(pw, rng, g2max=4.0):
    g = pw.gvec
    sel = g.G2 <= g2max
    c = np.zeros(pw.Npoints, dtype=np.complex128)
    c[g.idx_g2r[sel]] = rng.standard_normal(sel.sum()) + 1j * rng.standard_normal(sel.sum())
    N1, N2, N3 = pw.Ns
    f = np.fft.ifftn(c.reshape(N3, N2, N1)).real.ravel()
    return f / np.abs(f).max()


@pytest.fixture(scope="module")
def si64():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    H = systems.Ham_Si64(Nstates=160)
    pw = H.pw
    rng = np.random.default_rng(9)
    H.V_Total = H.V_Ps_loc + 0.01 * smooth(pw, rng)
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    ctx.set_vloc(H.V_Total)
    ctx.set_nonlocal(0, H.betaNL[0])
    ctx.set_nonlocal_coef(H.nl_triplets)
    ngw, nb = pw.gvecw.Ngw[0], 24
    psi = (rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb))) / np.sqrt(ngw)
    lam = (rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb))) / np.sqrt(ngw)
    w = np.linspace(2.0, 0.5, nb)
    yield H, ctx, psi, lam, w, rng
    ctx.close()


def to_dev(a, dt):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().to(dt).contiguous()


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_dE_dVloc_is_density_times_dvol(si64, prec):
    import torch
    from oracle import ops
    H, ctx, psi, lam, w, _ = si64
    pw = H.pw
    dt = torch.complex128 if prec == "c128" else torch.complex64
    dV = torch.zeros(pw.Npoints, dtype=torch.float64, device="cuda")
    ctx.vloc_vjp(0, to_dev(psi, dt), w, dV)
    ref = ops.calc_rhoe(H, [psi], Focc=w[:, None]) * pw.CellVolume / pw.Npoints
    assert rel(dV.cpu().numpy(), ref) < (1e-11 if prec == "c128" else 2e-5)


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_vjp_general_cotangent_vs_oracle(si64, prec):
    import torch
    from oracle.ham import G_to_R
    H, ctx, psi, lam, w, _ = si64
    pw = H.pw
    dt = torch.complex128 if prec == "c128" else torch.complex64
    dV = torch.zeros(pw.Npoints, dtype=torch.float64, device="cuda")
    ctx.vloc_vjp(0, to_dev(psi, dt), w, dV, lam=to_dev(lam, dt))

    def real_space(a):
        ct = np.zeros((a.shape[1], pw.Npoints), dtype=np.complex128)
        ct[:, pw.gvecw.idx_gw2r[0]] = a.T
        return G_to_R(pw.Ns, ct)
    up, ul = real_space(psi), real_space(lam)
    ref = pw.Npoints * (w[:, None] * np.real(np.conj(ul) * up)).sum(axis=0)
    # FP32: the polarised form carries an error of ~1e-7 (|psi|^2 + |lam|^2)
    assert rel(dV.cpu().numpy(), ref) < (1e-10 if prec == "c128" else 5e-5)


def test_central_differences_of_device_energies(si64):
    import torch
    import pwb200
    H, ctx, psi, lam, w, rng = si64
    pw = H.pw
    x = to_dev(psi, torch.complex128)
    l = to_dev(lam, torch.complex128)
    dV = torch.zeros(pw.Npoints, dtype=torch.float64, device="cuda")
    dL = torch.zeros_like(dV)
    ctx.vloc_vjp(0, x, w, dV)
    ctx.vloc_vjp(0, x, w, dL, lam=l)
    dpot = smooth(pw, rng, g2max=6.0)
    wt = torch.from_numpy(w).cuda()

    def energies(V):
        ctx.set_vloc(V)
        y = torch.empty_like(x)
        ctx.apply(0, 0, x, y, pwb200.PW_OP_H)
        e_band = float((wt * torch.real(torch.sum(x.conj() * y, dim=1))).sum())
        ctx.apply(0, 0, x, y, pwb200.PW_OP_VLOC)
        e_l = float((wt * torch.real(torch.sum(l.conj() * y, dim=1))).sum())
        return e_band, e_l
    h = 1e-3
    ep, lp = energies(H.V_Total + h * dpot)
    em, lm = energies(H.V_Total - h * dpot)
    ctx.set_vloc(H.V_Total)
    d = torch.from_numpy(dpot).cuda()
    an_e = float(torch.dot(dV, d))
    an_l = float(torch.dot(dL, d))
    assert abs((ep - em) / (2 * h) - an_e) < 1e-9 * abs(an_e)
    assert abs((lp - lm) / (2 * h) - an_l) < 1e-8 * max(abs(an_l), 1e-3)


def test_hellmann_feynman_self_consistent_energy():
    """Si fcc (Gamma only): E_tot(h) of two device SCFs with V_ps + h dV,
    central difference against sum_r dE/dV_loc(r) dV(r) at h = 0."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from pwb200 import scf
    from oracle import systems
    Ho = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    sysm = pwb200.System(["Si", "Si"], Ho.atoms.positions, Ho.atoms.LatVecs)
    H = pwb200.Hamiltonian(sysm, [systems.psp("Si-q4.gth")], 15.0)
    V0 = H.V_Ps_loc.copy()
    dpot = 0.05 * smooth(Ho.pw, np.random.default_rng(2), g2max=3.0)
    kw = dict(betamix=0.3, mix_method="pulay", etot_conv_thr=1e-12, NiterMax=200, precision="fp64", seed=1)
    res0 = scf.KS_solve_SCF(H, **kw)
    nb = res0["psiks"][0].shape[0]
    dV = torch.zeros(H.basis.Npoints, dtype=torch.float64, device="cuda")
    H.ctx.vloc_vjp(0, res0["psiks"][0], H.wk[0] * res0["Focc"][:, 0], dV)
    an = float(torch.dot(dV, torch.from_numpy(dpot).cuda()))
    h = 1e-3
    E = []
    for s in (1, -1):
        H.V_Ps_loc = V0 + s * h * dpot
        E.append(scf.KS_solve_SCF(H, **kw)["energies"]["Total"])
    H.V_Ps_loc = V0
    fd = (E[0] - E[1]) / (2 * h)
    assert nb >= 4 and abs(fd - an) < 1e-5 * abs(an) + 1e-7, (fd, an)
    H.ctx.close()


def test_autograd_wrappers(si64):
    import torch
    from pwb200 import adjoint
    H, ctx, psi, lam, w, rng = si64
    pw = H.pw
    x = to_dev(psi, torch.complex128)
    V = torch.from_numpy(H.V_Total.copy()).cuda().requires_grad_(True)
    E = adjoint.local_band_energy(ctx, 0, V, x, w)
    E.backward()
    dV = torch.zeros(pw.Npoints, dtype=torch.float64, device="cuda")
    ctx.vloc_vjp(0, x, w, dV)
    assert torch.allclose(V.grad, dV, rtol=0, atol=1e-14 * float(dV.abs().max()))
    assert abs(float(E) - float(torch.dot(V.detach(), dV))) < 1e-12 * abs(float(E))
