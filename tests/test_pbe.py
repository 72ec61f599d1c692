"""PBE exchange-correlation (GGA_PBE_internal.jl, XC_funcs/XC_x_pbe.jl,
XC_c_pw.jl, XC_c_pbe.jl; op_nabla / op_nabla_dot of PWGrid.jl:351-398).

Oracle pins:
  test/validations_old/Si_fcc_PBE.jl:15     Etot(Si fcc, PBE) = -7.8539427130 (ABINIT, atol 1e-5)
  test/LOG_runtest_v.1.1.1:2002-2012        logged components of that run (Libxc PBE,
                                            SCF stopped at dE ~ 1e-6: components to 3e-6)
  V_xc = dE_xc/drho                         central differences of the oracle's E_xc
Device (pw_update with pw_set_xc(PW_XC_PBE)) against the oracle: V_xc and
V_tot within 1e-10 relative, E_xc within 1e-10 Ha; the device SCF on Si fcc
PBE (3x3x3 k) against ABINIT and the oracle.
"""
import numpy as np
import pytest

from conftest import cuda_ok

ABINIT_PBE = -7.8539427130


def _ham_pbe(meshk=(3, 3, 3)):
    from oracle import systems, ham
    return ham.Hamiltonian(systems.si_fcc_atoms(), [systems.psp("Si-q4-pbe.gth")], 15.0, meshk=meshk, xcfunc="PBE")


def test_pbe_potential_is_functional_derivative():
    """sum V_xc drho dVol = (E_xc[rho + h drho] - E_xc[rho - h drho]) / 2h for a
    smooth perturbation drho of the starting density (checks v1, v2 and the
    divergence term together)."""
    from oracle import pbe
    H = _ham_pbe(meshk=(1, 1, 1))
    pw = H.pw
    rho = H.guess_rhoe()
    dVol = pw.CellVolume / pw.Npoints
    idx = np.arange(pw.Npoints)
    drho = 0.01 * rho * np.cos(0.001 * idx) + 1e-3 * np.sin(0.0007 * idx) ** 2

    def Exc(r):
        return float(np.sum(pbe.calc_epsxc_PBE(pw, r) * r)) * dVol

    h = 1e-4
    fd = (Exc(rho + h * drho) - Exc(rho - h * drho)) / (2 * h)
    an = float(np.sum(pbe.calc_Vxc_PBE(pw, rho) * drho)) * dVol
    assert abs(fd - an) < 1e-7 * abs(an), (fd, an)


@pytest.mark.slow
def test_si_fcc_pbe_total_energy():
    from oracle import scf
    H = _ham_pbe()
    E, _, _ = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8)
    assert abs(E["Total"] - ABINIT_PBE) < 1e-5
    assert abs(E["Kinetic"] - 3.1938247323) < 3e-6
    assert abs(E["Ps_loc"] - (-2.1493161546 - 0.2098909668)) < 3e-6
    assert abs(E["Ps_nloc"] - 1.5608465719) < 3e-6
    assert abs(E["Hartree"] - 0.5765247087) < 3e-6
    assert abs(E["XC"] - (-2.4280048103)) < 3e-6


def _device_ham(xcfunc, meshk=(1, 1, 1)):
    import pwb200
    from pwb200.system import kpoint_grid
    from oracle import systems
    at = systems.si_fcc_atoms()
    kw = {}
    if meshk != (1, 1, 1):
        k, w = kpoint_grid(at.LatVecs, meshk)
        kw = dict(kpts=k, wk=w)
    sysm = pwb200.System(["Si", "Si"], at.positions, at.LatVecs)
    return pwb200.Hamiltonian(sysm, [systems.psp("Si-q4-pbe.gth")], 15.0, xcfunc=xcfunc, **kw)


@pytest.mark.gpu
def test_device_pbe_update_vs_oracle():
    """pw_update with PBE on the starting density of Si fcc: V_xc, V_tot and
    the three energy sums against the oracle's update! and calc_E_local."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    from oracle import energies
    Ho = _ham_pbe(meshk=(1, 1, 1))
    rho = Ho.guess_rhoe()
    Ho.update(rho)
    E_ps, E_h, E_xc = energies.calc_E_local(Ho, rho)
    H = _device_ham("PBE")
    H.setup_density()
    dev = "cuda:0"
    r = torch.from_numpy(rho).to(dev)
    Vps = torch.from_numpy(H.V_Ps_loc).to(dev)
    VH = torch.zeros_like(r)
    Vxc = torch.zeros_like(r)
    sums = H.ctx.update(r, Vps, VH, Vxc)
    dVol = Ho.pw.CellVolume / Ho.pw.Npoints
    vx = Vxc.cpu().numpy()
    assert np.abs(vx - Ho.V_xc).max() < 1e-10 * np.abs(Ho.V_xc).max()
    assert np.abs(VH.cpu().numpy() - Ho.V_Hartree).max() < 1e-10 * np.abs(Ho.V_Hartree).max()
    assert abs(sums[2] * dVol - E_xc) < 1e-10
    assert abs(0.5 * sums[0] * dVol - E_h) < 1e-10
    assert abs(sums[1] * dVol - E_ps) < 1e-10
    H.ctx.check_device()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_scf_si_fcc_pbe(precision):
    """KS_solve_SCF on the device with PBE (Si_fcc_PBE.jl, Pulay beta 0.2):
    |Etot - ABINIT| < 1e-5; the FP64 run within 2e-7 of the oracle's SCF."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from pwb200 import scf
    H = _device_ham("PBE", meshk=(3, 3, 3))
    res = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8, precision=precision)
    E = res["energies"]
    assert abs(E["Total"] - ABINIT_PBE) < 1e-5, res["log"][-3:]
    if precision == "fp64":
        from oracle import scf as oscf
        Eo, _, _ = oscf.KS_solve_SCF(_ham_pbe(), betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8)
        assert abs(E["Total"] - Eo["Total"]) < 2e-7
        assert abs(E["XC"] - Eo["XC"]) < 2e-6
    H.ctx.close()
