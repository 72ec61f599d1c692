"""The SCF-level drivers: KS_solve_Emin_PCG! (KS_solve_Emin_PCG.jl:27-270,
direct minimisation) and the host logic of KS_solve_SCF.

CPU:
  - the oracle's direct minimisation on Si fcc (3x3x3 MP, 14 k) reaches
    ABINIT's total energy (test/validations_old/Si_fcc.jl:15) within 1e-7 Ha;
  - the device drivers (pwb200.emin_scf, and pwb200.scf with LOBPCG and with
    CheFSI), run on the NumPy stand-in for the library (block operations,
    pw_update sums, pw_calc_rhoe and pw_band_energies through the oracle),
    reproduce the oracle drivers' energies step by step (1e-9 Ha) on a 2x2x2
    mesh.
GPU: the direct minimisation on Si fcc 3x3x3 reaches ABINIT's energy.
"""
import numpy as np
import pytest

from numpy_ctx import HostHam, SCFCtx  # noqa: F401

ABINIT = -7.9110087934


def test_oracle_emin_pcg_matches_abinit():
    from oracle import systems, scf, emin_scf
    H = systems.Ham_Si_fcc(meshk=(3, 3, 3))
    psiks = scf.rand_BlochWavefunc(H, seed=1234)
    E, ev, it = emin_scf.KS_solve_Emin_PCG(H, psiks, etot_conv_thr=1e-7)
    assert it < 60 and abs(E["Total"] - ABINIT) < 1e-7, (it, E["Total"])


def test_device_driver_matches_oracle_driver():
    import torch
    from oracle import systems, scf, emin_scf
    from pwb200.emin_scf import KS_solve_Emin_PCG
    Ho = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    start = scf.rand_BlochWavefunc(Ho, seed=7)
    log_o = []
    E_o, ev_o, it_o = emin_scf.KS_solve_Emin_PCG(Ho, [p.copy() for p in start], etot_conv_thr=1e-7, log=log_o)
    Hd = HostHam(systems.Ham_Si_fcc(meshk=(2, 2, 2)), (2, 2, 2))
    assert Hd.basis.Nkpt == Ho.pw.kpoints.Nkpt
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    res = KS_solve_Emin_PCG(Hd, ps, etot_conv_thr=1e-7)
    assert res["iterations"] == it_o
    for (i1, e1, _), (i2, e2, _) in zip(log_o, res["log"]):
        assert i1 == i2 and abs(e1 - e2) < 1e-9, (i1, e1, e2)
    assert abs(res["energies"]["Total"] - E_o["Total"]) < 1e-9
    assert np.abs(res["evals"] - ev_o).max() < 1e-8


@pytest.mark.gpu
def test_emin_pcg_gpu_si_fcc():
    """The device driver on Si fcc (3x3x3 MP, 14 k) reaches ABINIT's energy."""
    from conftest import cuda_ok
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from pwb200.emin_scf import KS_solve_Emin_PCG
    from pwb200.system import kpoint_grid
    from oracle import systems
    Ho = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    k, w = kpoint_grid(Ho.atoms.LatVecs, (3, 3, 3))
    sysm = pwb200.System(["Si", "Si"], Ho.atoms.positions, Ho.atoms.LatVecs)
    H = pwb200.Hamiltonian(sysm, [systems.psp("Si-q4.gth")], 15.0, kpts=k, wk=w)
    try:
        res = KS_solve_Emin_PCG(H, etot_conv_thr=1e-7)
    finally:
        H.ctx.close()
    assert res["iterations"] < 60 and abs(res["energies"]["Total"] - ABINIT) < 1e-6, res["log"][-3:]


def test_scf_driver_matches_oracle_driver():
    """The device SCF driver (pwb200.scf.KS_solve_SCF, LOBPCG, Pulay 0.2) on
    the NumPy stand-in reproduces the oracle's KS_solve_SCF step by step:
    ethr schedule, Pulay mixing, the rho >= eps clamp, energies and the
    convergence test (KS_solve_SCF.jl:24-373)."""
    import torch
    from oracle import systems, scf as oscf
    from pwb200 import scf
    Ho = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    start = oscf.rand_BlochWavefunc(Ho, seed=11)
    log_o = []
    E_o, _, _ = oscf.KS_solve_SCF(Ho, psiks=[p.copy() for p in start], betamix=0.2, mix_method="pulay",
                                  etot_conv_thr=1e-7, log=log_o)
    Hd = HostHam(systems.Ham_Si_fcc(meshk=(2, 2, 2)), (2, 2, 2))
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    res = scf.KS_solve_SCF(Hd, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-7, precision="fp64", psiks=ps)
    assert res["iterations"] == len(log_o)
    for row_o, row_d in zip(log_o, res["log"]):
        assert row_o[0] == row_d[0] and abs(row_o[1] - row_d[1]) < 1e-9, (row_o, row_d)
    assert abs(res["energies"]["Total"] - E_o["Total"]) < 1e-9


def test_chefsi_scf_driver_matches_oracle():
    """KS_solve_SCF(update_psi="CheFSI") on the NumPy stand-in follows the
    oracle's SCF driven by diag_CheFSI (CheFSI.jl:1-31) step by step, with
    the same Lanczos start vectors (first 12 iterations, 1e-9 Ha)."""
    import torch
    from oracle import systems, scf as oscf, chefsi
    from pwb200 import scf

    class CheCtx(SCFCtx):
        def chebyfilt(self, ik, ispin, X, Y, degree, lb, ub):
            Y.copy_(torch.from_numpy(np.ascontiguousarray(
                chefsi.chebyfilt(self.H, X.numpy().T.copy(), degree, lb, ub, ik).T)))

        def lanczos_bounds(self, ik, ispin, nlancz, v0):
            ub, lb, _ = chefsi.get_ub_lb_lanczos(self.H, nlancz, v0.numpy(), ik)
            return ub, lb

    seed = 5
    Ho = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    start = oscf.rand_BlochWavefunc(Ho, seed=seed)
    rng = np.random.default_rng(seed + 1)      # the driver's Lanczos generator

    def diag(Ham, psiks, tol, nconv):
        ev = []
        for ik in range(len(psiks)):
            ngw = psiks[ik].shape[0]
            v0 = rng.standard_normal(ngw) + 1j * rng.standard_normal(ngw)
            psiks[ik], e = chefsi.diag_CheFSI_k(Ham, psiks[ik], 8, v0, ik)
            ev.append(e)
        return np.stack(ev, axis=1)

    log_o = []
    oscf.KS_solve_SCF(Ho, psiks=[p.copy() for p in start], betamix=0.2, mix_method="pulay", NiterMax=12,
                      etot_conv_thr=1e-12, diag=diag, log=log_o)
    Hd = HostHam(systems.Ham_Si_fcc(meshk=(2, 2, 2)), (2, 2, 2))
    Hd.ctx = CheCtx(Hd.ctx.H)
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    res = scf.KS_solve_SCF(Hd, betamix=0.2, mix_method="pulay", NiterMax=12, etot_conv_thr=1e-12, precision="fp64",
                           psiks=ps, update_psi="CheFSI", cheby_degree=8, seed=seed)
    assert len(res["log"]) == len(log_o) == 12
    for row_o, row_d in zip(log_o, res["log"]):
        assert abs(row_o[1] - row_d[1]) < 1e-9, (row_o, row_d)


def test_pcg_scf_driver_matches_oracle():
    """KS_solve_SCF(update_psi="PCG") on the NumPy stand-in follows the
    oracle's SCF driven by diag_Emin_PCG! (KS_solve_SCF.jl:199-203) step by
    step, and converges to the LOBPCG SCF's energy.  The PCG's line search
    amplifies rounding differences (traces of Grams against vdot) from step
    to step, so the steps agree to 1e-6 Ha rather than 1e-9 and the step
    counts to within 2."""
    import torch
    from oracle import systems, scf as oscf, emin_pcg
    from pwb200 import scf

    Ho = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    start = oscf.rand_BlochWavefunc(Ho, seed=3)

    def diag(Ham, psiks, tol, nconv):
        ev = []
        for ik in range(len(psiks)):
            e, _, _ = emin_pcg.diag_Emin_PCG(Ham, psiks[ik], ik, tol=tol, NiterMax=100, Nstates_conv=nconv)
            ev.append(e)
        return np.stack(ev, axis=1)

    log_o = []
    E_o, _, _ = oscf.KS_solve_SCF(Ho, psiks=[p.copy() for p in start], betamix=0.2, mix_method="pulay",
                                  etot_conv_thr=1e-7, diag=diag, log=log_o)
    Hd = HostHam(systems.Ham_Si_fcc(meshk=(2, 2, 2)), (2, 2, 2))
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    res = scf.KS_solve_SCF(Hd, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-7, precision="fp64", psiks=ps,
                           update_psi="PCG")
    assert abs(len(res["log"]) - len(log_o)) <= 2
    for row_o, row_d in zip(log_o, res["log"]):
        assert abs(row_o[1] - row_d[1]) < 1e-6, (row_o, row_d)
    assert abs(res["energies"]["Total"] - E_o["Total"]) < 1e-6
    Ho2 = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    E_l, _, _ = oscf.KS_solve_SCF(Ho2, psiks=[p.copy() for p in start], betamix=0.2, mix_method="pulay",
                                  etot_conv_thr=1e-7)
    assert abs(res["energies"]["Total"] - E_l["Total"]) < 1e-6


def test_davidson_scf_driver_matches_oracle():
    """KS_solve_SCF(update_psi="davidson") runs the 2-block diag_davidson! per
    k-point, as KS_solve_SCF.jl:194-198 does: on the NumPy stand-in it follows
    the oracle's SCF driven by the oracle's diag_davidson step by step (same
    energies to 1e-9 Ha, same number of SCF steps)."""
    import torch
    from oracle import systems, scf as oscf, davidson
    from pwb200 import scf

    Ho = systems.Ham_Si_fcc(meshk=(2, 2, 2))
    start = oscf.rand_BlochWavefunc(Ho, seed=5)

    def diag(Ham, psiks, tol, nconv):
        ev = []
        for ik in range(len(psiks)):
            e, _, _ = davidson.diag_davidson(Ham, psiks[ik], ik, tol=tol, NiterMax=100, Nstates_conv=nconv)
            ev.append(e)
        return np.stack(ev, axis=1)

    log_o = []
    E_o, _, _ = oscf.KS_solve_SCF(Ho, psiks=[p.copy() for p in start], betamix=0.2, mix_method="pulay",
                                  etot_conv_thr=1e-8, diag=diag, log=log_o)
    Hd = HostHam(systems.Ham_Si_fcc(meshk=(2, 2, 2)), (2, 2, 2))
    ps = [torch.from_numpy(np.ascontiguousarray(p.T)) for p in start]
    res = scf.KS_solve_SCF(Hd, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8, precision="fp64", psiks=ps,
                           update_psi="davidson")
    assert len(res["log"]) == len(log_o)
    for row_o, row_d in zip(log_o, res["log"]):
        assert abs(row_o[1] - row_d[1]) < 1e-9, (row_o, row_d)
    assert abs(res["energies"]["Total"] - E_o["Total"]) < 1e-9


def test_scf_rejects_unsupported_choices():
    from oracle import systems
    from pwb200 import scf
    Hd = HostHam(systems.Ham_Si_fcc(meshk=(1, 1, 1)), (1, 1, 1))
    with pytest.raises(ValueError):
        scf.KS_solve_SCF(Hd, update_psi="PCG", precision="mixed")
    with pytest.raises(ValueError):
        scf.KS_solve_SCF(Hd, update_psi="nonexistent")
    with pytest.raises(ValueError):
        scf.KS_solve_SCF(Hd, update_psi="davidson", precision="mixed")
    for m in ("broyden", "anderson", "nonexistent"):
        with pytest.raises(ValueError):
            scf.KS_solve_SCF(Hd, mix_method=m)
