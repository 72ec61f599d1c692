"""KS_solve_SCF! on the device (pwb200.scf) against the reference's golden
total energy and the FP64 oracle's converged SCF.

  Si fcc, GTH-Pade, LDA, ecutwfc 15 Ha, 3x3x3 MP (time reversal: 14 k),
  Pulay mixing beta = 0.2, etot_conv_thr 1e-8:
    FP64 path:  |Etot - ABINIT| < 1e-5 (test/validations_old/Si_fcc.jl:15)
                |Etot - oracle| < 2e-7, components within 2e-6
    mixed path (FP64 switch at |dE| < 1e-5): |Etot - ABINIT| < 1e-5
  The same with the Davidson solvers (Pulay beta 0.5 as
  test/validations_old/Si_fcc.jl:94-101): update_psi = "davidson" (the 2-block
  diag_davidson! of KS_solve_SCF.jl:194-198, FP64) and "davidson_qe"
  (diag_davidson_qe!, FP64 and mixed): |Etot - ABINIT| < 1e-5 and the FP64
  results within 2e-7 of the LOBPCG-driven oracle SCF.
"""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu
ABINIT = -7.9110087934


@pytest.fixture(scope="module")
def si_fcc_gpu():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from pwb200.system import kpoint_grid
    from oracle import systems
    Ho = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    k, w = kpoint_grid(Ho.atoms.LatVecs, (3, 3, 3))
    sysm = pwb200.System(["Si", "Si"], Ho.atoms.positions, Ho.atoms.LatVecs)
    H = pwb200.Hamiltonian(sysm, [systems.psp("Si-q4.gth")], 15.0, kpts=k, wk=w)
    yield H
    H.ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_scf_si_fcc(si_fcc_gpu, si_fcc_scf, precision):
    from pwb200 import scf
    res = scf.KS_solve_SCF(si_fcc_gpu, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-8, precision=precision)
    E = res["energies"]
    assert abs(E["Total"] - ABINIT) < 1e-5, res["log"][-3:]
    if precision == "fp64":
        _, Eo, _, _ = si_fcc_scf
        assert abs(E["Total"] - Eo["Total"]) < 2e-7
        for key in ("Kinetic", "Ps_loc", "Ps_nloc", "Hartree", "XC", "NN"):
            assert abs(E[key] - Eo[key]) < 2e-6, key
    else:
        assert res["switched_to_fp64_at"] is not None


@pytest.mark.parametrize("solver,precision", [("davidson", "fp64"), ("davidson_qe", "fp64"),
                                              ("davidson_qe", "mixed")])
def test_scf_si_fcc_davidson(si_fcc_gpu, si_fcc_scf, solver, precision):
    from pwb200 import scf
    res = scf.KS_solve_SCF(si_fcc_gpu, betamix=0.5, mix_method="pulay", etot_conv_thr=1e-8, precision=precision,
                           update_psi=solver)
    E = res["energies"]
    assert abs(E["Total"] - ABINIT) < 1e-5, res["log"][-3:]
    if precision == "fp64":
        _, Eo, _, _ = si_fcc_scf
        assert abs(E["Total"] - Eo["Total"]) < 2e-7


def test_device_pulay_mixing_matches_oracle():
    """pw_mix_pulay (ring history, F'F updated by one row per iteration,
    on-device solve) against the oracle's mix_pulay (mix_pulay.jl:1-41)
    step by step on seeded densities: mixdim 3, 9 iterations (Pulay from
    the 4th), clamping at eps(); then a new history (iter = 1) restarts."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from oracle.scf import mix_pulay
    from oracle import systems
    Ho = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    pw = Ho.pw
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    rng = np.random.default_rng(17)
    n, mixdim, beta = pw.Npoints, 3, 0.3
    for rep in range(2):
        x_o = np.abs(rng.standard_normal(n)) * 0.05
        x_d = torch.from_numpy(x_o.copy()).cuda()
        X, F, state = np.zeros((n, mixdim)), np.zeros((n, mixdim)), {}
        for it in range(1, 10):
            # a contracting "SCF map" with a little noise
            gx = 0.6 * x_o + 0.4 * np.abs(np.sin(0.001 * np.arange(n) * it)) * 0.05 + 1e-4 * rng.standard_normal(n)
            x_o = np.maximum(mix_pulay(x_o, gx, beta, X, F, it, mixdim, state), np.finfo(np.float64).eps)
            ctx.mix_pulay(x_d, torch.from_numpy(gx).cuda(), beta, it, mixdim, clamp=True)
            got = x_d.cpu().numpy()
            assert np.abs(got - x_o).max() < 1e-10 * np.abs(x_o).max(), (rep, it)
            x_d = torch.from_numpy(x_o.copy()).cuda()   # both continue from the oracle's x
    ctx.close()
