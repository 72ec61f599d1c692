"""Fermi-Dirac smearing (occupations.jl, KS_solve_SCF.jl:218-223).

  host: pwb200.scf.smeared_occupations vs the oracle's calc_Focc / calc_entropy
        on seeded eigenvalues (Focc 1e-12, E_fermi 1e-10, mTS 1e-12)
  device SCF: Pt fcc (test/validations_old/Pt_fcc.jl:1-50, GTH Pt-q10 with d
        projectors, ecutwfc 30, 3x3x3 k, kT = 1e-3, simple mixing beta 0.5):
        free energy vs ABINIT -26.2945054360 (1e-5), FP64 components and -TS vs
        the reference log (test/LOG_runtest_v.1.1.1:2649-2660, its Ps_loc plus
        PspCore) within 1e-6, mixed precision vs ABINIT within 1e-5
"""
import numpy as np
import pytest

from conftest import cuda_ok

ABINIT_PT = -26.2945054360


def test_smeared_occupations_match_oracle():
    from oracle import occupations
    from pwb200.scf import smeared_occupations
    rng = np.random.default_rng(4)
    evals = np.sort(rng.uniform(-0.3, 0.6, (10, 35)), axis=0)
    wk = rng.uniform(0.5, 1.5, 35)
    wk /= wk.sum()
    for kT in (1e-3, 1e-2):
        F, Ef, mTS = smeared_occupations(12.0, wk, kT, evals)
        Fo, Efo = occupations.calc_Focc(12.0, wk, kT, evals)
        assert abs(Ef - Efo) < 1e-10
        assert np.abs(F - Fo).max() < 1e-9
        assert abs(mTS - occupations.calc_entropy(wk, kT, evals, Efo)) < 1e-11
        assert abs(float(np.sum(wk[None, :] * F)) - 12.0) < 1e-8


def _pt_device():
    import pwb200
    from pwb200.system import kpoint_grid
    from oracle import systems
    at = systems.pt_fcc_atoms()
    k, w = kpoint_grid(at.LatVecs, (3, 3, 3))
    sysm = pwb200.System(["Pt"], at.positions, at.LatVecs)
    return pwb200.Hamiltonian(sysm, [systems.psp("Pt-q10.gth")], 30.0, kpts=k, wk=w)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_scf_pt_fcc_smearing(precision):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from pwb200 import scf
    H = _pt_device()
    res = scf.KS_solve_SCF(H, Nstates=9, betamix=0.5, mix_method="simple", etot_conv_thr=1e-8, precision=precision,
                           use_smearing=True, kT=1e-3)
    E = res["energies"]
    assert abs(E["Total"] - ABINIT_PT) < 1e-5, res["log"][-3:]
    if precision == "fp64":
        assert abs(E["mTS"] - (-0.0005158875)) < 1e-8
        assert abs(E["Kinetic"] - 19.2060140731) < 1e-6
        assert abs(E["Ps_loc"] - (-3.5178517592 + 6.3258423493)) < 1e-6
        assert abs(E["Ps_nloc"] - (-14.7734350216)) < 1e-6
        assert abs(E["Hartree"] - 1.8623453874) < 1e-6
        assert abs(E["XC"] - (-4.4748717329)) < 1e-6
        assert abs(res["E_fermi"] - (-0.0148842322 + 6.3258423493 / 10.0)) < 1e-6
    H.ctx.close()
