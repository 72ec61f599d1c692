"""Ionic forces (calc_forces.jl: NN + Ps_loc + Ps_nloc for GTH).

The reference has no force golden numbers, so the oracle's forces are
pinned against central finite differences of its own SCF total energy,
and the device forces against the oracle on the same wavefunctions and
density (FP64 1e-10 Ha/bohr, mixed 1e-6), and against finite differences
of the device SCF energy on a displaced Si64 cell with PBE (config C4).
"""
import numpy as np
import pytest

from conftest import cuda_ok


def _si_fcc_displaced():
    from oracle import systems
    at0 = systems.si_fcc_atoms()
    pos = at0.positions.copy()
    pos[:, 1] += np.array([0.05, -0.03, 0.02])
    return at0, pos


def _oracle_ham(pos, meshk=(1, 1, 1)):
    from oracle import systems, ham
    from oracle.ham import Atoms
    at0 = systems.si_fcc_atoms()
    return ham.Hamiltonian(Atoms(at0.atsymbs, pos, at0.LatVecs), [systems.psp("Si-q4.gth")], 15.0, meshk=meshk)


def test_oracle_forces_match_finite_differences():
    """-dE/dx of the converged FP64 oracle SCF (central differences, h = 1e-3
    bohr) against calc_forces for one component of a displaced Si fcc cell."""
    from oracle import scf, forces
    _, pos = _si_fcc_displaced()
    H = _oracle_ham(pos)
    E, psiks, rho = scf.KS_solve_SCF(H, etot_conv_thr=1e-11, ethr_evals_last=1e-11)
    F = forces.calc_forces(H, psiks, rho)
    assert np.abs(F.sum(axis=1)).max() < 1e-6          # no net force
    h = 1e-3
    Es = []
    for s in (+1, -1):
        p = pos.copy()
        p[0, 1] += s * h
        Es.append(scf.KS_solve_SCF(_oracle_ham(p), etot_conv_thr=1e-11, ethr_evals_last=1e-11)[0]["Total"])
    fd = -(Es[0] - Es[1]) / (2 * h)
    assert abs(fd - F[0, 1]) < 2e-6, (fd, F[0, 1])


def test_ewald_forces_host_vs_oracle():
    from oracle import forces
    from pwb200 import forces as pf
    _, pos = _si_fcc_displaced()
    H = _oracle_ham(pos)
    g = H.pw.gvec
    Fh = pf.ewald_forces(H.atoms.LatVecs, pos, H.Zvals[H.atoms.atm2species], g.G.T, g.G2, H.pw.ecutrho)
    Fo = forces.calc_forces_NN(H)
    assert np.abs(Fh - Fo).max() < 1e-12
    assert np.abs(Fh.sum(axis=1)).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_device_forces_vs_oracle(prec):
    """pw_forces_local / pw_forces_nonlocal against the oracle formulas on the
    same orthonormal wavefunctions and density (Si fcc, displaced, 2x2x2 k)."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from pwb200 import forces as pf
    from oracle import forces, lobpcg
    _, pos = _si_fcc_displaced()
    Ho = _oracle_ham(pos, meshk=(2, 2, 2))
    pw = Ho.pw
    rng = np.random.default_rng(5)
    psiks = [lobpcg.ortho_sqrt(rng.standard_normal((pw.gvecw.Ngw[ik], Ho.Nstates))
                               + 1j * rng.standard_normal((pw.gvecw.Ngw[ik], Ho.Nstates))) for ik in range(pw.kpoints.Nkpt)]
    rho = Ho.guess_rhoe()
    F_ref = {"Ps_loc": forces.calc_forces_Ps_loc(Ho, rho), "Ps_nloc": forces.calc_forces_Ps_nloc(Ho, psiks)}
    sysm = pwb200.System(["Si", "Si"], pos, pw.LatVecs)
    H = pwb200.Hamiltonian(sysm, [_psp()], 15.0, kpts=pw.kpoints.k, wk=pw.kpoints.wk)
    dt = torch.complex128 if prec == "c128" else torch.complex64
    dev = [torch.from_numpy(np.ascontiguousarray(p.T)).cuda().to(dt).contiguous() for p in psiks]
    F, parts = pf.calc_forces(H, dev, torch.from_numpy(rho).cuda(), Ho.Focc, parts=True)
    tol = 1e-10 if prec == "c128" else 1e-6
    for k in ("Ps_loc", "Ps_nloc"):
        assert np.abs(parts[k] - F_ref[k]).max() < tol, (k, np.abs(parts[k] - F_ref[k]).max())
    H.ctx.check_device()


def _psp():
    from oracle import systems
    return systems.psp("Si-q4.gth")


@pytest.mark.gpu
def test_device_forces_match_finite_differences_si64():
    """Config C4: Si64, every atom moved by seeded uniform noise in
    [-0.05, 0.05] bohr, GTH-PBE Si-q4, PBE: forces from the device SCF (FP64)
    against central finite differences (h = 1e-4 bohr) of the device SCF
    energy for one Cartesian component, and the mixed-precision SCF's
    forces against the FP64 ones."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from pwb200 import scf
    from pwb200 import forces as pf
    from oracle import systems
    at = systems.diamond_supercell(2, 10.2631, displace=0.05, seed=7)
    nat = at.positions.shape[1]

    def run(pos, precision="fp64"):
        H = pwb200.Hamiltonian(pwb200.System(["Si"] * nat, pos, at.LatVecs), [systems.psp("Si-q4-pbe.gth")], 15.0,
                               xcfunc="PBE")
        res = scf.KS_solve_SCF(H, Nstates=136, etot_conv_thr=1e-11, ethr_evals_last=1e-11, precision=precision,
                               fp64_switch=1e-5 * nat)
        return H, res

    pos = at.positions.copy()
    H, res = run(pos)
    Focc, _ = scf.occupations(H.Nelectrons, 136, 1)
    F = pf.calc_forces(H, res["psiks"], res["rho"], Focc)
    assert np.abs(F.sum(axis=1)).max() < 1e-4
    h = 1e-4
    Es = []
    for s in (+1, -1):
        p = pos.copy()
        p[0, 5] += s * h
        Es.append(run(p)[1]["energies"]["Total"])
    fd = -(Es[0] - Es[1]) / (2 * h)
    assert abs(fd - F[0, 5]) < 1e-5, (fd, F[0, 5])
    Hm, rm = run(pos, "mixed")
    Fm = pf.calc_forces(Hm, rm["psiks"], rm["rho"], Focc)
    assert np.abs(Fm - F).max() < 1e-5
