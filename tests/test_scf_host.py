"""The SCF driver's host-side set-up (k-point grid, starting density, Ewald
energy, occupations) against the oracle's restatement of the reference."""
import numpy as np

import pwb200
from pwb200.system import kpoint_grid, guess_rhoe, ewald_energy, System, GTH, Basis
from pwb200.scf import occupations
from oracle import systems, pwgrid, energies


def test_kpoint_grid_matches_reference_reduction():
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    for mesh in [(3, 3, 3), (2, 2, 2), (4, 4, 4)]:
        ref = pwgrid.gen_kpoint_grid(H.atoms.LatVecs, mesh)
        k, w = kpoint_grid(H.atoms.LatVecs, mesh)
        assert k.shape == ref.k.shape
        assert np.allclose(k, ref.k, atol=1e-14) and np.allclose(w, ref.wk, atol=1e-15)


def test_guess_rhoe_and_ewald():
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    sysm = System(["Si", "Si"], H.atoms.positions, H.atoms.LatVecs)
    b = Basis(H.atoms.LatVecs, 15.0)
    rho = guess_rhoe(sysm, b, [GTH(systems.psp("Si-q4.gth"))], 8.0)
    assert np.allclose(rho, H.guess_rhoe(), atol=1e-12)
    e = ewald_energy(H.atoms.LatVecs, H.atoms.positions, np.array([4.0, 4.0]))
    assert abs(e - (-8.397927400714764)) < 1e-10


def test_occupations():
    F, nocc = occupations(8.0, 8, 3)
    assert nocc == 4 and np.all(F[:4] == 2.0) and np.all(F[4:] == 0.0)
    F, nocc = occupations(7.0, 5, 1)
    assert nocc == 4 and F[3, 0] == 1.0
