"""The benchmark systems, built the way the reference's scripts build them.

Oracle (test infrastructure only).

  Si2 fcc   test/validations_old/Si_fcc.jl:1-12 (a = 10.2631 bohr, 3x3x3 MP)
  Si64      2x2x2 conventional diamond cells, a = 20.5262 bohr, Gamma
  Si216     3x3x3 conventional diamond cells, a = 30.7893 bohr, Gamma
  Al4       conventional fcc cell, a = 7.6524 bohr
  Pt fcc    test/validations_old/Pt_fcc.jl:1-12 (a = 3.9231 angstrom, ecutwfc 30, 3x3x3 MP,
            4 extra states)

The pseudopotential files are shipped under tests/golden/psp (copied from the
reference's pseudopotentials/ folder: they are data, read by both the oracle
and the product's set-up code).
"""
import os
import numpy as np

from .pwgrid import gen_lattice_fcc, gen_lattice_cubic
from .ham import Atoms, Hamiltonian

PSP_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "tests", "golden", "psp")

DIAMOND_BASIS = np.array([
    [0.00, 0.00, 0.00], [0.00, 0.50, 0.50], [0.50, 0.00, 0.50], [0.50, 0.50, 0.00],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25]])


def psp(name):
    return os.path.join(PSP_DIR, name)


def si_fcc_atoms():
    LL = gen_lattice_fcc(10.2631)
    return Atoms.from_frac(["Si", "Si"], np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]]).T, LL)


def diamond_supercell(n, a_conv, displace=0.0, seed=0):
    """n x n x n conventional diamond cells (8 atoms each), cubic a = n*a_conv.
    Optional seeded uniform displacement in [-displace, displace] bohr."""
    frac = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                for b in DIAMOND_BASIS:
                    frac.append((b + np.array([i, j, k])) / n)
    frac = np.array(frac).T
    LL = gen_lattice_cubic(n * a_conv)
    atoms = Atoms.from_frac(["Si"] * frac.shape[1], frac, LL)
    if displace > 0:
        rng = np.random.default_rng(seed)
        atoms.positions = atoms.positions + rng.uniform(-displace, displace, atoms.positions.shape)
    return atoms


ANG2BOHR = 1.8897261254578281


def pt_fcc_atoms():
    LL = gen_lattice_fcc(3.9231 * ANG2BOHR)
    return Atoms.from_frac(["Pt"], np.zeros((3, 1)), LL)


def Ham_Pt_fcc(meshk=(3, 3, 3)):
    return Hamiltonian(pt_fcc_atoms(), [psp("Pt-q10.gth")], 30.0, meshk=meshk, extra_states=4)


def al4_atoms():
    """Conventional fcc Al cell, a = 7.6524 bohr, 4 atoms."""
    frac = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]]).T
    return Atoms.from_frac(["Al"] * 4, frac, gen_lattice_cubic(7.6524))


def Ham_Al4(meshk=(8, 8, 8), Nstates=10):
    return Hamiltonian(al4_atoms(), [psp("Al-q3.gth")], 15.0, meshk=meshk, Nstates=Nstates)


def Ham_Si_fcc(meshk=(3, 3, 3), extra_states=None):
    return Hamiltonian(si_fcc_atoms(), [psp("Si-q4.gth")], 15.0, meshk=meshk,
                       extra_states=extra_states)


def Ham_Si64(Nstates=160):
    return Hamiltonian(diamond_supercell(2, 10.2631), [psp("Si-q4.gth")], 15.0, Nstates=Nstates)
