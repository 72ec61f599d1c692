"""Generates al4_smearing_444.json: the oracle's converged SCF for the Al4
conventional fcc cell (a = 7.6524 bohr, GTH Al-q3, LDA-VWN, ecutwfc 15 Ha,
4x4x4 mesh reduced by the crystal's symmetry, 10 states, Fermi-Dirac
kT = 0.01 Ha, Pulay mixing beta 0.2, etot_conv_thr 1e-9): config C3's
system on a smaller mesh, for the device SCF's parity test.

    python tests/golden/make_al4_smearing.py     (about a minute, CPU)
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ham, scf, systems  # noqa: E402


def main():
    H = ham.Hamiltonian(systems.al4_atoms(), [systems.psp("Al-q3.gth")], 15.0, meshk=(4, 4, 4), Nstates=10,
                        use_symmetry=True)
    E, _, _ = scf.KS_solve_SCF(H, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-9, use_smearing=True, kT=0.01)
    out = {"system": "Al4 fcc conventional, a=7.6524, Al-q3, LDA-VWN, ecutwfc 15, 4x4x4 with symmetry, 10 states, "
                     "Fermi-Dirac kT 0.01, Pulay 0.2, etot_conv_thr 1e-9",
           "Nkpt": int(H.pw.kpoints.Nkpt), "Nsyms": int(H.sym.Nsyms), "wk": [float(w) for w in H.pw.kpoints.wk],
           "E_fermi": float(H.E_fermi), "energies": {k: float(v) for k, v in E.items()}}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "al4_smearing_444.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
