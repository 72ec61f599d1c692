"""Config C3's system (Al4 conventional fcc cell, GTH Al-q3, LDA-VWN,
Fermi-Dirac kT = 0.01 Ha) on a 4x4x4 mesh reduced by symmetry (10 k-points):
the device SCF against the oracle's converged SCF committed in
tests/golden/al4_smearing_444.json (made by tests/golden/make_al4_smearing.py).
The reference has no golden numbers for this system."""
import json
import os

import numpy as np
import pytest

from conftest import cuda_ok

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "al4_smearing_444.json")


def _fixture():
    with open(FIX) as f:
        return json.load(f)


def test_host_kpoints_match_fixture():
    from pwb200 import symmetry as ps
    from oracle import systems
    ref = _fixture()
    at = systems.al4_atoms()
    s, ft = ps.crystal_symmetry(at.LatVecs, at.positions, at.atm2species)
    assert s.shape[2] == ref["Nsyms"]
    k, w = ps.kpoint_grid_sym(at.LatVecs, (4, 4, 4), s)
    assert k.shape[1] == ref["Nkpt"]
    assert np.abs(w - np.array(ref["wk"])).max() < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_al4_smearing_scf_vs_oracle(precision):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from pwb200 import scf
    from oracle import systems
    ref = _fixture()
    at = systems.al4_atoms()
    H = pwb200.Hamiltonian(pwb200.System(["Al"] * 4, at.positions, at.LatVecs), [systems.psp("Al-q3.gth")], 15.0,
                           meshk=(4, 4, 4), use_symmetry=True)
    assert H.basis.Nkpt == ref["Nkpt"]
    res = scf.KS_solve_SCF(H, Nstates=10, betamix=0.2, mix_method="pulay", etot_conv_thr=1e-9, precision=precision,
                           use_smearing=True, kT=0.01, fp64_switch=1e-5 * 4)
    E = res["energies"]
    tol = 1e-7 if precision == "fp64" else 1e-6
    assert abs(E["Total"] - ref["energies"]["Total"]) < tol, (E["Total"], ref["energies"]["Total"], res["log"][-3:])
    assert abs(res["E_fermi"] - ref["E_fermi"]) < 1e-5
    if precision == "fp64":
        for key in ("Kinetic", "Ps_loc", "Ps_nloc", "Hartree", "XC", "mTS"):
            assert abs(E[key] - ref["energies"][key]) < 1e-6, key
    H.ctx.close()
