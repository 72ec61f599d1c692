"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point include/pwb200.h declares, and its host-side basis builders
reproduce the reference's index maps bit for bit (PWGrid.jl:199-322, as
restated by the oracle)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import pwb200
from pwb200 import _lib
from oracle import pwgrid, systems

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pwb200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pw_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    L = pwb200.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, "binding missing for " + n


def test_abi_version():
    assert pwb200.lib().pw_abi_version() == 1


def test_good_fft_order_matches_oracle():
    L = pwb200.lib()
    for n in range(1, 400):
        assert L.pw_good_fft_order(n) == pwgrid.good_fft_order(n)


@pytest.mark.parametrize("case", ["si_fcc", "si64", "al_kpt"])
def test_gvec_maps_bit_exact(case):
    if case == "si_fcc":
        LL = pwgrid.gen_lattice_fcc(10.2631)
        kp = pwgrid.gen_kpoint_grid(LL, (3, 3, 3))
    elif case == "si64":
        LL = pwgrid.gen_lattice_cubic(2 * 10.2631)
        kp = None
    else:
        LL = pwgrid.gen_lattice_cubic(7.6524)
        kp = pwgrid.gen_kpoint_grid(LL, (4, 4, 4))
    ref = pwgrid.PWGrid(15.0, LL, kpoints=kp)
    kpts = ref.kpoints.k
    b = pwb200.Basis(LL, 15.0, kpts=kpts)
    assert b.Ns == ref.Ns and b.Ng == ref.gvec.Ng
    assert np.array_equal(b.idx_g2r, ref.gvec.idx_g2r)
    assert np.array_equal(b.G2, ref.gvec.G2)             # bitwise
    assert np.array_equal(b.G, ref.gvec.G.T)
    for ik in range(ref.kpoints.Nkpt):
        assert np.array_equal(b.idx_gw2g[ik], ref.gvecw.idx_gw2g[ik])
        assert np.array_equal(b.idx_gw2r[ik], ref.gvecw.idx_gw2r[ik])
        assert np.array_equal(b.Gk2[ik], ref.Gk2(ik))


def test_create_without_device_fails_cleanly():
    """pw_create reports an error status (never crashes) when it cannot run."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    L = pwb200.lib()
    d = _lib.pw_grid_desc()
    h = C.c_void_p()
    st = L.pw_create(0, C.byref(d), C.byref(h))
    assert st != 0 and not h.value
    assert len(L.pw_last_error(None)) > 0


def test_product_setup_matches_oracle():
    """The device path's host set-up (V_Ps_loc, betaNL, h_ij) equals the
    oracle's restatement of Hamiltonian.jl / PsPotNL.jl."""
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    sysm = pwb200.System(["Si", "Si"], H.atoms.positions, H.atoms.LatVecs)
    b = pwb200.Basis(H.atoms.LatVecs, 15.0)
    from pwb200.system import local_potential, projectors, GTH
    psp = [GTH(systems.psp("Si-q4.gth"))]
    V = local_potential(sysm, b, psp)
    assert np.allclose(V, H.V_Ps_loc, rtol=0, atol=1e-12 * np.abs(H.V_Ps_loc).max())
    beta, trip = projectors(sysm, b, psp, 0)
    assert beta.shape == H.betaNL[0].shape
    assert np.allclose(beta, H.betaNL[0], rtol=0, atol=1e-13 * np.abs(H.betaNL[0]).max())
    assert [(i, j) for i, j, _ in trip] == [(i, j) for i, j, _ in H.nl_triplets]
    assert np.allclose([h for *_, h in trip], [h for *_, h in H.nl_triplets])
