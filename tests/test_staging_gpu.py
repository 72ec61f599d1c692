"""The call sequences of the Julia binding (pwdft.jl_b200/julia/PWDFTB200.jl),
replayed through ctypes with host arrays only, against the FP64 oracle.

Julia is not installed in this image, so the binding itself cannot run; this
file drives the C ABI exactly as it does -- 1-based index maps
(index_base = 1), Fortran-ordered host arrays, device buffers through
pw_device_alloc / pw_copy_to_device / pw_copy_to_host -- for the methods it
adds to PWDFT: calc_grad (calc_grad.jl:1-57), the band energies of
calc_E_Ps_nloc (calc_energies.jl:7-58), dE_dVloc (pw_vloc_vjp), and the
local and nonlocal forces (calc_forces_Ps_loc.jl:13-72,
calc_forces_Ps_nloc.jl:291-411).  Si fcc on a 2x2x2 mesh (4 k-points),
fractional occupations.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def setup():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    H = systems.Ham_Si_fcc(meshk=(2, 2, 2), extra_states=2)
    pw = H.pw
    rng = np.random.default_rng(21)
    H.V_Total = H.V_Ps_loc + 0.02 * np.cos(0.013 * np.arange(pw.Npoints))
    nk = pw.kpoints.Nkpt
    # the binding hands over Julia's 1-based idx_gw2r
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, [np.asarray(i) + 1 for i in pw.gvecw.idx_gw2r],
                         [pw.Gk2(k) for k in range(nk)], index_base=1)
    ctx.set_vloc(H.V_Total)
    for ik in range(nk):
        ctx.set_nonlocal(ik, H.betaNL[ik])
    ctx.set_nonlocal_coef(H.nl_triplets)
    nb = H.Nstates
    psiks = []
    for ik in range(nk):
        q, _ = np.linalg.qr(rng.standard_normal((pw.gvecw.Ngw[ik], nb)) + 1j * rng.standard_normal((pw.gvecw.Ngw[ik], nb)))
        psiks.append(np.asfortranarray(q))
    Focc = np.tile(np.linspace(2.0, 0.3, nb)[:, None], (1, nk))
    H.Focc = Focc
    yield H, ctx, psiks, Focc
    ctx.close()


class Staged:
    """DeviceBuffer of the binding: pw_device_alloc + copies."""

    def __init__(self, ctx, a):
        self.ctx, self.L = ctx, ctx._L
        self.bytes = a.nbytes
        p = C.c_void_p()
        ctx._chk(self.L.pw_device_alloc(ctx.h, self.bytes, C.byref(p)))
        self.ptr = p
        ctx._chk(self.L.pw_copy_to_device(ctx.h, p, a.ctypes.data_as(C.c_void_p), self.bytes))

    def to_host(self, out):
        self.ctx._chk(self.L.pw_copy_to_host(self.ctx.h, out.ctypes.data_as(C.c_void_p), self.ptr, out.nbytes))
        return out

    def free(self):
        self.ctx._chk(self.L.pw_device_free(self.ctx.h, self.ptr))


def test_calc_grad_through_staging(setup):
    from oracle import ops
    H, ctx, psiks, Focc = setup
    wk = H.pw.kpoints.wk
    for ik in (0, len(psiks) - 1):
        psi = psiks[ik]
        p = Staged(ctx, psi)
        g = Staged(ctx, np.zeros_like(psi))
        f = np.ascontiguousarray(Focc[:, ik])
        ctx._chk(ctx._L.pw_calc_grad(ctx.h, ik, 0, 0, p.ptr, g.ptr, psi.shape[0], psi.shape[1],
                                     f.ctypes.data_as(_dp), float(wk[ik])))
        got = g.to_host(np.zeros_like(psi))
        ref = ops.calc_grad(H, psi, ik, Focc[:, ik], wk[ik])
        assert np.abs(got - ref).max() < 1e-11 * np.abs(ref).max()
        p.free()
        g.free()


def test_band_energies_and_dE_dVloc_through_staging(setup):
    from oracle import energies, ops
    H, ctx, psiks, Focc = setup
    pw = H.pw
    wk = pw.kpoints.wk
    E = np.zeros(2)
    dV = Staged(ctx, np.zeros(pw.Npoints))
    for ik, psi in enumerate(psiks):
        p = Staged(ctx, psi)
        w = np.ascontiguousarray(wk[ik] * Focc[:, ik])
        E2 = np.zeros(2)
        ctx._chk(ctx._L.pw_band_energies(ctx.h, ik, 0, p.ptr, psi.shape[0], psi.shape[1], w.ctypes.data_as(_dp),
                                         E2.ctypes.data_as(_dp)))
        E += E2
        ctx._chk(ctx._L.pw_vloc_vjp(ctx.h, ik, 0, p.ptr, None, psi.shape[0], psi.shape[1], w.ctypes.data_as(_dp),
                                    dV.ptr, int(ik > 0)))
        p.free()
    assert abs(E[0] - energies.calc_E_kin(H, psiks)) < 1e-11
    assert abs(E[1] - energies.calc_E_Ps_nloc(H, psiks)) < 1e-11
    got = dV.to_host(np.zeros(pw.Npoints))
    ref = ops.calc_rhoe(H, psiks, Focc=Focc) * pw.CellVolume / pw.Npoints
    assert np.abs(got - ref).max() < 1e-11 * np.abs(ref).max()
    dV.free()


def test_forces_through_staging(setup):
    from oracle import forces, ops
    H, ctx, psiks, Focc = setup
    pw = H.pw
    gv = pw.gvec
    # PWDFTB200.setup_forces!: 1-based density sphere, V_sp(G), G+k, atom of each projector
    idx = np.ascontiguousarray(np.asarray(gv.idx_g2r, dtype=np.int64) + 1)
    G2 = np.ascontiguousarray(gv.G2)
    ctx._chk(ctx._L.pw_set_density_sphere(ctx.h, len(idx), idx.ctypes.data_as(C.POINTER(C.c_int64)),
                                          G2.ctypes.data_as(_dp), 1))
    from oracle.gth import eval_Vloc_G
    VlocG = np.stack([eval_Vloc_G(psp, gv.G2) for psp in H.pspots], axis=1)
    ctx.set_force_tables(VlocG, gv.G.T)
    for ik in range(pw.kpoints.Nkpt):
        ctx.set_gkvec(ik, (gv.G[:, pw.gvecw.idx_gw2g[ik]] + pw.kpoints.k[:, ik][:, None]).T)
    ctx.set_nonlocal_atoms(H.atoms.Natoms, forces.beta_atom(H))
    rho = ops.calc_rhoe(H, psiks, Focc=Focc)
    r = Staged(ctx, rho)
    pos = np.asfortranarray(H.atoms.positions)
    sp = np.ascontiguousarray(np.asarray(H.atoms.atm2species, dtype=np.int32))
    F = np.zeros((3, H.atoms.Natoms), order="F")
    ctx._chk(ctx._L.pw_forces_local(ctx.h, r.ptr, H.atoms.Natoms, pos.ctypes.data_as(_dp),
                                    sp.ctypes.data_as(C.POINTER(C.c_int32)), F.ctypes.data_as(_dp)))
    Fref = forces.calc_forces_Ps_loc(H, rho)
    assert np.abs(F - Fref).max() < 1e-10 * max(1.0, np.abs(Fref).max())
    Fnl = np.zeros((3, H.atoms.Natoms), order="F")
    for ik, psi in enumerate(psiks):
        p = Staged(ctx, psi)
        w = np.ascontiguousarray(pw.kpoints.wk[ik] * Focc[:, ik])
        Fk = np.zeros((3, H.atoms.Natoms), order="F")
        ctx._chk(ctx._L.pw_forces_nonlocal(ctx.h, ik, 0, p.ptr, psi.shape[0], psi.shape[1], w.ctypes.data_as(_dp),
                                           Fk.ctypes.data_as(_dp)))
        Fnl += Fk
        p.free()
    Fnl_ref = forces.calc_forces_Ps_nloc(H, psiks)
    assert np.abs(Fnl - Fnl_ref).max() < 1e-10 * max(1.0, np.abs(Fnl_ref).max())
    r.free()


def test_device_free_rejects_foreign_pointer(setup):
    import pwb200
    H, ctx, psiks, Focc = setup
    with pytest.raises(pwb200.PWError) as e:
        ctx._chk(ctx._L.pw_device_free(ctx.h, C.c_void_p(0x1000)))
    assert e.value.status == pwb200._lib.PW_ERR_ARG
