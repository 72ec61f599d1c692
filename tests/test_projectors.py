"""betaNL built on the device (pw_build_nonlocal: PsPotNL.jl:16-77 with
eval_proj_G and Ylm_real) against the host construction and the oracle,
through op_V_Ps_nloc on the same wavefunctions: FP64 1e-12 relative.
Cases: Si fcc 2x2x2 k-points (s, p projectors, k != 0), Pt fcc (d
projectors), the displaced Si64 cell of the force tests (64 atoms)."""
import numpy as np
import pytest

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


def _system(name):
    import pwb200
    from pwb200.system import kpoint_grid
    from oracle import systems
    if name == "si":
        at, psp, ec, mesh = systems.si_fcc_atoms(), "Si-q4.gth", 15.0, (2, 2, 2)
    elif name == "pt":
        at, psp, ec, mesh = systems.pt_fcc_atoms(), "Pt-q10.gth", 30.0, (2, 2, 2)
    else:
        at, psp, ec, mesh = systems.diamond_supercell(2, 10.2631, displace=0.05, seed=7), "Si-q4.gth", 15.0, None
    syms = [at.SpeciesSymbols[i] for i in at.atm2species]
    kw = {}
    if mesh:
        k, w = kpoint_grid(at.LatVecs, mesh)
        kw = dict(kpts=k, wk=w)
    mk = lambda dev: pwb200.Hamiltonian(pwb200.System(syms, at.positions, at.LatVecs), [systems.psp(psp)], ec,
                                        device_projectors=dev, **kw)
    return mk(False), mk(True)


@pytest.mark.parametrize("name", ["si", "pt", "si64"])
def test_device_projectors_match_host(name):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    Hh, Hd = _system(name)
    assert Hh.NbetaNL == Hd.NbetaNL > 0 and Hh.nl_triplets == Hd.nl_triplets
    rng = np.random.default_rng(3)
    for ik in range(Hh.basis.Nkpt):
        ngw = Hh.basis.Ngw[ik]
        x = torch.from_numpy(rng.standard_normal((6, ngw)) + 1j * rng.standard_normal((6, ngw))).cuda()
        a, b = torch.empty_like(x), torch.empty_like(x)
        Hh.ctx.apply(ik, 0, x, a, pwb200.PW_OP_VNL)
        Hd.ctx.apply(ik, 0, x, b, pwb200.PW_OP_VNL)
        err = (a - b).abs().max().item() / a.abs().max().item()
        assert err < 1e-12, (ik, err)
        x32 = x.to(torch.complex64)
        a32, b32 = torch.empty_like(x32), torch.empty_like(x32)
        Hh.ctx.apply(ik, 0, x32, a32, pwb200.PW_OP_VNL)
        Hd.ctx.apply(ik, 0, x32, b32, pwb200.PW_OP_VNL)
        assert (a32 - b32).abs().max().item() < 1e-5 * a32.abs().max().item()
    for H in (Hh, Hd):
        H.ctx.check_device()
        H.ctx.close()
