"""Host logic of the autograd wrappers (pwb200.adjoint), on CPU: the library
calls are replaced by the oracle (a stand-in context whose vloc_vjp is the
oracle's density times dVol, and a stand-in force routine), so that what is
tested is the wrappers' bookkeeping: the value, the gradient's routing and
sign, and the chain rule through a downstream loss."""
import numpy as np
import torch

from oracle import systems, ops


class OracleCtx:
    def __init__(self, H):
        self.H = H
        self.N = H.pw.Npoints

    def vloc_vjp(self, ik, psi, w, dV, lam=None, accumulate=False):
        from oracle.ham import G_to_R
        pw = self.H.pw
        p = psi.numpy().T
        l = p if lam is None else lam.numpy().T

        def rs(a):
            ct = np.zeros((a.shape[1], pw.Npoints), dtype=np.complex128)
            ct[:, pw.gvecw.idx_gw2r[ik]] = a.T
            return G_to_R(pw.Ns, ct)
        g = pw.Npoints * (np.asarray(w)[:, None] * np.real(np.conj(rs(l)) * rs(p))).sum(axis=0)
        dV.copy_(torch.from_numpy(g) + (dV if accumulate else 0))


def test_local_band_energy_value_and_gradient():
    from pwb200 import adjoint
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1))
    pw = H.pw
    rng = np.random.default_rng(3)
    ngw = pw.gvecw.Ngw[0]
    psi = (rng.standard_normal((ngw, 4)) + 1j * rng.standard_normal((ngw, 4))) / np.sqrt(ngw)
    w = np.array([2.0, 2.0, 1.0, 0.5])
    V = torch.from_numpy(H.V_Ps_loc.copy()).requires_grad_(True)
    x = torch.from_numpy(np.ascontiguousarray(psi.T))
    E = adjoint.local_band_energy(OracleCtx(H), 0, V, x, w)
    # the value: sum_b w_b <psi_b|V psi_b> from the oracle's op_V_loc
    Vpsi = np.zeros_like(psi)
    H.V_Total = H.V_Ps_loc.copy()
    ops.op_V_loc(H, psi, Vpsi, 0)
    ref = float(np.real(np.einsum("gb,gb,b->", psi.conj(), Vpsi, w)))
    assert abs(float(E.detach()) - ref) < 1e-10 * abs(ref)
    # chain rule through a downstream loss: d(E^2)/dV = 2E rho dVol
    (E * E).backward()
    rho = ops.calc_rhoe(H, [psi], Focc=w[:, None]) * pw.CellVolume / pw.Npoints
    e0 = float(E.detach())
    assert np.abs(V.grad.numpy() - 2 * e0 * rho).max() < 1e-10 * np.abs(2 * e0 * rho).max()


def test_ionic_energy_gradient_is_minus_force(monkeypatch):
    from pwb200 import adjoint, forces
    F = np.array([[0.1, -0.2], [0.3, 0.0], [-0.05, 0.07]])
    monkeypatch.setattr(forces, "calc_forces", lambda Ham, psiks, rho, Focc: F)
    pos = torch.zeros((3, 2), dtype=torch.float64, requires_grad=True)
    E = adjoint.ionic_energy(None, pos, -7.9, None, None, None)
    assert float(E) == -7.9
    (3.0 * E).backward()
    assert np.allclose(pos.grad.numpy(), -3.0 * F)
