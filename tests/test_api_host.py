"""Host logic of the reference-named eigensolver wrappers of pwb200
(diag_LOBPCG!, diag_davidson_qe!, diag_CheFSI!, chebyfilt,
get_ub_lb_lanczos, ortho_sqrt!) against a recording stand-in for the device
context: k-point loop, Ham.ik bookkeeping, argument order and the
(Nstates, Nkpt) eigenvalue layout.  No device code runs here; the device
paths have their own parity tests (test_lobpcg_gpu, test_chefsi_gpu)."""
import numpy as np
import pytest


class FakeCtx:
    def __init__(self, Ngw):
        self.Ngw = Ngw
        self.device = 0
        self.calls = []

    def lobpcg(self, ik, ispin, X, tol, nitermax, nconv):
        self.calls.append(("lobpcg", ik, ispin, tol, nitermax, nconv))
        return np.arange(X.shape[0]) + 10.0 * ik, 3

    def davidson(self, ik, ispin, X, tol, nitermax):
        self.calls.append(("davidson", ik, ispin, tol, nitermax))
        return np.arange(X.shape[0]) - 1.0 * ik, 2

    def chebyfilt(self, ik, ispin, X, Y, degree, lb, ub):
        self.calls.append(("chebyfilt", ik, ispin, degree, lb, ub))
        Y.copy_(X)

    def lanczos_bounds(self, ik, ispin, nlancz, v0):
        self.calls.append(("lanczos", ik, ispin, nlancz, tuple(v0.shape)))
        return 5.0, -1.0


class FakeHam:
    def __init__(self, ctx):
        self.ctx = ctx
        self.ik = 0
        self.ispin = 0


def blocks(nb, ngws):
    import torch
    return [torch.zeros((nb, n), dtype=torch.complex128) for n in ngws]


def test_diag_wrappers_loop_over_kpoints():
    import pwb200
    ctx = FakeCtx([30, 40, 50])
    H = FakeHam(ctx)
    ps = blocks(4, ctx.Ngw)
    ev = pwb200.diag_LOBPCG_(H, ps, tol=1e-7, NiterMax=50, Nstates_conv=3)
    assert ev.shape == (4, 3) and np.allclose(ev[:, 2], np.arange(4) + 20.0)
    assert [c[1] for c in ctx.calls] == [0, 1, 2] and ctx.calls[0][3:] == (1e-7, 50, 3)
    assert H.ik == 2
    ctx.calls.clear()
    ev = pwb200.diag_davidson_qe_(H, ps, tol=1e-6, NiterMax=20)
    assert ev.shape == (4, 3) and np.allclose(ev[:, 1], np.arange(4) - 1.0)
    assert all(c[0] == "davidson" and c[3:] == (1e-6, 20) for c in ctx.calls)


def test_chefsi_wrapper_order_and_bounds():
    """diag_CheFSI! per k-point: Lanczos with nlancz = 2 Nstates first, then
    the filter of cheby_degree over [lb, ub] in the reference's order
    (get_ub_lb_lanczos returns (ub, lb))."""
    import pwb200
    from pwb200 import chefsi

    class Ctx2(FakeCtx):
        def ortho_sqrt(self, Y):
            self.calls.append(("ortho",))

        def apply(self, ik, ispin, psi, Hpsi):
            self.calls.append(("apply", ik))

        def gram(self, A, B, out):
            self.calls.append(("gram",))

        def eigh(self, T, G=None, k=None, vectors=True):
            import torch
            self.calls.append(("eigh", k, vectors))
            return torch.arange(k, dtype=torch.float64), None

    ctx = Ctx2([20, 24])
    H = FakeHam(ctx)
    ps = blocks(3, ctx.Ngw)
    ev = pwb200.diag_CheFSI_(H, ps, 8, seed=3)
    assert ev.shape == (3, 2)
    names = [c[0] for c in ctx.calls]
    assert names == ["lanczos", "chebyfilt", "ortho", "apply", "gram", "eigh"] * 2
    lz = [c for c in ctx.calls if c[0] == "lanczos"]
    assert lz[0][1:] == (0, 0, 6, (20,)) and lz[1][1:] == (1, 0, 6, (24,))
    cf = [c for c in ctx.calls if c[0] == "chebyfilt"]
    assert cf[0][3:] == (8, -1.0, 5.0)
    assert [c for c in ctx.calls if c[0] == "eigh"][0][1:] == (3, False)
    # the same generator draws give the same start vectors
    r1, r2 = np.random.default_rng(3), np.random.default_rng(3)
    assert np.array_equal(r1.standard_normal(5), r2.standard_normal(5))
    assert chefsi.diag_chefsi_k.__doc__


def test_lanczos_and_filter_wrappers():
    import torch
    import pwb200
    ctx = FakeCtx([16])
    H = FakeHam(ctx)
    X = torch.ones((2, 16), dtype=torch.complex128)
    Y = pwb200.chebyfilt(H, X, 4, 0.5, 9.0)
    assert torch.equal(Y, X) and ctx.calls[-1] == ("chebyfilt", 0, 0, 4, 0.5, 9.0)
    v0 = torch.ones(16, dtype=torch.complex128)
    assert pwb200.get_ub_lb_lanczos(H, 8, v0=v0) == (5.0, -1.0)
    assert ctx.calls[-1] == ("lanczos", 0, 0, 8, (16,))


def test_driver_aliases_forward_arguments(monkeypatch):
    import pwb200
    from pwb200 import scf, emin_scf
    seen = {}
    monkeypatch.setattr(scf, "KS_solve_SCF", lambda Ham, **kw: seen.setdefault("scf", (Ham, kw)))
    monkeypatch.setattr(emin_scf, "KS_solve_Emin_PCG", lambda Ham, psiks, **kw: seen.setdefault("emin", (Ham, psiks, kw)))
    pwb200.KS_solve_SCF_("H", update_psi="PCG", etot_conv_thr=1e-7, print_final_ebands=True)
    pwb200.KS_solve_Emin_PCG_("H", None, i_cg_beta=3, **{"\u03b1_t": 1e-5, "\u03b1_max": 1.5})
    assert seen["scf"] == ("H", {"update_psi": "PCG", "etot_conv_thr": 1e-7})
    assert seen["emin"] == ("H", None, {"i_cg_beta": 3, "alpha_t": 1e-5, "alpha_max": 1.5})
    from pwb200 import emin_pcg
    import numpy as np

    def fake_k(ctx, ik, ispin, X, **kw):
        seen.setdefault("pcg", []).append((ik, kw["alpha_t"], kw["I_CG_BETA"]))
        return np.zeros(X.shape[0]), 1
    monkeypatch.setattr(emin_pcg, "diag_Emin_PCG_k", fake_k)

    class H:
        ctx, ispin, ik = None, 0, 0
    pwb200.diag_Emin_PCG_(H, [np.zeros((2, 4)), np.zeros((2, 4))], verbose_last=True, I_CG_BETA=3,
                          **{"\u03b1_t": 2e-5})
    assert seen["pcg"] == [(0, 2e-5, 3), (1, 2e-5, 3)]
    with pytest.raises(TypeError):
        pwb200.diag_Emin_PCG_(H, [np.zeros((2, 4))], alpha_typo=1.0)
