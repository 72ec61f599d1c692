"""PBE exchange-correlation with the reference's internal formulas.

Oracle (test infrastructure only).  Restates PWDFT.jl (Nspin = 1):
  XC_funcs/XC_x_pbe.jl:3-49     XC_x_pbe   (PBE exchange enhancement, no Slater part)
  XC_funcs/XC_c_pw.jl:1-31      XC_c_pw    (Perdew-Wang 92 correlation)
  XC_funcs/XC_c_pbe.jl:3-53     XC_c_pbe   (PBE gradient correction to PW92)
  GGA_PBE_internal.jl:29-53     calc_epsxc_PBE!
  GGA_PBE_internal.jl:98-145    calc_Vxc_PBE!
  PWGrid.jl:351-375             op_nabla
  PWGrid.jl:378-398             op_nabla_dot
All functions are vectorised over grid points; the thresholds (rho <= 1e-6
or |grad rho|^2 <= 1e-10 zero the gradient terms, rho <= 1e-10 the local
ones) are the reference's.
"""
import numpy as np

from .ham import G_to_R, R_to_G, xc_x_slater


def xc_x_pbe(rho, grho):
    """XC_x_pbe.jl:3-49: (sx, v1x, v2x)."""
    rho = np.asarray(rho, dtype=np.float64)
    grho = np.asarray(grho, dtype=np.float64)
    ok = (rho > 1e-6) & (grho > 1e-10)
    r = np.where(ok, rho, 1.0)
    g = np.where(ok, grho, 1.0)
    third = 1.0 / 3.0
    k, mu = 0.804, 0.2195149727645171
    c1, c2, c5 = 0.75 / np.pi, 3.093667726280136, 4.0 * third
    agrho = np.sqrt(g)
    kf = c2 * np.cbrt(r)
    dsg = 0.5 / kf
    s1 = agrho * dsg / r
    s2 = s1 * s1
    ds = -c5 * s1
    f1 = s2 * mu / k
    f2 = 1.0 + f1
    f3 = k / f2
    fx = k - f3
    exunif = -c1 * kf
    sx_s = exunif * fx
    dxunif = exunif * third
    dfx = 2.0 * mu * s1 / (f2 * f2)
    v1x = sx_s + dxunif * fx + exunif * dfx * ds
    v2x = exunif * dfx * dsg / agrho
    sx = sx_s * r
    z = np.zeros_like(rho)
    return np.where(ok, sx, z), np.where(ok, v1x, z), np.where(ok, v2x, z)


def xc_c_pw(rho):
    """XC_c_pw.jl:1-31: (ec, vc)."""
    rho = np.asarray(rho, dtype=np.float64)
    ok = rho > 1e-10
    r = np.where(ok, rho, 1.0)
    pi34 = 0.6203504908994
    rs = pi34 / np.cbrt(r)
    a, a1, b1, b2, b3, b4 = 0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294
    rs12 = np.sqrt(rs)
    rs32 = rs * rs12
    rs2 = rs * rs
    om = 2.0 * a * (b1 * rs12 + b2 * rs + b3 * rs32 + b4 * rs2)
    dom = 2.0 * a * (0.5 * b1 * rs12 + b2 * rs + 1.5 * b3 * rs32 + 2.0 * b4 * rs2)
    olog = np.log(1.0 + 1.0 / om)
    ec = -2.0 * a * (1.0 + a1 * rs) * olog
    vc = -2.0 * a * (1.0 + 2.0 / 3.0 * a1 * rs) * olog - 2.0 / 3.0 * a * (1.0 + a1 * rs) * dom / (om * (om + 1.0))
    z = np.zeros_like(rho)
    return np.where(ok, ec, z), np.where(ok, vc, z)


def xc_c_pbe(rho, grho):
    """XC_c_pbe.jl:3-53: (sc, v1c, v2c)."""
    rho = np.asarray(rho, dtype=np.float64)
    grho = np.asarray(grho, dtype=np.float64)
    ok = (rho > 1e-6) & (grho > 1e-10)
    r = np.where(ok, rho, 1.0)
    g = np.where(ok, grho, 1.0)
    ga, be = 0.0310906908696548950, 0.06672455060314922
    pi34, xkf, xks = 0.6203504908994, 1.919158292677513, 1.128379167095513
    rs = pi34 / np.cbrt(r)
    ec, vc = xc_c_pw(r)
    kf = xkf / rs
    ks = xks * np.sqrt(kf)
    t = np.sqrt(g) / (2.0 * ks * r)
    expe = np.exp(-ec / ga)
    af = be / ga * (1.0 / (expe - 1.0))
    bf = expe * (vc - ec)
    y = af * t * t
    xy = (1.0 + y) / (1.0 + y + y * y)
    qy = y * y * (2.0 + y) / (1.0 + y + y * y) ** 2
    s1 = 1.0 + be / ga * t * t * xy
    h0 = ga * np.log(s1)
    dh0 = be * t * t / s1 * (-7.0 / 3.0 * xy - qy * (af * bf / be - 7.0 / 3.0))
    ddh0 = be / (2.0 * ks * ks * r) * (xy - qy) / s1
    z = np.zeros_like(rho)
    return np.where(ok, r * h0, z), np.where(ok, h0 + dh0, z), np.where(ok, ddh0, z)


def op_nabla(pw, rho):
    """PWGrid.jl:351-375: grad rho (3, N) from the density-sphere components."""
    g = pw.gvec
    rhoG = R_to_G(pw.Ns, rho.astype(np.complex128))[g.idx_g2r]
    out = np.zeros((3, pw.Npoints))
    for d in range(3):
        full = np.zeros(pw.Npoints, dtype=np.complex128)
        full[g.idx_g2r] = 1j * g.G[d] * rhoG
        out[d] = np.real(G_to_R(pw.Ns, full))
    return out


def op_nabla_dot(pw, h):
    """PWGrid.jl:378-398: div h (N) over the density sphere, h (3, N) real."""
    g = pw.gvec
    div = np.zeros(g.Ng, dtype=np.complex128)
    for d in range(3):
        div += g.G[d] * R_to_G(pw.Ns, h[d].astype(np.complex128))[g.idx_g2r]
    full = np.zeros(pw.Npoints, dtype=np.complex128)
    full[g.idx_g2r] = 1j * div
    return np.real(G_to_R(pw.Ns, full))


def calc_epsxc_PBE(pw, rho):
    """GGA_PBE_internal.jl:29-53."""
    gr = op_nabla(pw, rho)
    g2 = (gr * gr).sum(axis=0)
    ex = xc_x_slater(rho)[0]
    ec = xc_c_pw(rho)[0]
    sx = xc_x_pbe(rho, g2)[0]
    sc = xc_c_pbe(rho, g2)[0]
    with np.errstate(divide="ignore", invalid="ignore"):
        grad = np.where(rho != 0.0, (sx + sc) / rho, 0.0)
    return ex + ec + grad


def calc_Vxc_PBE(pw, rho):
    """GGA_PBE_internal.jl:98-145."""
    gr = op_nabla(pw, rho)
    g2 = (gr * gr).sum(axis=0)
    vx = xc_x_slater(rho)[1]
    vc = xc_c_pw(rho)[1]
    _, v1x, v2x = xc_x_pbe(rho, g2)
    _, v1c, v2c = xc_c_pbe(rho, g2)
    V = vx + vc + v1x + v1c
    h = (v2x + v2c)[None, :] * gr
    return V - op_nabla_dot(pw, h)
