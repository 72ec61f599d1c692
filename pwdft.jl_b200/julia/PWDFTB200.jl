"""
    PWDFTB200

Julia binding of libpwb200.so, the B200 implementation of PWDFT.jl's
op_H / calc_rhoe / eigensolver hot path.

The drop-in works through Julia's dispatch on the Hamiltonian's type
parameter.  `on_device(Ham)` returns a `Hamiltonian{PsPot_GTH_B200}` -- a
genuine PWDFT `Hamiltonian` sharing every field of `Ham`, whose species
wrap the GTH pseudopotentials together with the device context.  PWDFT's own
drivers (`KS_solve_SCF!`, `KS_solve_Emin_PCG!`, `diag_davidson!`,
`diag_Emin_PCG!`, `diag_CheFSI!`, ...) accept it unchanged, and every call
they make to the methods below -- more specific than PWDFT's
`Ham::Hamiltonian` methods -- runs on the GPU:

    op_H!, op_H, op_K!, op_V_loc!, op_V_Ps_nloc!      (op_H.jl, op_K.jl, op_V_loc.jl, op_V_Ps_nloc.jl)
    calc_rhoe!                                       (calc_rhoe.jl:9-135)
    diag_LOBPCG!, diag_davidson_qe!                  (whole solves on the device)
    calc_grad                                        (calc_grad.jl:1-57)
    update!                                          (PWDFT's update!, then V_loc re-uploaded)
    calc_E_Ps_nloc, op_S!, calc_forces_nlcc!,        (the GTH methods PWDFT types on Hamiltonian{PsPot_GTH})
    calc_forces_scf_corr!
    calc_forces_Ps_loc!, calc_forces_Ps_nloc!        (calc_forces_Ps_loc.jl:13-72, calc_forces_Ps_nloc.jl:291-411)

and the per-species GTH functions (eval_Vloc_G, eval_proj_G, ...) read
through to the wrapped PsPot_GTH.

Differentiation: `dE_dVloc` (pw_vloc_vjp) and ChainRulesCore rrules for
`local_band_energy` (gradient in V_loc) and `ionic_energy` (gradient in the
atomic positions, -F from the device force kernels).

Written against include/pwb200.h.  Julia is not installed in the build
image, so this file is not run by the test suite: the same ABI call
sequences are exercised from Python (pwdft.jl_b200/pwb200 and
tests/test_staging_gpu.py), and tests/test_julia_shim.py checks this text
against PWDFT.jl's declared types, method names and drivers' call sites.
"""
module PWDFTB200

using PWDFT
using LinearAlgebra
using ChainRulesCore

export on_device, B200Hamiltonian, PsPot_GTH_B200, dE_dVloc, local_band_energy, ionic_energy

const libpwb200 = joinpath(@__DIR__, "..", "pwb200", "libpwb200.so")

const PW_C128 = Cint(0)
const PW_C64 = Cint(1)
const PW_OP_K = Cuint(1)
const PW_OP_VLOC = Cuint(2)
const PW_OP_VNL = Cuint(4)
const PW_OP_H = Cuint(7)
const PW_ACCUMULATE = Cuint(0x100)

# struct pw_grid_desc (include/pwb200.h)
struct PwGridDesc
    Ns::NTuple{3,Int32}
    Nkpt::Int32
    Nspin::Int32
    index_base::Int32
    CellVolume::Float64
    Ngw::Ptr{Int64}
    idx_gw2r::Ptr{Ptr{Int64}}
    Gk2::Ptr{Ptr{Float64}}
end

function check(st::Cint, ctx::Ptr{Cvoid})
    st == 0 && return nothing
    msg = unsafe_string(ccall((:pw_last_error, libpwb200), Cstring, (Ptr{Cvoid},), ctx))
    error("libpwb200 status $st: $msg")   # the reference raises in the same places
end

# ------------------------------------------------------------ the device side
"One pw_ctx (one basis on one GPU) shared by the species of a Hamiltonian."
mutable struct DeviceContext
    ctx::Ptr{Cvoid}
    dtype::Cint
    forces_ready::Bool
end

"""
    PsPot_GTH_B200

A GTH pseudopotential (every field of `psp` reads through) carrying the
device context of the Hamiltonian it belongs to.  As the type parameter of
`Hamiltonian` it selects this package's GPU methods.
"""
struct PsPot_GTH_B200 <: PWDFT.AbstractPsPot
    psp::PsPot_GTH
    dev::DeviceContext
end
function Base.getproperty(p::PsPot_GTH_B200, s::Symbol)
    (s === :psp || s === :dev) && return getfield(p, s)
    return getproperty(getfield(p, :psp), s)
end
Base.propertynames(p::PsPot_GTH_B200) = (:psp, :dev, propertynames(getfield(p, :psp))...)
# the GTH tables PWDFT dispatches on (PsPot_GTH.jl:123-260, 338-391)
PWDFT.eval_Vloc_G(p::PsPot_GTH_B200, args...) = PWDFT.eval_Vloc_G(p.psp, args...)
PWDFT.eval_Vloc_G!(p::PsPot_GTH_B200, args...) = PWDFT.eval_Vloc_G!(p.psp, args...)
PWDFT.eval_Vloc_G_short(p::PsPot_GTH_B200, args...) = PWDFT.eval_Vloc_G_short(p.psp, args...)
PWDFT.eval_Vloc_R(p::PsPot_GTH_B200, args...) = PWDFT.eval_Vloc_R(p.psp, args...)
PWDFT.eval_proj_G(p::PsPot_GTH_B200, args...) = PWDFT.eval_proj_G(p.psp, args...)
PWDFT.eval_proj_R(p::PsPot_GTH_B200, args...) = PWDFT.eval_proj_R(p.psp, args...)
PWDFT.print(io::IO, p::PsPot_GTH_B200; kw...) = PWDFT.print(io, p.psp; kw...)
PWDFT.print(p::PsPot_GTH_B200; kw...) = PWDFT.print(p.psp; kw...)
PWDFT.write_psp10(p::PsPot_GTH_B200; kw...) = PWDFT.write_psp10(p.psp; kw...)
# the methods PWDFT types on Vector{PsPot_GTH} (PsPot_GTH.jl:394, calc_PspCore_ene.jl:1,
# PsPotNL.jl:16, calc_forces_Ps_nloc.jl:347) take the wrapped GTH records
gth(pspots::Vector{PsPot_GTH_B200}) = [p.psp for p in pspots]
PWDFT.calc_Natomwfc(atoms::Atoms, pspots::Vector{PsPot_GTH_B200}) = PWDFT.calc_Natomwfc(atoms, gth(pspots))
PWDFT.calc_PspCore_ene(atoms::Atoms, pspots::Vector{PsPot_GTH_B200}) = PWDFT.calc_PspCore_ene(atoms, gth(pspots))
PWDFT.PsPotNL(atoms::Atoms, pw::PWGrid, pspots::Vector{PsPot_GTH_B200}; kw...) = PWDFT.PsPotNL(atoms, pw, gth(pspots); kw...)
PWDFT.calc_dbetaNL(atoms::Atoms, pw::PWGrid, pspots::Vector{PsPot_GTH_B200}, args...) =
    PWDFT.calc_dbetaNL(atoms, pw, gth(pspots), args...)

const B200Hamiltonian = Hamiltonian{PsPot_GTH_B200}
device(Ham::B200Hamiltonian) = Ham.pspots[1].dev

"""
    on_device(Ham; device=0, precision=:fp64) -> Hamiltonian{PsPot_GTH_B200}

Uploads the basis (PWGrid.gvecw), V_loc (Ham.potentials.Total) and the GTH
projectors (Ham.pspotNL) of a PWDFT `Hamiltonian` to one GPU and returns a
`Hamiltonian` with the same fields (shared, not copied) whose hot path runs
there.  precision = :fp64 (ComplexF64 throughout, the reference's
arithmetic) or :mixed (FP32 FFTs, split-BF16x3 tensor-core contractions,
FP64 small matrices).
"""
function on_device(Ham::Hamiltonian{PsPot_GTH}; device::Integer=0, precision::Symbol=:fp64)
    pw = Ham.pw
    gw = pw.gvecw
    Nkpt = gw.kpoints.Nkpt
    G = pw.gvec.G
    kpts = gw.kpoints.k
    Gk2 = [vec(sum(abs2, G[:, gw.idx_gw2g[ik]] .+ kpts[:, ik], dims=1)) for ik in 1:Nkpt]   # op_K.jl:70
    idx = [Vector{Int64}(gw.idx_gw2r[ik]) for ik in 1:Nkpt]
    Ngw = Vector{Int64}(gw.Ngw)
    pidx = [pointer(v) for v in idx]
    pgk2 = [pointer(v) for v in Gk2]
    desc = PwGridDesc(Int32.(pw.Ns), Int32(Nkpt), Int32(Ham.electrons.Nspin_wf), Int32(1), pw.CellVolume,
                      pointer(Ngw), pointer(pidx), pointer(pgk2))
    out = Ref{Ptr{Cvoid}}(C_NULL)
    st = GC.@preserve idx Gk2 Ngw pidx pgk2 ccall((:pw_create, libpwb200), Cint,
                                                  (Cint, Ref{PwGridDesc}, Ref{Ptr{Cvoid}}), device, desc, out)
    check(st, C_NULL)
    dev = DeviceContext(out[], precision == :mixed ? PW_C64 : PW_C128, false)
    finalizer(d -> ccall((:pw_destroy, libpwb200), Cvoid, (Ptr{Cvoid},), d.ctx), dev)
    pspots = [PsPot_GTH_B200(p, dev) for p in Ham.pspots]
    H = Hamiltonian{PsPot_GTH_B200}(Ham.pw, Ham.potentials, Ham.energies, Ham.rhoe_core, Ham.electrons, Ham.atoms,
                                    Ham.sym_info, Ham.rhoe_symmetrizer, pspots, Ham.pspotNL, Ham.xcfunc,
                                    Ham.xc_calc, Ham.ik, Ham.ispin, Ham.need_overlap, Ham.exx, Ham.options)
    upload_vloc!(H)
    upload_projectors!(H)
    return H
end

"After Ham.potentials.Total changed outside update! (update! re-uploads by itself)."
function upload_vloc!(Ham::B200Hamiltonian)
    V = Ham.potentials.Total
    c = device(Ham).ctx
    check(ccall((:pw_set_vloc, libpwb200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint), c, V, size(V, 2)), c)
end

# the (ibeta, jbeta, h_ij) pairs visited by op_V_Ps_nloc.jl:59-76, 0-based
function projector_pairs(Ham::B200Hamiltonian)
    ib, jb, h = Int32[], Int32[], Float64[]
    atoms = Ham.atoms
    for ia in 1:atoms.Natoms
        psp = Ham.pspots[atoms.atm2species[ia]].psp
        for l in 0:psp.lmax, m in -l:l, iprj in 1:psp.Nproj_l[l+1], jprj in 1:psp.Nproj_l[l+1]
            push!(ib, Ham.pspotNL.prj2beta[iprj, ia, l+1, m+psp.lmax+1] - 1)
            push!(jb, Ham.pspotNL.prj2beta[jprj, ia, l+1, m+psp.lmax+1] - 1)
            push!(h, psp.h[l+1, iprj, jprj])
        end
    end
    return ib, jb, h
end

function upload_projectors!(Ham::B200Hamiltonian)
    NbetaNL = Ham.pspotNL.NbetaNL
    NbetaNL == 0 && return
    c = device(Ham).ctx
    for ik in 1:Ham.pw.gvecw.kpoints.Nkpt
        beta = Ham.pspotNL.betaNL[ik]
        check(ccall((:pw_set_nonlocal, libpwb200), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Cint),
                    c, ik - 1, beta, NbetaNL), c)
    end
    ib, jb, h = projector_pairs(Ham)
    check(ccall((:pw_set_nonlocal_coef, libpwb200), Cint, (Ptr{Cvoid}, Cint, Ptr{Int32}, Ptr{Int32}, Ptr{Float64}),
                c, length(h), ib, jb, h), c)
end

# ------------------------------------------------------------ device staging
"A device buffer of the context (pw_device_alloc), freed with the object."
mutable struct DeviceBuffer
    ctx::Ptr{Cvoid}
    ptr::Ptr{Cvoid}
    bytes::UInt64
end
function DeviceBuffer(c::Ptr{Cvoid}, bytes::Integer)
    p = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:pw_device_alloc, libpwb200), Cint, (Ptr{Cvoid}, UInt64, Ref{Ptr{Cvoid}}), c, bytes, p), c)
    b = DeviceBuffer(c, p[], UInt64(bytes))
    finalizer(x -> ccall((:pw_device_free, libpwb200), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), x.ctx, x.ptr), b)
    return b
end
function to_device(c::Ptr{Cvoid}, a::Array)
    b = DeviceBuffer(c, sizeof(a))
    check(ccall((:pw_copy_to_device, libpwb200), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, UInt64),
                c, b.ptr, a, sizeof(a)), c)
    return b
end
function to_host!(a::Array, b::DeviceBuffer)
    check(ccall((:pw_copy_to_host, libpwb200), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, UInt64),
                b.ctx, a, b.ptr, sizeof(a)), b.ctx)
    return a
end
dense(psi::AbstractMatrix{ComplexF64}) = (psi isa StridedMatrix && stride(psi, 1) == 1) ? psi : Matrix(psi)

# ---------------------------------------------------------------- operators
function apply!(Ham::B200Hamiltonian, psi::AbstractMatrix{ComplexF64}, Hpsi::AbstractMatrix{ComplexF64}, ops::Cuint)
    dev = device(Ham)
    p = dense(psi)
    h = (Hpsi isa StridedMatrix && stride(Hpsi, 1) == 1) ? Hpsi : Matrix(Hpsi)
    if stride(h, 2) != stride(p, 2)   # pw_op_H_host takes one leading dimension for both blocks
        p = Matrix(psi)
        h === Hpsi && (h = Matrix(Hpsi))
    end
    check(ccall((:pw_op_H_host, libpwb200), Cint,
                (Ptr{Cvoid}, Cint, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}, Int64, Cint, Cuint, Cint),
                dev.ctx, Ham.ik - 1, Ham.ispin - 1, p, h, stride(p, 2), size(p, 2), ops, dev.dtype), dev.ctx)
    h === Hpsi || copyto!(Hpsi, h)
    return
end
apply!(Ham::B200Hamiltonian, psi::AbstractVector{ComplexF64}, Hpsi::AbstractVector{ComplexF64}, ops::Cuint) =
    apply!(Ham, reshape(psi, :, 1), reshape(Hpsi, :, 1), ops)

# op_H.jl:53-63 (zero-fill, then K + V_loc + V_Ps_nloc)
PWDFT.op_H!(Ham::B200Hamiltonian, psi::AbstractVecOrMat{ComplexF64}, Hpsi::AbstractVecOrMat{ComplexF64}) =
    apply!(Ham, psi, Hpsi, PW_OP_H)
# op_H.jl:4-27
function PWDFT.op_H(Ham::B200Hamiltonian, psi::AbstractVecOrMat{ComplexF64})
    Hpsi = zeros(ComplexF64, size(psi))
    apply!(Ham, psi, Hpsi, PW_OP_H)
    return Hpsi
end
# accumulating pieces: op_K.jl:44-75, op_V_loc.jl:33-92, op_V_Ps_nloc.jl:39-78
PWDFT.op_K!(Ham::B200Hamiltonian, psi::AbstractVecOrMat{ComplexF64}, Hpsi::AbstractVecOrMat{ComplexF64}) =
    apply!(Ham, psi, Hpsi, PW_OP_K | PW_ACCUMULATE)
PWDFT.op_V_loc!(Ham::B200Hamiltonian, psi::AbstractVecOrMat{ComplexF64}, Hpsi::AbstractVecOrMat{ComplexF64}) =
    apply!(Ham, psi, Hpsi, PW_OP_VLOC | PW_ACCUMULATE)
PWDFT.op_V_Ps_nloc!(Ham::B200Hamiltonian, psi::AbstractVecOrMat{ComplexF64}, Hpsi::AbstractVecOrMat{ComplexF64}) =
    apply!(Ham, psi, Hpsi, PW_OP_VNL | PW_ACCUMULATE)
# op_S.jl:82-89: norm-conserving GTH, S = identity
function PWDFT.op_S!(Ham::B200Hamiltonian, psi::AbstractArray{ComplexF64}, Spsi::AbstractArray{ComplexF64})
    @views Spsi[:, :] = psi[:, :]
    return
end

# calc_rhoe.jl:9-135 (Nspin = 1), then PWDFT's symmetrize_rhoe! as the reference does
function PWDFT.calc_rhoe!(Ham::B200Hamiltonian, psiks::BlochWavefunc, Rhoe::Array{Float64,2})
    dev = device(Ham)
    wk = Ham.pw.gvecw.kpoints.wk
    Focc = Ham.electrons.Focc
    rho = zeros(Float64, size(Rhoe, 1))
    for ik in 1:length(psiks)
        w = wk[ik] .* Focc[:, ik]
        p = dense(psiks[ik])
        check(ccall((:pw_calc_rhoe_host, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Int64, Cint, Ptr{Float64}, Ptr{Float64}, Cint, Cint),
                    dev.ctx, ik - 1, p, stride(p, 2), size(p, 2), w, rho, ik > 1, dev.dtype), dev.ctx)
    end
    Rhoe[:, 1] = rho
    if Ham.sym_info.Nsyms > 1
        PWDFT.symmetrize_rhoe!(Ham.pw, Ham.sym_info, Ham.rhoe_symmetrizer, Rhoe)
    end
    return
end

# update! (Hamiltonian.jl:510-645): PWDFT's own, then the new V_loc to the device
function PWDFT.update!(Ham::B200Hamiltonian, psiks::BlochWavefunc, Rhoe::Array{Float64,2})
    invoke(PWDFT.update!, Tuple{Hamiltonian,BlochWavefunc,Array{Float64,2}}, Ham, psiks, Rhoe)
    upload_vloc!(Ham)
end
function PWDFT.update!(Ham::B200Hamiltonian, psiks::BlochWavefunc, Rhoe::Vector{Float64})
    invoke(PWDFT.update!, Tuple{Hamiltonian,BlochWavefunc,Vector{Float64}}, Ham, psiks, Rhoe)
    upload_vloc!(Ham)
end
function PWDFT.update!(Ham::B200Hamiltonian, Rhoe::Array{Float64,2})
    invoke(PWDFT.update!, Tuple{Hamiltonian,Array{Float64,2}}, Ham, Rhoe)
    upload_vloc!(Ham)
end
function PWDFT.update!(Ham::B200Hamiltonian, rhoe::Vector{Float64})
    invoke(PWDFT.update!, Tuple{Hamiltonian,Vector{Float64}}, Ham, rhoe)
    upload_vloc!(Ham)
end

# ---------------------------------------------------------------- eigensolvers
# diag_LOBPCG.jl:51-225, the whole solve on the device (pw_lobpcg_host)
function PWDFT.diag_LOBPCG!(Ham::B200Hamiltonian, X::AbstractMatrix{ComplexF64}; tol=1e-5, NiterMax=100,
                            verbose=false, verbose_last=false, Nstates_conv=0)
    dev = device(Ham)
    Xd = dense(X)
    ev = zeros(Float64, size(X, 2))
    niter = Ref{Cint}(0)
    check(ccall((:pw_lobpcg_host, libpwb200), Cint,
                (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{ComplexF64}, Int64, Cint, Float64, Cint, Cint, Ptr{Float64}, Ref{Cint}),
                dev.ctx, Ham.ik - 1, Ham.ispin - 1, dev.dtype, Xd, stride(Xd, 2), size(Xd, 2), tol, NiterMax,
                Nstates_conv, ev, niter), dev.ctx)
    Xd === X || copyto!(X, Xd)
    return ev
end
# diag_LOBPCG.jl:1-28
function PWDFT.diag_LOBPCG!(Ham::B200Hamiltonian, psiks::BlochWavefunc; tol=1e-5, NiterMax=100,
                            verbose=false, verbose_last=false, Nstates_conv=0)
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    Nspin = Ham.electrons.Nspin_wf
    evals = zeros(Float64, Ham.electrons.Nstates, Nkpt * Nspin)
    for ispin in 1:Nspin, ik in 1:Nkpt
        Ham.ik, Ham.ispin = ik, ispin
        ikspin = ik + (ispin - 1) * Nkpt
        evals[:, ikspin] = PWDFT.diag_LOBPCG!(Ham, psiks[ikspin]; tol=tol, NiterMax=NiterMax,
                                              Nstates_conv=Nstates_conv)
    end
    return evals
end

# diag_davidson_qe_v2.jl:38-216 on the device (pw_davidson_host); EBANDS_THR = tol
function PWDFT.diag_davidson_qe!(Ham::B200Hamiltonian, psiks::BlochWavefunc; tol=1e-5, NiterMax=100,
                                 verbose=false, verbose_last=false, Nstates_conv=0)
    dev = device(Ham)
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    Nspin = Ham.electrons.Nspin_wf
    evals = zeros(Float64, Ham.electrons.Nstates, Nkpt * Nspin)
    niter = Ref{Cint}(0)
    for ispin in 1:Nspin, ik in 1:Nkpt
        Ham.ik, Ham.ispin = ik, ispin
        ikspin = ik + (ispin - 1) * Nkpt
        X = psiks[ikspin]
        ev = zeros(Float64, size(X, 2))
        check(ccall((:pw_davidson_host, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{ComplexF64}, Int64, Cint, Float64, Cint, Ptr{Float64}, Ref{Cint}),
                    dev.ctx, ik - 1, ispin - 1, dev.dtype, X, stride(X, 2), size(X, 2), tol, NiterMax, ev, niter),
              dev.ctx)
        evals[:, ikspin] = ev
    end
    return evals
end
# diag_davidson! (the 2-block solver of KS_solve_SCF.jl:194-198), diag_Emin_PCG!
# and diag_CheFSI! are PWDFT's own: they reach the device through op_H!,
# op_S!, calc_grad and Kprec on this Hamiltonian.

# calc_grad.jl:1-57 on the device (pw_calc_grad): the gradient of the
# band energy with the Hamiltonian's occupations of (Ham.ik, Ham.ispin)
function PWDFT.calc_grad(Ham::B200Hamiltonian, psi::Array{ComplexF64,2})
    dev = device(Ham)
    ik, ispin = Ham.ik, Ham.ispin
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    Focc = Vector{Float64}(Ham.electrons.Focc[:, ik + (ispin - 1) * Nkpt])
    wk = Ham.pw.gvecw.kpoints.wk[ik]
    # the device blocks are ComplexF64 (PW_C128), the reference's type
    p = to_device(dev.ctx, psi)
    g = DeviceBuffer(dev.ctx, sizeof(psi))
    check(ccall((:pw_calc_grad, libpwb200), Cint,
                (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Cint, Ptr{Float64}, Float64),
                dev.ctx, ik - 1, ispin - 1, PW_C128, p.ptr, g.ptr, size(psi, 1), size(psi, 2), Focc, wk), dev.ctx)
    return to_host!(similar(psi), g)
end

# ---------------------------------------------------------------- energies
# calc_energies.jl:7-58 (GTH): sum_k wk sum_b f_b sum_ij h_ij conj(B_i) B_j on
# the device (pw_band_energies), which also gives E_kin
function band_energies(Ham::B200Hamiltonian, psiks::BlochWavefunc)
    dev = device(Ham)
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    wk = Ham.pw.gvecw.kpoints.wk
    E = zeros(2)
    E2 = zeros(2)
    for ikspin in 1:length(psiks)
        ik = (ikspin - 1) % Nkpt + 1
        w = wk[ik] .* Ham.electrons.Focc[:, ikspin]
        p = to_device(dev.ctx, Matrix(psiks[ikspin]))
        check(ccall((:pw_band_energies, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Cint, Ptr{Cvoid}, Int64, Cint, Ptr{Float64}, Ptr{Float64}),
                    dev.ctx, ik - 1, PW_C128, p.ptr, size(psiks[ikspin], 1), size(psiks[ikspin], 2), w, E2), dev.ctx)
        E .+= E2
    end
    return E[1], E[2]
end
PWDFT.calc_E_Ps_nloc(Ham::B200Hamiltonian, psiks::BlochWavefunc) = band_energies(Ham, psiks)[2]

# ---------------------------------------------------------------- forces
function setup_forces!(Ham::B200Hamiltonian)
    dev = device(Ham)
    dev.forces_ready && return
    c = dev.ctx
    pw = Ham.pw
    gv = pw.gvec
    idx = Vector{Int64}(gv.idx_g2r)
    G2 = Vector{Float64}(gv.G2)
    check(ccall((:pw_set_density_sphere, libpwb200), Cint, (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Float64}, Cint),
                c, length(idx), idx, G2, 1), c)
    Nspecies = Ham.atoms.Nspecies
    VlocG = zeros(Float64, length(G2), Nspecies)
    for isp in 1:Nspecies
        VlocG[:, isp] = PWDFT.eval_Vloc_G(Ham.pspots[isp].psp, G2)   # PsPot_GTH.jl:164-189
    end
    G = Matrix{Float64}(gv.G)
    check(ccall((:pw_set_force_tables, libpwb200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Float64}),
                c, Nspecies, VlocG, G), c)
    gw = pw.gvecw
    for ik in 1:gw.kpoints.Nkpt
        gk = G[:, gw.idx_gw2g[ik]] .+ gw.kpoints.k[:, ik]
        check(ccall((:pw_set_gkvec, libpwb200), Cint, (Ptr{Cvoid}, Cint, Ptr{Float64}), c, ik - 1, gk), c)
    end
    if Ham.pspotNL.NbetaNL > 0
        atom_of_beta = zeros(Int32, Ham.pspotNL.NbetaNL)
        for ia in 1:Ham.atoms.Natoms
            psp = Ham.pspots[Ham.atoms.atm2species[ia]].psp
            for l in 0:psp.lmax, m in -l:l, iprj in 1:psp.Nproj_l[l+1]
                atom_of_beta[Ham.pspotNL.prj2beta[iprj, ia, l+1, m+psp.lmax+1]] = ia - 1
            end
        end
        check(ccall((:pw_set_nonlocal_atoms, libpwb200), Cint, (Ptr{Cvoid}, Cint, Ptr{Int32}),
                    c, Ham.atoms.Natoms, atom_of_beta), c)
    end
    dev.forces_ready = true
end

# calc_forces_Ps_loc.jl:13-72 on the device (pw_forces_local)
function PWDFT.calc_forces_Ps_loc!(Ham::B200Hamiltonian, Rhoe, F_Ps_loc::Array{Float64,2})
    setup_forces!(Ham)
    c = device(Ham).ctx
    r = to_device(c, Vector{Float64}(Rhoe[:, 1]))
    pos = Matrix{Float64}(Ham.atoms.positions)
    species = Int32.(Ham.atoms.atm2species .- 1)
    check(ccall((:pw_forces_local, libpwb200), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Cint, Ptr{Float64}, Ptr{Int32}, Ptr{Float64}),
                c, r.ptr, Ham.atoms.Natoms, pos, species, F_Ps_loc), c)
    return
end

# calc_forces_Ps_nloc.jl:291-411 for GTH on the device (pw_forces_nonlocal), summed over k
function PWDFT.calc_forces_Ps_nloc!(Ham::B200Hamiltonian, psiks::BlochWavefunc, F_Ps_nloc::Array{Float64,2})
    setup_forces!(Ham)
    c = device(Ham).ctx
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    wk = Ham.pw.gvecw.kpoints.wk
    F_Ps_nloc .= 0.0
    Fk = zeros(Float64, 3, Ham.atoms.Natoms)
    for ikspin in 1:length(psiks)
        ik = (ikspin - 1) % Nkpt + 1
        w = wk[ik] .* Ham.electrons.Focc[:, ikspin]
        p = to_device(c, Matrix(psiks[ikspin]))
        check(ccall((:pw_forces_nonlocal, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Cint, Ptr{Cvoid}, Int64, Cint, Ptr{Float64}, Ptr{Float64}),
                    c, ik - 1, PW_C128, p.ptr, size(psiks[ikspin], 1), size(psiks[ikspin], 2), w, Fk), c)
        F_Ps_nloc .+= Fk
    end
    return
end

# GTH pseudopotentials carry no core correction: the nonlinear-core and SCF
# correction forces are zero, as PWDFT's Hamiltonian{PsPot_GTH} methods
# (calc_forces_nlcc.jl:20-23, calc_forces_scf_corr.jl:8-11) make them
function PWDFT.calc_forces_nlcc!(Ham::B200Hamiltonian, F_nlcc)
    fill!(F_nlcc, 0.0)
    return
end
function PWDFT.calc_forces_scf_corr!(Ham::B200Hamiltonian, F_scf_corr)
    fill!(F_scf_corr, 0.0)
    return
end

"Total force: Ewald (PWDFT's calc_forces_NN) + the device local and nonlocal parts (symmetrised as calc_forces.jl:11)."
function forces(Ham::B200Hamiltonian, psiks::BlochWavefunc, Rhoe::Array{Float64,2})
    F_NN = PWDFT.calc_forces_NN(Ham.pw, Ham.atoms)
    F_loc = zeros(Float64, 3, Ham.atoms.Natoms)
    PWDFT.calc_forces_Ps_loc!(Ham, Rhoe, F_loc)
    F_nl = zeros(Float64, 3, Ham.atoms.Natoms)
    PWDFT.calc_forces_Ps_nloc!(Ham, psiks, F_nl)
    PWDFT.symmetrize_vector!(Ham.pw.LatVecs, Ham.sym_info, F_nl)
    return F_NN + F_loc + F_nl
end

# ---------------------------------------------------------------- adjoints
"""
    dE_dVloc(Ham, psiks) -> Vector{Float64}

dE/dV_loc(r) of the band energy sum_k wk sum_b f_b <psi_b|H|psi_b> at fixed
psi (pw_vloc_vjp, the adjoint of op_V_loc with respect to V): rho(r) dVol.
"""
function dE_dVloc(Ham::B200Hamiltonian, psiks::BlochWavefunc)
    c = device(Ham).ctx
    Npoints = prod(Ham.pw.Ns)
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    wk = Ham.pw.gvecw.kpoints.wk
    dV = DeviceBuffer(c, Npoints * sizeof(Float64))
    for ikspin in 1:length(psiks)
        ik = (ikspin - 1) % Nkpt + 1
        w = wk[ik] .* Ham.electrons.Focc[:, ikspin]
        p = to_device(c, Matrix(psiks[ikspin]))
        check(ccall((:pw_vloc_vjp, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Cint, Ptr{Cvoid}, Ptr{Cvoid}, Int64, Cint, Ptr{Float64}, Ptr{Cvoid}, Cint),
                    c, ik - 1, PW_C128, p.ptr, C_NULL, size(psiks[ikspin], 1), size(psiks[ikspin], 2), w, dV.ptr,
                    ikspin > 1), c)
    end
    return to_host!(zeros(Float64, Npoints), dV)
end

"The local-potential part of the band energy, sum_r V(r) dE/dV_loc(r), as a function of V at fixed psi."
local_band_energy(Ham::B200Hamiltonian, V::Vector{Float64}, psiks::BlochWavefunc) = dot(V, dE_dVloc(Ham, psiks))

function ChainRulesCore.rrule(::typeof(local_band_energy), Ham::B200Hamiltonian, V::Vector{Float64},
                              psiks::BlochWavefunc)
    g = dE_dVloc(Ham, psiks)
    local_band_energy_pullback(dE) = (NoTangent(), NoTangent(), unthunk(dE) .* g, NoTangent())
    return dot(V, g), local_band_energy_pullback
end

"The converged total energy (Ham.energies) as a function of the atomic positions."
ionic_energy(Ham::B200Hamiltonian, positions::Matrix{Float64}, psiks::BlochWavefunc, Rhoe::Array{Float64,2}) =
    sum(Ham.energies)

function ChainRulesCore.rrule(::typeof(ionic_energy), Ham::B200Hamiltonian, positions::Matrix{Float64},
                              psiks::BlochWavefunc, Rhoe::Array{Float64,2})
    F = forces(Ham, psiks, Rhoe)   # Hellmann-Feynman: dE/dtau = -F at self-consistency
    ionic_energy_pullback(dE) = (NoTangent(), NoTangent(), -unthunk(dE) .* F, NoTangent(), NoTangent())
    return sum(Ham.energies), ionic_energy_pullback
end

end # module
