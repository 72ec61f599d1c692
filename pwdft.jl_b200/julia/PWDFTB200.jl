"""
    PWDFTB200

Julia binding of libpwb200.so, the B200 implementation of PWDFT.jl's
op_H / calc_rhoe / LOBPCG hot path.  It adds methods to PWDFT's generic
functions for a `B200Hamiltonian` wrapper, so that `KS_solve_SCF!`-style
drivers run the hot path on the GPU while the rest of the Hamiltonian
(set-up, update!, energies, mixing) stays in PWDFT.jl.

Written against include/pwb200.h.  Julia is not installed in the build
image, so this file is not exercised by the test suite; the same ABI is
exercised from Python (pwdft.jl_b200/pwb200) on every run.
"""
module PWDFTB200

using PWDFT
using LinearAlgebra

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

"""
    B200Hamiltonian(Ham; device=0, precision=:fp64)

Uploads the basis (PWGrid.gvecw), V_loc (Ham.potentials.Total) and the GTH
projectors (Ham.pspotNL) of a PWDFT `Hamiltonian` to one GPU.
precision = :fp64 (ComplexF64 throughout) or :mixed (FP32 FFTs, split-BF16x3
tensor-core contractions, FP64 small matrices).
"""
mutable struct B200Hamiltonian
    ctx::Ptr{Cvoid}
    Ham::Hamiltonian
    dtype::Cint
    keep::Vector{Any}   # arrays whose pointers the descriptor holds during pw_create
end

function B200Hamiltonian(Ham::Hamiltonian; device::Integer=0, precision::Symbol=:fp64)
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
    B = B200Hamiltonian(out[], Ham, precision == :mixed ? PW_C64 : PW_C128, Any[])
    finalizer(b -> ccall((:pw_destroy, libpwb200), Cvoid, (Ptr{Cvoid},), b.ctx), B)
    update_vloc!(B)
    upload_projectors!(B)
    return B
end

"After PWDFT.update!(Ham, ...) changed Ham.potentials.Total."
function update_vloc!(B::B200Hamiltonian)
    V = B.Ham.potentials.Total
    check(ccall((:pw_set_vloc, libpwb200), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint), B.ctx, V, size(V, 2)), B.ctx)
end

function upload_projectors!(B::B200Hamiltonian)
    Ham = B.Ham
    NbetaNL = Ham.pspotNL.NbetaNL
    NbetaNL == 0 && return
    for ik in 1:Ham.pw.gvecw.kpoints.Nkpt
        beta = Ham.pspotNL.betaNL[ik]
        check(ccall((:pw_set_nonlocal, libpwb200), Cint, (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Cint),
                    B.ctx, ik - 1, beta, NbetaNL), B.ctx)
    end
    # the (ibeta, jbeta, h_ij) pairs of op_V_Ps_nloc.jl:59-76
    ib, jb, h = Int32[], Int32[], Float64[]
    atoms = Ham.atoms
    for ia in 1:atoms.Natoms
        psp = Ham.pspots[atoms.atm2species[ia]]
        for l in 0:psp.lmax, m in -l:l, iprj in 1:psp.Nproj_l[l+1], jprj in 1:psp.Nproj_l[l+1]
            push!(ib, Ham.pspotNL.prj2beta[iprj, ia, l+1, m+psp.lmax+1] - 1)
            push!(jb, Ham.pspotNL.prj2beta[jprj, ia, l+1, m+psp.lmax+1] - 1)
            push!(h, psp.h[l+1, iprj, jprj])
        end
    end
    check(ccall((:pw_set_nonlocal_coef, libpwb200), Cint, (Ptr{Cvoid}, Cint, Ptr{Int32}, Ptr{Int32}, Ptr{Float64}),
                B.ctx, length(h), ib, jb, h), B.ctx)
end

# ---------------------------------------------------------------- operators
function apply!(B::B200Hamiltonian, psi::AbstractMatrix{ComplexF64}, Hpsi::AbstractMatrix{ComplexF64}, ops::Cuint)
    Ham = B.Ham
    check(ccall((:pw_op_H_host, libpwb200), Cint,
                (Ptr{Cvoid}, Cint, Cint, Ptr{ComplexF64}, Ptr{ComplexF64}, Int64, Cint, Cuint, Cint),
                B.ctx, Ham.ik - 1, Ham.ispin - 1, psi, Hpsi, stride(psi, 2), size(psi, 2), ops, B.dtype), B.ctx)
    return
end

# op_H.jl:53-63 (zero-fill, then K + V_loc + V_Ps_nloc)
PWDFT.op_H!(B::B200Hamiltonian, psi, Hpsi) = apply!(B, psi, Hpsi, PW_OP_H)
# op_H.jl:4-27
function PWDFT.op_H(B::B200Hamiltonian, psi::AbstractMatrix{ComplexF64})
    Hpsi = similar(psi)
    apply!(B, psi, Hpsi, PW_OP_H)
    return Hpsi
end
# accumulating pieces: op_K.jl:44-75, op_V_loc.jl:108-167, op_V_Ps_nloc.jl:39-78
PWDFT.op_K!(B::B200Hamiltonian, psi, Hpsi) = apply!(B, psi, Hpsi, PW_OP_K | PW_ACCUMULATE)
PWDFT.op_V_loc!(B::B200Hamiltonian, psi, Hpsi) = apply!(B, psi, Hpsi, PW_OP_VLOC | PW_ACCUMULATE)
PWDFT.op_V_Ps_nloc!(B::B200Hamiltonian, psi, Hpsi) = apply!(B, psi, Hpsi, PW_OP_VNL | PW_ACCUMULATE)

# calc_rhoe.jl:9-135 (Nspin = 1, no symmetrisation: symmetrize_rhoe! stays in PWDFT)
function PWDFT.calc_rhoe!(B::B200Hamiltonian, psiks::BlochWavefunc, Rhoe::Matrix{Float64})
    Ham = B.Ham
    wk = Ham.pw.gvecw.kpoints.wk
    Focc = Ham.electrons.Focc
    rho = @view Rhoe[:, 1]
    for ik in 1:length(psiks)
        w = wk[ik] .* Focc[:, ik]
        check(ccall((:pw_calc_rhoe_host, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Ptr{ComplexF64}, Int64, Cint, Ptr{Float64}, Ptr{Float64}, Cint, Cint),
                    B.ctx, ik - 1, psiks[ik], stride(psiks[ik], 2), size(psiks[ik], 2), w, rho, ik > 1, B.dtype),
              B.ctx)
    end
    if Ham.sym_info.Nsyms > 1
        PWDFT.symmetrize_rhoe!(Ham.pw, Ham.sym_info, Ham.rhoe_symmetrizer, Rhoe)
    end
    return
end

# diag_LOBPCG.jl:1-28: every (ispin, ik) block solved on the device by
# pw_lobpcg_host; psiks stay host arrays, copied in and out around each solve.
function PWDFT.diag_LOBPCG!(B::B200Hamiltonian, psiks::BlochWavefunc; tol=1e-5, NiterMax=100,
                            verbose=false, verbose_last=false, Nstates_conv=0)
    Ham = B.Ham
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    Nspin = Ham.electrons.Nspin_wf
    Nstates = Ham.electrons.Nstates
    evals = zeros(Float64, Nstates, Nkpt * Nspin)
    niter = Ref{Cint}(0)
    for ispin in 1:Nspin, ik in 1:Nkpt
        Ham.ik, Ham.ispin = ik, ispin
        ikspin = ik + (ispin - 1) * Nkpt
        X = psiks[ikspin]
        ev = zeros(Float64, Nstates)
        check(ccall((:pw_lobpcg_host, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{ComplexF64}, Int64, Cint, Float64, Cint, Cint, Ptr{Float64}, Ref{Cint}),
                    B.ctx, ik - 1, ispin - 1, B.dtype, X, stride(X, 2), size(X, 2), tol, NiterMax, Nstates_conv, ev, niter),
              B.ctx)
        evals[:, ikspin] = ev
    end
    return evals
end

# diag_davidson_qe_v2.jl:6-34: every (ispin, ik) block through
# pw_davidson_host (diag_davidson_qe!, S = identity); EBANDS_THR = tol.
function PWDFT.diag_davidson_qe!(B::B200Hamiltonian, psiks::BlochWavefunc; tol=1e-5, NiterMax=100,
                                 verbose=false, verbose_last=false, Nstates_conv=0)
    Ham = B.Ham
    Nkpt = Ham.pw.gvecw.kpoints.Nkpt
    Nspin = Ham.electrons.Nspin_wf
    Nstates = Ham.electrons.Nstates
    evals = zeros(Float64, Nstates, Nkpt * Nspin)
    niter = Ref{Cint}(0)
    for ispin in 1:Nspin, ik in 1:Nkpt
        Ham.ik, Ham.ispin = ik, ispin
        ikspin = ik + (ispin - 1) * Nkpt
        X = psiks[ikspin]
        ev = zeros(Float64, Nstates)
        check(ccall((:pw_davidson_host, libpwb200), Cint,
                    (Ptr{Cvoid}, Cint, Cint, Cint, Ptr{ComplexF64}, Int64, Cint, Float64, Cint, Ptr{Float64}, Ref{Cint}),
                    B.ctx, ik - 1, ispin - 1, B.dtype, X, stride(X, 2), size(X, 2), tol, NiterMax, ev, niter),
              B.ctx)
        evals[:, ikspin] = ev
    end
    return evals
end

end # module
