"""FP64 CPU oracle for the PWDFT.jl op_H / calc_rhoe / LOBPCG hot path.

TEST INFRASTRUCTURE ONLY.  This package is a NumPy/SciPy restatement of the
reference algorithms (PWDFT.jl, Julia) used as the checker for the CUDA path:
it may be imported only by ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The product
(``pwdft.jl_b200/pwb200`` and ``libpwb200.so``) never imports or calls it.

Parity pinning: the reference's own Julia code cannot run in this image (no
Julia, FFTW or Libxc), so the oracle is pinned to the reference's published
golden numbers instead -- the Si fcc LDA total energy (-7.9110087934 Ha,
test/validations_old/Si_fcc.jl:15) and its logged components
(test/LOG_runtest_v.1.1.1:1171-1181), the Ewald energy
(test/test_energies.jl:19), the VWN known answers (test/test_xc.jl:3-4), the
lattice matrices (test/test_gen_lattice.jl) and the free-electron spectrum
(timing/time_diag_LOBPCG.jl:5-84).  See tests/test_oracle_golden.py.

Module map (each function cites the reference file:line it follows):
  pwgrid     PWGrid.jl, fft_support.jl, KPoints.jl, gen_lattice.jl
  gth        PsPot_GTH.jl, Ylm_real.jl
  ham        Hamiltonian.jl, PsPotNL.jl, calc_strfact.jl, Electrons.jl,
             guess_rhoe.jl, Poisson_solve.jl, XC_funcs/*.jl
  ops        op_K.jl, op_V_loc.jl, op_V_Ps_nloc.jl, op_H.jl, Kprec.jl,
             calc_rhoe.jl
  lobpcg     diag_LOBPCG.jl, ortho_sqrt.jl
  energies   calc_energies.jl, calc_E_NN.jl
  scf        KS_solve_SCF.jl, mix_pulay.jl
  systems    the synthetic benchmark systems (Si2 fcc, Si64, Si216, Al4)
"""
