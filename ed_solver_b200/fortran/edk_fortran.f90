! edk_fortran -- ISO_C_BINDING interface to libedk.so for the ed_solver code.
!
! The bind(C) interfaces mirror include/edk.h one to one.  The wrappers at
! the bottom (edk_new_H, edk_Hmult_real, edk_delete_H) show how the module
! procedures of H_class.f90 (new_H :28, Hmult__/Hmultr :69-136, delete_H :48)
! forward to the library; see the integration notes for the call-site edits.
! Vectors handed to edk_hmult must be device pointers (c_devptr from CUDA
! Fortran, or cudaMalloc'd memory); edk_hmult_host takes host arrays.
module edk_fortran
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: EDK_OK = 0, EDK_F64 = 0, EDK_F32 = 1
  integer(c_int), parameter :: EDK_KRYLOV_EXHAUSTED = 4

  type, bind(C) :: edk_model
    integer(c_int32_t) :: nc, nb
    type(c_ptr) :: ec, eb, vbc, u, jj
    real(c_double) :: jhund
    real(c_double) :: cutoff_hamilt_param
  end type

  ! Nambu (Sz) sectors: the normal part plus Pb(k,k') and PVbc_s(k,c) (bath_class.f90:956-1022)
  type, bind(C) :: edk_model_sz
    type(edk_model) :: base
    type(c_ptr) :: pb, pvbc
    integer(c_int32_t) :: on_fly
  end type

  ! one eigenstate of a GS.raw checkpoint (write_raw_eigensectorlist, eigen_sector_class.f90:514-567)
  type, bind(C) :: edk_gs_entry
    integer(c_int32_t) :: kind, norbs, nup, ndn
    real(c_double) :: val
    integer(c_int32_t) :: converged, rank
    integer(c_int64_t) :: n, offset
  end type

  ! the sectors and c+ matrices of chi_tilde_loc_ (Chiloc_Wenhu_version3.cpp:106-150)
  type, bind(C) :: edk_chiloc_sectors
    integer(c_int32_t) :: dim(11)
    type(c_ptr) :: E(11)
    type(c_ptr) :: C(14)
  end type

  type, bind(C) :: edk_lanczos_opts
    integer(c_int32_t) :: nitermax, neigen
    real(c_double) :: tolerance, demax, cutoff_min_lanczos_vec
    integer(c_int32_t) :: dtype, check_every
    type(c_ptr) :: ran_tab, start_dev
    integer(c_int32_t) :: use_target
    real(c_double) :: target, residual_tol
    integer(c_int32_t) :: keep_basis
  end type

  ! parameter of the adjoint: kind EDK_PARAM_EC=0, EB=1, VBC=2, U=3 (0-based i, j);
  ! spin 0 up, 1 down, 2 both
  type, bind(C) :: edk_param
    integer(c_int32_t) :: kind, i, j, spin
  end type

  ! one Green channel of an eigenstate (0-based site; site2 < 0: single operator)
  type, bind(C) :: edk_green_spec
    integer(c_int32_t) :: site, spin, dagger, site2, sign2
  end type

  type, bind(C) :: edk_grad_stats
    integer(c_int64_t) :: forward_steps, replay_steps, reverse_steps
    integer(c_int32_t) :: cg_iterations
    real(c_double) :: cg_residual
    integer(c_int32_t) :: stored_vectors
  end type

  ! block Lanczos options (edk_block_lanczos)
  type, bind(C) :: edk_block_opts
    integer(c_int32_t) :: block, nitermax, neigen
    real(c_double) :: tolerance
    integer(c_int32_t) :: check_every
    type(c_ptr) :: ran_tab
  end type

  ! one chain of a batched Green-function launch (edk_green_batch)
  type, bind(C) :: edk_chain
    type(c_ptr) :: target, start_dev
    real(c_double) :: e0
    integer(c_int32_t) :: iph
    real(c_double) :: weight
    integer(c_int32_t) :: out
  end type

  type, bind(C) :: edk_batch_stats
    integer(c_int64_t) :: steps
    integer(c_int32_t) :: chains
    real(c_double) :: kernel_ms
    integer(c_int32_t) :: block, rows, blocks_per_sm, tuned_shapes
  end type

  ! one impurity solve (edk_solve): options and results
  type, bind(C) :: edk_solve_opts
    integer(c_int32_t) :: dtype, nsectors
    type(c_ptr) :: sectors
    integer(c_int32_t) :: neigen, nitermax
    real(c_double) :: tolerance, tolerance_lowprec
    integer(c_int32_t) :: check_every
    real(c_double) :: beta, demax0
    integer(c_int32_t) :: nitergreen, nw, spin_mask, npairs
    type(c_ptr) :: pairs
    real(c_double) :: cutoff_dynamic
    type(c_ptr) :: ran_tab
    real(c_double) :: residual_tol
    integer(c_int32_t) :: green_mode
    type(c_ptr) :: gs_in, gs_out, sector_bound_file
    integer(c_int32_t) :: iwindow, recompute_pass2, reference_small_sectors
    integer(c_int64_t) :: lowprec_min_dim
    integer(c_int32_t) :: fp32_sums, batch_gs
  end type

  type, bind(C) :: edk_solve_result
    real(c_double) :: e0, z, e0_lowprec, residual
    integer(c_int32_t) :: nstates, lanczos_steps, green_steps
    type(c_ptr) :: G, docc, energies, state_sectors
  end type

  type, bind(C) :: edk_lanczos_result
    integer(c_int32_t) :: nkept, niter, status
    real(c_double) :: E(64)
    integer(c_int32_t) :: converged(64)
    type(c_ptr) :: diag, subdiag, vecp
  end type

  interface
    integer(c_int) function edk_ctx_create(device, stream, ctx) bind(C, name="edk_ctx_create")
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr), value :: stream
      type(c_ptr) :: ctx
    end function
    integer(c_int) function edk_ctx_destroy(ctx) bind(C, name="edk_ctx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function edk_h_create(ctx, m, nup, ndn, h) bind(C, name="edk_h_create")
      import :: c_int, c_ptr, edk_model
      type(c_ptr), value :: ctx
      type(edk_model), intent(in) :: m
      integer(c_int), value :: nup, ndn
      type(c_ptr) :: h
    end function
    integer(c_int) function edk_h_destroy(h) bind(C, name="edk_h_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function edk_h_dims(h, dim, dim_up, dim_dn) bind(C, name="edk_h_dims")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: h
      integer(c_int64_t) :: dim, dim_up, dim_dn
    end function
    integer(c_int) function edk_hmult(h, dtype, n, x, y) bind(C, name="edk_hmult")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: h
      integer(c_int), value :: dtype
      integer(c_int64_t), value :: n
      type(c_ptr), value :: x, y
    end function
    integer(c_int) function edk_hmult_split(h, dtype, n, x, y) bind(C, name="edk_hmult_split")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: h
      integer(c_int), value :: dtype
      integer(c_int64_t), value :: n
      type(c_ptr), value :: x, y
    end function
    integer(c_int) function edk_hmult_host(h, dtype, n, x, y) bind(C, name="edk_hmult_host")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: dtype
      integer(c_int64_t), value :: n
      real(c_double), intent(in) :: x(*)
      real(c_double), intent(out) :: y(*)
    end function
    integer(c_int) function edk_lanczos_e0(h, o, r) bind(C, name="edk_lanczos_e0")
      import :: c_int, c_ptr, edk_lanczos_opts, edk_lanczos_result
      type(c_ptr), value :: h
      type(edk_lanczos_opts), intent(in) :: o
      type(edk_lanczos_result), intent(inout) :: r
    end function
    integer(c_int) function edk_lanczos_gs(h, o, niter, coef, psi) bind(C, name="edk_lanczos_gs")
      import :: c_int, c_ptr, c_int32_t, c_double, edk_lanczos_opts
      type(c_ptr), value :: h
      type(edk_lanczos_opts), intent(in) :: o
      integer(c_int32_t), value :: niter
      real(c_double), intent(in) :: coef(*)
      type(c_ptr), value :: psi
    end function
    integer(c_int) function edk_apply_c(src, dtype, site, spin, dagger, site2, sign2, vin, vout, out_dim) &
        bind(C, name="edk_apply_c")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: src
      integer(c_int), value :: dtype, site, spin, dagger, site2, sign2
      type(c_ptr), value :: vin, vout
      integer(c_int64_t) :: out_dim
    end function
    integer(c_int) function edk_green_chain(t, dtype, start, nitergreen, e0, iph, nw, wn, cutoff_dynamic, &
        G, diag, subdiag, niter_done) bind(C, name="edk_green_chain")
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: t
      integer(c_int), value :: dtype, iph
      type(c_ptr), value :: start
      integer(c_int32_t), value :: nitergreen, nw
      real(c_double), value :: e0, cutoff_dynamic
      real(c_double), intent(in) :: wn(*)
      real(c_double), intent(out) :: G(*), diag(*), subdiag(*)
      integer(c_int32_t) :: niter_done
    end function

    ! ED_diago (ED_ARPACK.f90:590-715): every eigenpair of a small sector
    integer(c_int) function edk_full_ed(h, E, V) bind(C, name="edk_full_ed")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double) :: E(*), V(*)
    end function
    ! chi_tilde_loc_ for nf frequency triples (w: nf x 6 doubles)
    integer(c_int) function edk_chiloc(ctx, op_mask, beta, Z, gs_e, phi_eps, sites, nup, ndn, s, nf, w, &
        pdndn, pupdn) bind(C, name="edk_chiloc")
      import :: c_int, c_ptr, c_int32_t, c_double, edk_chiloc_sectors
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: op_mask, sites, nup, ndn, nf
      real(c_double), value :: beta, Z, gs_e, phi_eps
      type(edk_chiloc_sectors), intent(in) :: s
      real(c_double), intent(in) :: w(*)
      real(c_double) :: pdndn(*), pupdn(*)
    end function

    ! apply_Csz on Nambu impurity orbitals (0-based orb < 2nc), + sign2 * the same on orb2 >= 0
    integer(c_int) function edk_apply_cnambu(src, dtype, orb, dagger, orb2, sign2, vin, vout, out_dim, out_npart) &
        bind(C, name="edk_apply_cnambu")
      import :: c_int, c_ptr, c_int32_t, c_int64_t
      type(c_ptr), value :: src
      integer(c_int), value :: dtype, orb, dagger, orb2, sign2
      type(c_ptr), value :: vin, vout
      integer(c_int64_t) :: out_dim
      integer(c_int32_t) :: out_npart
    end function

    ! GS.raw checkpoints and ed.sector_bound_file (host-only)
    integer(c_int) function edk_gs_write(path, nentries, entries, pool) bind(C, name="edk_gs_write")
      import :: c_int, c_char, c_int32_t, c_double, edk_gs_entry
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: nentries
      type(edk_gs_entry), intent(in) :: entries(*)
      real(c_double), intent(in) :: pool(*)
    end function
    integer(c_int) function edk_gs_read(path, cap, entries, nentries, vec_cap, pool, vec_total) &
        bind(C, name="edk_gs_read")
      import :: c_int, c_char, c_int32_t, c_int64_t, c_double, edk_gs_entry
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), value :: cap
      type(edk_gs_entry) :: entries(*)
      integer(c_int32_t) :: nentries
      integer(c_int64_t), value :: vec_cap
      real(c_double) :: pool(*)
      integer(c_int64_t) :: vec_total
    end function
    integer(c_int) function edk_sector_bounds_read(path, bounds, has_sz) bind(C, name="edk_sector_bounds_read")
      import :: c_int, c_char, c_int32_t
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t) :: bounds(6), has_sz
    end function
    integer(c_int) function edk_sector_bounds_write(path, bounds) bind(C, name="edk_sector_bounds_write")
      import :: c_int, c_char, c_int32_t
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int32_t), intent(in) :: bounds(6)
    end function

    ! new_HAIMsz (HAIMsz.f90:51-82): the sector of npart Nambu particles
    integer(c_int) function edk_h_create_sz(ctx, m, npart, h) bind(C, name="edk_h_create_sz")
      import :: c_int, c_ptr, edk_model_sz
      type(c_ptr), value :: ctx
      type(edk_model_sz), intent(in) :: m
      integer(c_int), value :: npart
      type(c_ptr) :: h
    end function
    integer(c_int) function edk_h_sz_info(h, npart, energy_shift) bind(C, name="edk_h_sz_info")
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: h
      integer(c_int32_t) :: npart
      real(c_double) :: energy_shift
    end function
    ! apply_Csz_updo / apply_Csz_N_updo (apply_C.f90:344-483)
    integer(c_int) function edk_apply_csz_ab(src, dtype, site, proj, site2, proj2, spin, dagger, vin, vout, &
        out_dim, out_npart) bind(C, name="edk_apply_csz_ab")
      import :: c_int, c_ptr, c_int32_t, c_int64_t
      type(c_ptr), value :: src
      integer(c_int), value :: dtype, site, proj, site2, proj2, spin, dagger
      type(c_ptr), value :: vin, vout
      integer(c_int64_t) :: out_dim
      integer(c_int32_t) :: out_npart
    end function
    integer(c_int) function edk_apply_csz(src, dtype, site, spin, dagger, projected, site2, sign2, vin, vout, &
        out_dim, out_npart) bind(C, name="edk_apply_csz")
      import :: c_int, c_ptr, c_int32_t, c_int64_t
      type(c_ptr), value :: src
      integer(c_int), value :: dtype, site, spin, dagger, projected, site2, sign2
      type(c_ptr), value :: vin, vout
      integer(c_int64_t) :: out_dim
      integer(c_int32_t) :: out_npart
    end function

    ! <a| dH/dtheta_q |b> for every parameter (FP64 device vectors a, b)
    integer(c_int) function edk_dh_bilinear(h, a, b, np, params, out) bind(C, name="edk_dh_bilinear")
      import :: c_int, c_ptr, c_int32_t, c_double, edk_param
      type(c_ptr), value :: h, a, b
      integer(c_int32_t), value :: np
      type(edk_param), intent(in) :: params(*)
      real(c_double), intent(out) :: out(*)
    end function

    ! Hellmann-Feynman dE/dtheta_q of the state psi (FP64 device vector)
    integer(c_int) function edk_grad_e0(h, psi, np, params, grad) bind(C, name="edk_grad_e0")
      import :: c_int, c_ptr, c_int32_t, c_double, edk_param
      type(c_ptr), value :: h, psi
      integer(c_int32_t), value :: np
      type(edk_param), intent(in) :: params(*)
      real(c_double), intent(out) :: grad(*)
    end function

    ! vector-Jacobian product of the Green functions and of E0 of the eigenstate psi
    integer(c_int) function edk_grad_green(h, psi, e0, nchain, chains, nitergreen, nw, wn, gbar, e0bar, &
        np, params, cg_tol, grad, G, stats) bind(C, name="edk_grad_green")
      import :: c_int, c_ptr, c_int32_t, c_double, edk_param, edk_green_spec, edk_grad_stats
      type(c_ptr), value :: h, psi
      real(c_double), value :: e0, e0bar, cg_tol
      integer(c_int32_t), value :: nchain, nitergreen, nw, np
      type(edk_green_spec), intent(in) :: chains(*)
      real(c_double), intent(in) :: wn(*), gbar(*)
      type(edk_param), intent(in) :: params(*)
      real(c_double), intent(out) :: grad(*), G(*)
      type(edk_grad_stats), intent(out) :: stats
    end function

    ! ---- context utilities ----
    integer(c_int) function edk_ctx_set_stream(ctx, stream) bind(C, name="edk_ctx_set_stream")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, stream
    end function
    type(c_ptr) function edk_ctx_last_error(ctx) bind(C, name="edk_ctx_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int64_t) function edk_ctx_launch_count(ctx) bind(C, name="edk_ctx_launch_count")
      import :: c_int64_t, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function edk_ctx_timing(ctx, enable) bind(C, name="edk_ctx_timing")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: enable
    end function
    integer(c_int) function edk_ctx_set_kernel_path(ctx, path) bind(C, name="edk_ctx_set_kernel_path")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: path
    end function
    integer(c_int) function edk_ctx_set_graphs(ctx, enable) bind(C, name="edk_ctx_set_graphs")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: enable
    end function
    integer(c_int) function edk_ctx_timing_report(ctx, which, launches, total_ms) &
        bind(C, name="edk_ctx_timing_report")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: which
      integer(c_int64_t) :: launches
      real(c_double) :: total_ms
    end function
    integer(c_int) function edk_ctx_timing_elements(ctx, which, elements) bind(C, name="edk_ctx_timing_elements")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: which
      real(c_double) :: elements
    end function
    integer(c_int) function edk_ctx_transfer_bytes(ctx, h2d, d2h) bind(C, name="edk_ctx_transfer_bytes")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int64_t) :: h2d, d2h
    end function
    integer(c_int) function edk_ctx_clear_cache(ctx) bind(C, name="edk_ctx_clear_cache")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function edk_h_launch_shape_chosen(h, dtype, fp32_sums, desc) &
        bind(C, name="edk_h_launch_shape_chosen")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: h
      integer(c_int), value :: dtype, fp32_sums
      integer(c_int32_t) :: desc(5)
    end function
    integer(c_int) function edk_h_launch_shapes(h, dtype, desc, cap) bind(C, name="edk_h_launch_shapes")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: h
      integer(c_int), value :: dtype
      integer(c_int32_t) :: desc(*)
      integer(c_int32_t), value :: cap
    end function
    integer(c_int) function edk_ctx_set_fp32_sums(ctx, enable, min_dim) bind(C, name="edk_ctx_set_fp32_sums")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: enable
      integer(c_int64_t), value :: min_dim
    end function
    integer(c_int) function edk_ctx_trim(ctx) bind(C, name="edk_ctx_trim")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function edk_ctx_set_workspace_limit(ctx, bytes) bind(C, name="edk_ctx_set_workspace_limit")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: bytes
    end function

    ! ---- basis and tables (host-only) ----
    integer(c_int64_t) function edk_binom(n, k) bind(C, name="edk_binom")
      import :: c_int64_t, c_int
      integer(c_int), value :: n, k
    end function
    ! states as unsigned 64-bit patterns, read through integer(c_int64_t)
    integer(c_int) function edk_basis(ns, npart, states) bind(C, name="edk_basis")
      import :: c_int, c_int64_t
      integer(c_int), value :: ns, npart
      integer(c_int64_t) :: states(*)
    end function
    integer(c_int) function edk_rank_table(ns, rank) bind(C, name="edk_rank_table")
      import :: c_int, c_int32_t
      integer(c_int), value :: ns
      integer(c_int32_t) :: rank(*)
    end function
    integer(c_int) function edk_default_ran_tab(tab) bind(C, name="edk_default_ran_tab")
      import :: c_int, c_double
      real(c_double) :: tab(10001)
    end function
    ! arrays may be c_null_ptr for the size query
    integer(c_int) function edk_build_table(m, spin, npart, dim, nnz, ptr, tgt, val, diag) &
        bind(C, name="edk_build_table")
      import :: c_int, c_ptr, c_int64_t, edk_model
      type(edk_model), intent(in) :: m
      integer(c_int), value :: spin, npart
      integer(c_int64_t) :: dim, nnz
      type(c_ptr), value :: ptr, tgt, val, diag
    end function
    integer(c_int) function edk_h_table(h, spin, nnz, ptr, tgt, val, diag) bind(C, name="edk_h_table")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: h
      integer(c_int), value :: spin
      integer(c_int64_t) :: nnz
      type(c_ptr), value :: ptr, tgt, val, diag
    end function

    ! ---- vectors and observables ----
    integer(c_int) function edk_convert(ctx, from_dtype, to_dtype, n, vin, vout) bind(C, name="edk_convert")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: from_dtype, to_dtype
      integer(c_int64_t), value :: n
      type(c_ptr), value :: vin, vout
    end function
    integer(c_int) function edk_residual(h, psi, e, res_norm, psi_norm) bind(C, name="edk_residual")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h, psi
      real(c_double), value :: e
      real(c_double) :: res_norm, psi_norm
    end function
    integer(c_int) function edk_double_occ(h, dtype, psi, site, docc, norm2) bind(C, name="edk_double_occ")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h, psi
      integer(c_int), value :: dtype, site
      real(c_double) :: docc, norm2
    end function

    ! ---- continued fractions (invert_zmtridiag, matrices_tridiag.f90:163-198) ----
    integer(c_int) function edk_cf_eval(ctx, nchain, ld, n, diag, subdiag, e, ph, scale, nw, wn, G) &
        bind(C, name="edk_cf_eval")
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nchain, ld, nw
      integer(c_int32_t), intent(in) :: n(*)
      real(c_double), intent(in) :: diag(*), subdiag(*), e(*), ph(*), scale(*), wn(*)
      real(c_double), intent(out) :: G(*)
    end function
    ! the same without device allocation (static device scratch; no counterpart in the reference)
    integer(c_int) function edk_cf_eval_noalloc(ctx, nchain, ld, n, diag, subdiag, e, ph, scale, nw, wn, G) &
        bind(C, name="edk_cf_eval_noalloc")
      import :: c_int, c_ptr, c_int32_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: nchain, ld, nw
      integer(c_int32_t), intent(in) :: n(*)
      real(c_double), intent(in) :: diag(*), subdiag(*), e(*), ph(*), scale(*), wn(*)
      real(c_double), intent(out) :: G(*)
    end function

    ! ---- block Lanczos, batched chains, the solve driver ----
    integer(c_int) function edk_block_lanczos(h, opts, E, vecs, niter, converged) bind(C, name="edk_block_lanczos")
      import :: c_int, c_ptr, c_int32_t, c_double, edk_block_opts
      type(c_ptr), value :: h
      type(edk_block_opts), intent(in) :: opts
      real(c_double) :: E(*)
      type(c_ptr), value :: vecs
      integer(c_int32_t) :: niter, converged
    end function
    integer(c_int) function edk_green_batch(ctx, dtype, nchain, chains, nitergreen, nw, wn, cutoff_dynamic, &
        nout, G, mode, stats) bind(C, name="edk_green_batch")
      import :: c_int, c_ptr, c_int32_t, c_double, edk_chain, edk_batch_stats
      type(c_ptr), value :: ctx
      integer(c_int), value :: dtype
      integer(c_int32_t), value :: nchain, nitergreen, nw, nout, mode
      type(edk_chain), intent(in) :: chains(*)
      real(c_double), intent(in) :: wn(*)
      real(c_double), value :: cutoff_dynamic
      real(c_double) :: G(*)
      type(edk_batch_stats) :: stats
    end function
    integer(c_int) function edk_solve(ctx, m, o, r) bind(C, name="edk_solve")
      import :: c_int, c_ptr, edk_model, edk_solve_opts, edk_solve_result
      type(c_ptr), value :: ctx
      type(edk_model), intent(in) :: m
      type(edk_solve_opts), intent(in) :: o
      type(edk_solve_result), intent(inout) :: r
    end function
    integer(c_int) function edk_chiloc_set_kernel(plain) bind(C, name="edk_chiloc_set_kernel")
      import :: c_int
      integer(c_int), value :: plain
    end function
  end interface

  ! one sector Hamiltonian at a time, as H_class.f90 keeps sector_h (H_class.f90:11)
  type(c_ptr), save :: edk_ctx_handle = c_null_ptr, edk_h_handle = c_null_ptr

contains

  ! new_H(AIM, sector) for an (nup, ndn) sector: Ec/Eb/Vbc per spin, U, JJ from the AIM type
  subroutine edk_new_H(nc, nb, ec, eb, vbc, u, jj, jhund, cutoff, nup, ndn)
    integer, intent(in) :: nc, nb, nup, ndn
    real(c_double), intent(in), target :: ec(nc, nc, 2), eb(nb, nb, 2), vbc(nb, nc, 2), u(nc, nc), jj(nc, nc)
    real(c_double), intent(in) :: jhund, cutoff
    ! the C side reads row-major matrices: pass transposes of the Fortran arrays
    real(c_double), allocatable, target, save :: ec_t(:, :, :), eb_t(:, :, :), vbc_t(:, :, :), u_t(:, :), jj_t(:, :)
    type(edk_model) :: m
    integer :: s, ierr
    if (.not. c_associated(edk_ctx_handle)) then
      ierr = edk_ctx_create(0_c_int, c_null_ptr, edk_ctx_handle)
      if (ierr /= EDK_OK) stop 'edk_ctx_create failed'
    end if
    if (allocated(ec_t)) deallocate(ec_t, eb_t, vbc_t, u_t, jj_t)
    allocate(ec_t(nc, nc, 2), eb_t(nb, nb, 2), vbc_t(nc, nb, 2), u_t(nc, nc), jj_t(nc, nc))
    do s = 1, 2
      ec_t(:, :, s) = transpose(ec(:, :, s))
      eb_t(:, :, s) = transpose(eb(:, :, s))
      vbc_t(:, :, s) = transpose(vbc(:, :, s))
    end do
    u_t = transpose(u)
    jj_t = transpose(jj)
    m%nc = nc
    m%nb = nb
    m%ec = c_loc(ec_t)
    m%eb = c_loc(eb_t)
    m%vbc = c_loc(vbc_t)
    m%u = c_loc(u_t)
    m%jj = c_loc(jj_t)
    m%jhund = jhund
    m%cutoff_hamilt_param = cutoff
    if (c_associated(edk_h_handle)) ierr = edk_h_destroy(edk_h_handle)
    ierr = edk_h_create(edk_ctx_handle, m, int(nup, c_int), int(ndn, c_int), edk_h_handle)
    if (ierr /= EDK_OK) stop 'edk_h_create failed'
  end subroutine

  ! Hmult__ on host arrays (REAL(DBL) build of H_class.f90:109)
  subroutine edk_Hmult_real(n, vec_out, vec_in)
    integer, intent(in) :: n
    real(c_double), intent(out) :: vec_out(n)
    real(c_double), intent(in) :: vec_in(n)
    integer(c_int) :: ierr
    ierr = edk_hmult_host(edk_h_handle, EDK_F64, int(n, c_int64_t), vec_in, vec_out)
    if (ierr /= EDK_OK) stop 'edk_hmult_host failed'
  end subroutine

  subroutine edk_delete_H()
    integer(c_int) :: ierr
    if (c_associated(edk_h_handle)) ierr = edk_h_destroy(edk_h_handle)
    edk_h_handle = c_null_ptr
  end subroutine

end module edk_fortran
