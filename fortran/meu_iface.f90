! meu_iface.f90 -- ISO_C_BINDING interface of include/meu.h for the MEUMAPPS-SS
! Fortran driver (Multi_MEUMAPPS.f).  The driver keeps its set-up (Input.txt,
! ModGparams, ModInitials, ran_2) and its data_save writer; the body of its
! time loop (Multi_MEUMAPPS.f:548-1106) becomes one call of meu_run.
!
! Not compiled in the build image (it has no Fortran compiler); compile with
! any Fortran 2003 compiler:  gfortran -c meu_iface.f90
module meu_iface
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: MEU_MAX_VAR = 16, MEU_MAX_PH = 4, MEU_MAX_EL = 3
  integer(c_int), parameter :: MEU_MAX_GP = 2 * MEU_MAX_EL + 1
  integer(c_int), parameter :: MEU_MODEL_KKS = 0, MEU_MODEL_LANDAU = 1
  integer(c_int), parameter :: MEU_PREC_F64 = 0, MEU_PREC_F32 = 1
  integer(c_int), parameter :: MEU_ELAST_NONE = 0, MEU_ELAST_HOMOG = 1, MEU_ELAST_HETERO = 2

  ! mirror of struct meu_params (field order and kinds as in meu.h)
  type, bind(C) :: meu_params
    integer(c_int64_t) :: step, elastep0, noise_step
    integer(c_int32_t) :: nx, ny, nz, model, precision, nvar, numel, numph
    integer(c_int32_t) :: nvar_ph(MEU_MAX_PH)
    integer(c_int32_t) :: elastic, eig_coupling, el_min_iter, el_max_iter, clip_phi, diag_energy, flags
    real(c_double) :: dt, b_mob
    real(c_double) :: cmobs(MEU_MAX_EL)
    real(c_double) :: el_tol
    real(c_double) :: e_mean(6)
    real(c_double) :: grad_coeff(9, MEU_MAX_VAR)   ! grad_coeff(:,:,v) flattened column-major
    real(c_double) :: trans_ppt(6, MEU_MAX_VAR)
    real(c_double) :: cela(36, MEU_MAX_PH)         ! CEla(:,:,n) flattened column-major
    real(c_double) :: sela(36, MEU_MAX_PH)
    real(c_double) :: gparams(MEU_MAX_GP, MEU_MAX_PH)
    real(c_double) :: wellph(MEU_MAX_PH)
    real(c_double) :: lan_a, lan_b, lan_c, lan_d, lan_c1, lan_c2, kappa_c, cross_w
  end type meu_params

  ! mirror of struct meu_ran2_state (ran_2's SAVE variables)
  type, bind(C) :: meu_ran2_state
    integer(c_int32_t) :: idum, idum2, iy
    integer(c_int32_t) :: iv(32)
  end type meu_ran2_state

  ! mirror of struct meu_diag: one fort.98 / fort.99 line
  type, bind(C) :: meu_diag
    integer(c_int64_t) :: step
    integer(c_int32_t) :: el_iters, status
    real(c_double) :: fint, fw, fch, elen, etot
    real(c_double) :: glob_min, glob_max, phi_max, solid
    real(c_double) :: cmin, cmax, phimax, solid_now
    real(c_double) :: cavg(MEU_MAX_EL)
  end type meu_diag

  interface
    integer(c_int) function meu_create(params, handle) bind(C, name="meu_create")
      import :: c_int, c_ptr, meu_params
      type(meu_params), intent(in) :: params
      type(c_ptr), intent(out) :: handle
    end function
    integer(c_int) function meu_set_fields(h, cons, phi, u_state) bind(C, name="meu_set_fields")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, cons, phi, u_state
    end function
    integer(c_int) function meu_add_noise(h, incr) bind(C, name="meu_add_noise")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, incr
    end function
    integer(c_int) function meu_run(h, nsteps, diag) bind(C, name="meu_run")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: nsteps
      type(c_ptr), value :: diag
    end function
    ! meu_run with the Langevin noise drawn from the ran_2 state rng (type(meu_ran2_state))
    integer(c_int) function meu_run_noise(h, nsteps, rng, sd, diag) bind(C, name="meu_run_noise")
      import :: c_int, c_int32_t, c_ptr, c_double, meu_ran2_state
      type(c_ptr), value :: h, diag
      integer(c_int32_t), value :: nsteps
      type(meu_ran2_state), intent(inout) :: rng
      real(c_double), value :: sd
    end function
    ! n langevin(rng, sd) draws into out(1:n), the logarithms on up to `threads` host threads
    integer(c_int) function meu_langevin_fill(rng, sd, n, out, threads) bind(C, name="meu_langevin_fill")
      import :: c_int, c_int32_t, c_int64_t, c_double, meu_ran2_state
      type(meu_ran2_state), intent(inout) :: rng
      real(c_double), value :: sd
      integer(c_int64_t), value :: n
      real(c_double), intent(out) :: out(*)
      integer(c_int32_t), value :: threads
    end function
    integer(c_int) function meu_get_fields(h, cons, phi, el_en, u_state) bind(C, name="meu_get_fields")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, cons, phi, el_en, u_state
    end function
    integer(c_int64_t) function meu_get_step(h) bind(C, name="meu_get_step")
      import :: c_int64_t, c_ptr
      type(c_ptr), value :: h
    end function
    type(c_ptr) function meu_last_error(h) bind(C, name="meu_last_error")
      import :: c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function meu_destroy(h) bind(C, name="meu_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    ! dparams(5): dJ/dbeta (kappa_eta scale), dJ/dkappa_c, dJ/db_mob, dJ/dcmobs(1), dJ/dalpha (eigenstrain scale)
    integer(c_int) function meu_adjoint(h, nsteps, checkpoint_every, cons_target, phi_target, loss, dparams, dphi0) &
        bind(C, name="meu_adjoint")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: h, cons_target, phi_target, dparams, dphi0
      integer(c_int32_t), value :: nsteps, checkpoint_every
      real(c_double), intent(out) :: loss
    end function
    integer(c_int) function meu_schedule(h, out3) bind(C, name="meu_schedule")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), intent(out) :: out3(3)
    end function
    integer(c_int) function meu_set_schedule(h, in3) bind(C, name="meu_set_schedule")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), intent(in) :: in3(3)
    end function
    ! ensembles: params(n) decks stepped together (flags: MEU_ENS_AUTOTUNE = 1,
    ! MEU_ENS_PERSISTENT = 2: one persistent launch per run of steps, one order parameter each)
    integer(c_int) function meu_ensemble_create(n, params, flags, e) bind(C, name="meu_ensemble_create")
      import :: c_int, c_int32_t, c_ptr, meu_params
      integer(c_int32_t), value :: n, flags
      type(meu_params), intent(in) :: params(*)
      type(c_ptr), intent(out) :: e
    end function
    integer(c_int) function meu_ensemble_set_fields(e, member, cons, phi) bind(C, name="meu_ensemble_set_fields")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: e, cons, phi
      integer(c_int32_t), value :: member
    end function
    ! diag: NULL or n_members * nsteps rows, member-major
    integer(c_int) function meu_ensemble_run(e, nsteps, diag) bind(C, name="meu_ensemble_run")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: e, diag
      integer(c_int32_t), value :: nsteps
    end function
    integer(c_int) function meu_ensemble_get_fields(e, member, cons, phi, el_en) bind(C, name="meu_ensemble_get_fields")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: e, cons, phi, el_en
      integer(c_int32_t), value :: member
    end function
    integer(c_int) function meu_ensemble_destroy(e) bind(C, name="meu_ensemble_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: e
    end function
    ! one f_trans / inv_trans pair of host arrays (transform tests)
    integer(c_int) function meu_fft_roundtrip(nx, ny, nz, precision, in, spec_out, back_out) &
        bind(C, name="meu_fft_roundtrip")
      import :: c_int, c_int32_t, c_ptr
      integer(c_int32_t), value :: nx, ny, nz, precision
      type(c_ptr), value :: in, spec_out, back_out
    end function
    ! the same pair on the caller's device arrays with no device allocation, e.g. the
    ! c_loc of arrays inside "!$acc host_data use_device(...)".  The three arrays must
    ! be 16-byte aligned for MEU_PREC_F64 (8-byte for MEU_PREC_F32): an array section
    ! or an offset into a pool may not be; such calls return MEU_ERR_BADARG (100).
    integer(c_int) function meu_fft_roundtrip_noalloc(nx, ny, nz, precision, in_dev, spec_dev, back_dev) &
        bind(C, name="meu_fft_roundtrip_noalloc")
      import :: c_int, c_int32_t, c_ptr
      integer(c_int32_t), value :: nx, ny, nz, precision
      type(c_ptr), value :: in_dev, spec_dev, back_dev
    end function
    ! slab-decomposed f_trans / inv_trans over the MPI ranks (one GPU each) in place of
    ! P3DFFT: planes, then an all-to-all of nranks equal chunks (MPI_Alltoall on device
    ! buffers, or NCCL), then columns; device pointers, stream = c_null_ptr for the default
    integer(c_int) function meu_slab_fft_create(nx, ny, nz, nranks, rank, precision, h) &
        bind(C, name="meu_slab_fft_create")
      import :: c_int, c_int32_t, c_ptr
      integer(c_int32_t), value :: nx, ny, nz, nranks, rank, precision
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function meu_slab_fft_sizes(h, out4) bind(C, name="meu_slab_fft_sizes")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), intent(out) :: out4(4)
    end function
    integer(c_int) function meu_slab_fft_forward_planes(h, real_dev, send_dev, stream) &
        bind(C, name="meu_slab_fft_forward_planes")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, real_dev, send_dev, stream
    end function
    integer(c_int) function meu_slab_fft_forward_columns(h, kslab_dev, stream) &
        bind(C, name="meu_slab_fft_forward_columns")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, kslab_dev, stream
    end function
    integer(c_int) function meu_slab_fft_inverse_columns(h, kslab_dev, stream) &
        bind(C, name="meu_slab_fft_inverse_columns")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, kslab_dev, stream
    end function
    integer(c_int) function meu_slab_fft_inverse_planes(h, recv_dev, real_dev, stream) &
        bind(C, name="meu_slab_fft_inverse_planes")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, recv_dev, real_dev, stream
    end function
    integer(c_int) function meu_slab_fft_destroy(h) bind(C, name="meu_slab_fft_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
  end interface

contains

  ! Copy the ModGparams state (after the set-up of Multi_MEUMAPPS.f:153-417) into
  ! a meu_params block.  Arguments are the module variables of ModGparams.
  subroutine meu_fill_params(p, Nx, Ny, Nz, vartot, numel, numph, Nvar, step, elastep0, noise_step, &
                             t_step, b_mob, Cmobs, e_mean, grad_coeff, trans_ppt, CEla, SEla, Gparams, Wellph)
    type(meu_params), intent(out) :: p
    integer, intent(in) :: Nx, Ny, Nz, vartot, numel, numph, Nvar(numph), step, elastep0, noise_step
    real(8), intent(in) :: t_step, b_mob, Cmobs(numel), e_mean(6)
    real(8), intent(in) :: grad_coeff(3, 3, vartot), trans_ppt(6, vartot), CEla(6, 6, numph), SEla(6, 6, numph)
    real(8), intent(in) :: Gparams(2 * numel + 1, numph), Wellph(numph)
    integer :: v, n
    p%step = step; p%elastep0 = elastep0; p%noise_step = noise_step
    p%nx = Nx; p%ny = Ny; p%nz = Nz
    p%model = MEU_MODEL_KKS; p%precision = MEU_PREC_F64
    p%nvar = vartot; p%numel = numel; p%numph = numph
    p%nvar_ph = 0; p%nvar_ph(1:numph) = Nvar
    p%elastic = MEU_ELAST_HETERO; p%eig_coupling = 0
    p%el_min_iter = 4; p%el_max_iter = 10; p%clip_phi = 1; p%diag_energy = 1; p%flags = 0
    p%dt = t_step; p%b_mob = b_mob
    p%cmobs = 0; p%cmobs(1:numel) = Cmobs
    p%el_tol = 1.0d-7
    p%e_mean = e_mean
    p%grad_coeff = 0; p%trans_ppt = 0; p%cela = 0; p%sela = 0; p%gparams = 0; p%wellph = 0
    do v = 1, vartot
      p%grad_coeff(:, v) = reshape(grad_coeff(:, :, v), (/9/))
      p%trans_ppt(:, v) = trans_ppt(:, v)
    end do
    do n = 1, numph
      p%cela(:, n) = reshape(CEla(:, :, n), (/36/))
      p%sela(:, n) = reshape(SEla(:, :, n), (/36/))
      p%gparams(1:2 * numel + 1, n) = Gparams(:, n)
      p%wellph(n) = Wellph(n)
    end do
    p%lan_a = 0; p%lan_b = 0; p%lan_c = 0; p%lan_d = 0; p%lan_c1 = 0; p%lan_c2 = 0; p%kappa_c = 0; p%cross_w = 0
  end subroutine meu_fill_params

end module meu_iface
