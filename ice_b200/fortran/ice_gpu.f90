!> Fortran binding of the B200 solve stage (include/ice_gpu.h), for ICE's driver.
!>
!> The types are interoperable copies of the C structures; the procedures bind the C entry points.
!> The driver calls ice_gpu_create/set_block/set_records/set_gas/upload_state after setup_freeze
!> (driver/Wrap_Setup.f90:121), ice_gpu_step in place of Explicit_Step (driver/Wrap_Solve.f90:26),
!> and ice_gpu_download_state before Write_Solution (driver/Wrap_Postprocess.f90:120-196).
!> This file is source only here: it compiles wherever a Fortran 2008 compiler exists.
module ice_gpu
  use, intrinsic :: iso_c_binding
  implicit none
  private

  integer(c_int32_t), parameter, public :: ICE_GPU_MAX_FAMILIES = 4, ICE_GPU_NCOND_MAX = 12, ICE_GPU_NEP = 8
  integer(c_int32_t), parameter, public :: ICE_GPU_REC_INTS = 15, ICE_GPU_REC_REALS = 8
  integer(c_int),     parameter, public :: ICE_GPU_OK = 0, ICE_GPU_EINVAL = 1, ICE_GPU_ECUDA = 2, &
                                           ICE_GPU_ESTATE = 3, ICE_GPU_ENOMEM = 4, ICE_GPU_ENOTREADY = 5, &
                                           ICE_GPU_EEXCH = 6
  !> the kinds of a split run's exchanges (ice_gpu_set_halo, the exchange hook)
  integer(c_int32_t), parameter, public :: ICE_GPU_HALO_CELLS = 0, ICE_GPU_HALO_BETA = 1, ICE_GPU_HALO_FLUX = 2, &
                                           ICE_GPU_HALO_DT = 3, ICE_GPU_HALO_NORM = 4

  type, bind(C), public :: ice_gpu_family_t
    integer(c_int32_t) :: closure, riemann, nfrozen
    integer(c_int32_t) :: frozen(ICE_GPU_NCOND_MAX)
    real(c_double)     :: rho_al, cs_al, lv_al, emiss
    integer(c_int32_t) :: evap, intf, liq, boil
    real(c_double)     :: ep(ICE_GPU_NEP)
  end type ice_gpu_family_t

  type, bind(C), public :: ice_gpu_params_t
    integer(c_int32_t) :: nfam, ndir, nrk, time_accurate
    real(c_double)     :: cfl, dt_max, tau_factor
    integer(c_int32_t) :: cfl_ramp_iter, limiter, shock_detector, irs
    real(c_double)     :: irs_beta
    integer(c_int32_t) :: coupled, drag, heat, blow, precision, itermax, sol_diter, shell_diter, res_diter, no_realize
    real(c_double)     :: time_threshold, res_threshold, sol_dtime
    type(ice_gpu_family_t) :: fam(ICE_GPU_MAX_FAMILIES)
  end type ice_gpu_params_t

  type, bind(C), public :: ice_gpu_step_out_t
    real(c_double)     :: dtglobal, time
    integer(c_int32_t) :: iter, todo, status, have_norm
    integer(c_int64_t) :: nfloored
    real(c_double)     :: residual(5)
    real(c_double)     :: device_ms
    integer(c_int64_t) :: nrealized
  end type ice_gpu_step_out_t

  public :: ice_gpu_create, ice_gpu_set_block, ice_gpu_set_records, ice_gpu_set_chimera, ice_gpu_set_gas, &
            ice_gpu_set_imports, ice_gpu_set_exchange, ice_gpu_exchange_rate, ice_gpu_step_host, &
            ice_gpu_upload_state, &
            ice_gpu_download_state, ice_gpu_set_time, ice_gpu_set_res_reference, ice_gpu_get_res_reference, &
            ice_gpu_step, ice_gpu_residual_norm, ice_gpu_update_params, &
            ice_gpu_last_error, ice_gpu_destroy, ice_gpu_pair_connections, &
            ice_gpu_set_partition, ice_gpu_set_halo, ice_gpu_set_exchange_hook

  interface
    integer(c_int) function ice_gpu_create(params, nblocks, dims, ctx) bind(C, name='ice_gpu_create')
      import :: c_int, c_int32_t, c_ptr, ice_gpu_params_t
      type(ice_gpu_params_t), intent(in) :: params
      integer(c_int32_t), value          :: nblocks
      integer(c_int32_t), intent(in)     :: dims(*)
      type(c_ptr), intent(out)           :: ctx
    end function

    integer(c_int) function ice_gpu_set_block(ctx, b, face1, face2, face3, vol, dl, M) bind(C, name='ice_gpu_set_block')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value        :: ctx
      integer(c_int32_t), value :: b
      type(c_ptr), value        :: face1, face2, face3, vol, dl, M     ! c_loc(blk%dir(d)%f), ...
    end function

    integer(c_int) function ice_gpu_set_records(ctx, nrec, rec, inlet) bind(C, name='ice_gpu_set_records')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value             :: ctx
      integer(c_int32_t), value      :: nrec
      integer(c_int32_t), intent(in) :: rec(*)
      real(c_double), intent(in)     :: inlet(*)
    end function

    integer(c_int) function ice_gpu_set_imports(ctx, b, p, imports) bind(C, name='ice_gpu_set_imports')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value         :: ctx
      integer(c_int32_t), value  :: b, p
      real(c_double), intent(in) :: imports(*)
    end function

    integer(c_int) function ice_gpu_set_exchange(ctx, on) bind(C, name='ice_gpu_set_exchange')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value        :: ctx
      integer(c_int32_t), value :: on
    end function

    integer(c_int) function ice_gpu_exchange_rate(ctx, b, p, x) bind(C, name='ice_gpu_exchange_rate')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value          :: ctx
      integer(c_int32_t), value   :: b, p
      real(c_double), intent(out) :: x(*)
    end function

    integer(c_int) function ice_gpu_step_host(ctx, nsteps, prim_in, prim_out, out) bind(C, name='ice_gpu_step_host')
      import :: c_int, c_int32_t, c_ptr, ice_gpu_step_out_t
      type(c_ptr), value              :: ctx
      integer(c_int32_t), value       :: nsteps
      type(c_ptr), intent(in)         :: prim_in(*)
      type(c_ptr), intent(in)         :: prim_out(*)
      type(ice_gpu_step_out_t), intent(out) :: out
    end function

    integer(c_int) function ice_gpu_set_chimera(ctx, nrec, nchi, donor, weight) bind(C, name='ice_gpu_set_chimera')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value             :: ctx
      integer(c_int32_t), value      :: nrec
      integer(c_int32_t), intent(in) :: nchi(*)
      integer(c_int32_t), intent(in) :: donor(*)
      real(c_double), intent(in)     :: weight(*)
    end function

    integer(c_int) function ice_gpu_set_gas(ctx, b, prim5, R, gam, k, mu) bind(C, name='ice_gpu_set_gas')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value         :: ctx
      integer(c_int32_t), value  :: b
      real(c_double), intent(in) :: prim5(*), R(*), gam(*), k(*), mu(*)
    end function

    integer(c_int) function ice_gpu_upload_state(ctx, b, p, prim, inj) bind(C, name='ice_gpu_upload_state')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value         :: ctx
      integer(c_int32_t), value  :: b, p
      real(c_double), intent(in) :: prim(*)
      type(c_ptr), value         :: inj            ! c_null_ptr, or c_loc of a uint8 copy of inj
    end function

    integer(c_int) function ice_gpu_download_state(ctx, b, p, prim) bind(C, name='ice_gpu_download_state')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value          :: ctx
      integer(c_int32_t), value   :: b, p
      real(c_double), intent(out) :: prim(*)
    end function

    integer(c_int) function ice_gpu_set_time(ctx, time, iter, iter_from_call) bind(C, name='ice_gpu_set_time')
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value        :: ctx
      real(c_double), value     :: time
      integer(c_int32_t), value :: iter, iter_from_call
    end function

    integer(c_int) function ice_gpu_set_res_reference(ctx, ref) bind(C, name='ice_gpu_set_res_reference')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value    :: ctx
      real(c_double), value :: ref
    end function

    integer(c_int) function ice_gpu_get_res_reference(ctx, ref) bind(C, name='ice_gpu_get_res_reference')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value          :: ctx
      real(c_double), intent(out) :: ref
    end function

    integer(c_int) function ice_gpu_step(ctx, nsteps, out) bind(C, name='ice_gpu_step')
      import :: c_int, c_int32_t, c_ptr, ice_gpu_step_out_t
      type(c_ptr), value                    :: ctx
      integer(c_int32_t), value             :: nsteps
      type(ice_gpu_step_out_t), intent(out) :: out
    end function

    integer(c_int) function ice_gpu_residual_norm(ctx, total, fam) bind(C, name='ice_gpu_residual_norm')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value          :: ctx
      real(c_double), intent(out) :: total(5), fam(*)
    end function

    integer(c_int) function ice_gpu_update_params(ctx, params) bind(C, name='ice_gpu_update_params')
      import :: c_int, c_ptr, ice_gpu_params_t
      type(c_ptr), value                 :: ctx
      type(ice_gpu_params_t), intent(in) :: params
    end function

    integer(c_int) function ice_gpu_last_error(ctx, buf, buflen) bind(C, name='ice_gpu_last_error')
      import :: c_int, c_int32_t, c_char, c_ptr
      type(c_ptr), value                :: ctx
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int32_t), value         :: buflen
    end function

    integer(c_int) function ice_gpu_destroy(ctx) bind(C, name='ice_gpu_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function

    integer(c_int) function ice_gpu_pair_connections(nblocks, dims, ngroups, nrec, rec, err, errlen) &
        bind(C, name='ice_gpu_pair_connections')
      import :: c_int, c_int32_t, c_char
      integer(c_int32_t), value            :: nblocks, ngroups, nrec, errlen
      integer(c_int32_t), intent(in)       :: dims(*)
      integer(c_int32_t), intent(inout)    :: rec(*)
      character(kind=c_char), intent(out)  :: err(*)
    end function

    !> The block split over MPI ranks (one GPU each): the blocks this rank steps, the exchange lists,
    !> and the hook, a bind(C) function of the driver that moves the buffers with MPI (its interface:
    !> integer(c_int32_t) function hook(user, kind, family, nsend, send, nrecv, recv) bind(C), with
    !> user a c_ptr value, kind and family c_int32_t values, nsend and nrecv c_int64_t values, send
    !> and recv real(c_double) arrays).
    integer(c_int) function ice_gpu_set_partition(ctx, owned) bind(C, name='ice_gpu_set_partition')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value             :: ctx
      integer(c_int32_t), intent(in) :: owned(*)
    end function

    integer(c_int) function ice_gpu_set_halo(ctx, kind, p, nsend, send, nrecv, recv) bind(C, name='ice_gpu_set_halo')
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value             :: ctx
      integer(c_int32_t), value      :: kind, p, nsend, nrecv
      integer(c_int32_t), intent(in) :: send(*), recv(*)
    end function

    integer(c_int) function ice_gpu_set_exchange_hook(ctx, fn, user) bind(C, name='ice_gpu_set_exchange_hook')
      import :: c_int, c_ptr, c_funptr
      type(c_ptr), value    :: ctx
      type(c_funptr), value :: fn
      type(c_ptr), value    :: user
    end function
  end interface

end module ice_gpu
