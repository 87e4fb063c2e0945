!=============================================================================80
!
!> ISO_C_BINDING interface to libfvm3d.so (include/fvm3d.h).
!
!  The Fortran solver binds the B200 explicit residual-and-update path the
!  way it binds METIS (src/base/interface_metis5_c.f90): bind(c) interfaces
!  with plain pointers, sizes and integer status codes. fvm_config_t mirrors
!  struct fvm_config field by field; the scheme ids are the integers of
!  TypeDefs%Scheme (src/defs/type_defs_scheme.f90:12-35).
!
!  Arrays cross as they are: q is the real-range view of
!  ClassBlockData%get_q(), shape (ni,nj,nk,5); a connection range is
!  range(2,3) = (lo/hi, axis), the memory order of C's int64_t range[3][2].
!
!=============================================================================80

module fvm3d_c

  use, intrinsic :: iso_c_binding

  implicit none

  private

  public :: fvm_config_t
  public :: fvm_config_default, fvm_abi_version, fvm_create, fvm_destroy
  public :: fvm_add_block, fvm_set_boundary, fvm_connect
  public :: fvm_set_state, fvm_get_state, fvm_set_states, fvm_get_states, fvm_get_primitive, fvm_get_rhs
  public :: fvm_step, fvm_run, fvm_get_time, fvm_last_error
  public :: fvm_residual_norms, fvm_residual_norms_noalloc
  public :: fvm_server_config_t, fvm_connection_t, fvm_request_t
  public :: fvm_server_config_default, fvm_server_create, fvm_case_submit, fvm_poll, fvm_wait
  public :: fvm_fetch_state, fvm_release, fvm_server_stats, fvm_server_last_error, fvm_server_destroy
  public :: FVM_REQ_QUEUED, FVM_REQ_RUNNING, FVM_REQ_DONE, FVM_REQ_FAILED
  public :: FVM_OK, FVM_BC_TRANSMISSIVE, FVM_BC_PERIODIC, FVM_BC_CONNECTED
  public :: FVM_DT_FIXED, FVM_DT_CFL, FVM_DT_CFL_LOCAL
  public :: FVM_PREC_FP64_EXACT, FVM_PREC_FP64, FVM_PREC_FP32_FLUX

  integer(c_int), parameter :: FVM_OK = 0
  integer(c_int), parameter :: FVM_BC_TRANSMISSIVE = 0, FVM_BC_PERIODIC = 1, FVM_BC_CONNECTED = 2
  integer(c_int32_t), parameter :: FVM_DT_FIXED = 0, FVM_DT_CFL = 1, FVM_DT_CFL_LOCAL = 2
  integer(c_int32_t), parameter :: FVM_PREC_FP64_EXACT = 0, FVM_PREC_FP64 = 1, FVM_PREC_FP32_FLUX = 2
  integer(c_int), parameter :: FVM_REQ_QUEUED = 0, FVM_REQ_RUNNING = 1, FVM_REQ_DONE = 2, FVM_REQ_FAILED = 3

  type, bind(c) :: fvm_config_t
    integer(c_int32_t) :: struct_size
    integer(c_int32_t) :: idimension
    integer(c_int32_t) :: equation
    integer(c_int32_t) :: reconstruct
    integer(c_int32_t) :: limiter
    integer(c_int32_t) :: flux_split
    integer(c_int32_t) :: time_scheme
    integer(c_int32_t) :: rk_stages
    integer(c_int32_t) :: timestep_set
    integer(c_int32_t) :: compat
    integer(c_int32_t) :: precision
    integer(c_int32_t) :: store_rhs
    real(c_double)     :: kappa
    real(c_double)     :: entropy_fix
    real(c_double)     :: gamma
    real(c_double)     :: dt
    real(c_double)     :: cfl
    real(c_double)     :: mu
    real(c_double)     :: prandtl
  end type fvm_config_t

  ! struct fvm_server_config / fvm_connection / fvm_request (serving)
  type, bind(c) :: fvm_server_config_t
    integer(c_int32_t) :: struct_size
    integer(c_int32_t) :: chunk_steps
    integer(c_int64_t) :: budget_cells
    integer(c_int64_t) :: max_active_cells
    integer(c_int32_t) :: max_queued
    integer(c_int32_t) :: pad_
  end type fvm_server_config_t

  type, bind(c) :: fvm_connection_t
    integer(c_int32_t) :: blk, donor
    integer(c_int64_t) :: range(2, 3)
    integer(c_int64_t) :: donor_range(2, 3)
    integer(c_int32_t) :: donor_type(3)
    integer(c_int32_t) :: pad_
  end type fvm_connection_t

  ! nvert / dr: c_loc of (3, nblocks) arrays; q: c_loc of an array of
  ! nblocks c_ptr, each c_loc(get_q()) of one block; bc: c_loc of (3, nbc)
  type, bind(c) :: fvm_request_t
    integer(c_int32_t) :: struct_size
    integer(c_int32_t) :: nblocks
    type(c_ptr)        :: cfg
    type(c_ptr)        :: nvert
    type(c_ptr)        :: dr
    type(c_ptr)        :: q
    integer(c_int32_t) :: nbc, nconn
    type(c_ptr)        :: bc
    type(c_ptr)        :: conn
    integer(c_int64_t) :: steps
  end type fvm_request_t

  interface

    integer(c_int) function fvm_config_default(cfg) bind(c, name="fvm_config_default")
      import :: c_int, fvm_config_t
      type(fvm_config_t), intent(out) :: cfg
    end function fvm_config_default

    integer(c_int) function fvm_abi_version() bind(c, name="fvm_abi_version")
      import :: c_int
    end function fvm_abi_version

    integer(c_int) function fvm_create(cfg, ctx) bind(c, name="fvm_create")
      import :: c_int, c_ptr, fvm_config_t
      type(fvm_config_t), intent(in) :: cfg
      type(c_ptr), intent(out) :: ctx
    end function fvm_create

    integer(c_int) function fvm_destroy(ctx) bind(c, name="fvm_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function fvm_destroy

    integer(c_int) function fvm_add_block(ctx, nvert, dr, blk) bind(c, name="fvm_add_block")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int64_t), intent(in) :: nvert(3)
      real(c_double), intent(in) :: dr(3)
      integer(c_int), intent(out) :: blk
    end function fvm_add_block

    integer(c_int) function fvm_set_boundary(ctx, blk, region, kind) bind(c, name="fvm_set_boundary")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, region, kind
    end function fvm_set_boundary

    integer(c_int) function fvm_connect(ctx, blk, range, donor, donor_range, donor_type) &
        bind(c, name="fvm_connect")
      import :: c_int, c_ptr, c_int64_t, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, donor
      integer(c_int64_t), intent(in) :: range(2,3), donor_range(2,3)
      integer(c_int32_t), intent(in) :: donor_type(3)
    end function fvm_connect

    integer(c_int) function fvm_set_state(ctx, blk, q) bind(c, name="fvm_set_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
      real(c_double), intent(in) :: q(*)
    end function fvm_set_state

    integer(c_int) function fvm_get_state(ctx, blk, q) bind(c, name="fvm_get_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
      real(c_double), intent(out) :: q(*)
    end function fvm_get_state

    ! several blocks in one call: blk(1:n) block ids, q(1:n) = c_loc of each
    ! block's get_q() array; the copies of consecutive blocks overlap
    integer(c_int) function fvm_set_states(ctx, n, blk, q) bind(c, name="fvm_set_states")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      integer(c_int), intent(in) :: blk(*)
      type(c_ptr), intent(in) :: q(*)
    end function fvm_set_states

    integer(c_int) function fvm_get_states(ctx, n, blk, q) bind(c, name="fvm_get_states")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      integer(c_int), intent(in) :: blk(*)
      type(c_ptr), intent(in) :: q(*)
    end function fvm_get_states

    integer(c_int) function fvm_get_primitive(ctx, blk, p) bind(c, name="fvm_get_primitive")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
      real(c_double), intent(out) :: p(*)
    end function fvm_get_primitive

    integer(c_int) function fvm_get_rhs(ctx, blk, rhs) bind(c, name="fvm_get_rhs")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
      real(c_double), intent(out) :: rhs(*)
    end function fvm_get_rhs

    integer(c_int) function fvm_step(ctx, nsteps, t, res_abs, res_rel) bind(c, name="fvm_step")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nsteps
      real(c_double), intent(out) :: t
      real(c_double), intent(out) :: res_abs(6), res_rel(6)
    end function fvm_step

    integer(c_int) function fvm_run(ctx, max_step, total_time, absolute_residual, relative_residual, &
        steps_done, reason) bind(c, name="fvm_run")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: ctx
      integer(c_int64_t), value :: max_step
      real(c_double), value :: total_time, absolute_residual, relative_residual
      integer(c_int64_t), intent(out) :: steps_done
      integer(c_int), intent(out) :: reason
    end function fvm_run

    integer(c_int) function fvm_get_time(ctx, t, dt, step) bind(c, name="fvm_get_time")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: t, dt
      integer(c_int64_t), intent(out) :: step
    end function fvm_get_time

    integer(c_int) function fvm_last_error(ctx, buf, n) bind(c, name="fvm_last_error")
      import :: c_int, c_ptr, c_char, c_size_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_size_t), value :: n
    end function fvm_last_error

    integer(c_int) function fvm_residual_norms(rhs_dev, nvert, res_dev, stream) &
        bind(c, name="fvm_residual_norms")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: rhs_dev, res_dev, stream
      integer(c_int64_t), intent(in) :: nvert(3)
    end function fvm_residual_norms

    ! the same without any device allocation, for hosts whose GPU memory all
    ! belongs to their own pool (limits in include/fvm3d.h)
    integer(c_int) function fvm_residual_norms_noalloc(rhs_dev, nvert, res_dev, stream) &
        bind(c, name="fvm_residual_norms_noalloc")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: rhs_dev, res_dev, stream
      integer(c_int64_t), intent(in) :: nvert(3)
    end function fvm_residual_norms_noalloc

    ! ---- serving: many cases queued and run with continuous batching
    integer(c_int) function fvm_server_config_default(cfg) bind(c, name="fvm_server_config_default")
      import :: c_int, fvm_server_config_t
      type(fvm_server_config_t), intent(out) :: cfg
    end function fvm_server_config_default

    integer(c_int) function fvm_server_create(cfg, srv) bind(c, name="fvm_server_create")
      import :: c_int, c_ptr, fvm_server_config_t
      type(fvm_server_config_t), intent(in) :: cfg
      type(c_ptr), intent(out) :: srv
    end function fvm_server_create

    integer(c_int) function fvm_case_submit(srv, req, request_id) bind(c, name="fvm_case_submit")
      import :: c_int, c_ptr, c_int64_t, fvm_request_t
      type(c_ptr), value :: srv
      type(fvm_request_t), intent(in) :: req
      integer(c_int64_t), intent(out) :: request_id
    end function fvm_case_submit

    integer(c_int) function fvm_poll(srv, request_id, state, steps_done, t, latency_s, status) &
        bind(c, name="fvm_poll")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: srv
      integer(c_int64_t), value :: request_id
      integer(c_int), intent(out) :: state, status
      integer(c_int64_t), intent(out) :: steps_done
      real(c_double), intent(out) :: t, latency_s
    end function fvm_poll

    integer(c_int) function fvm_wait(srv, request_id, timeout_s, state) bind(c, name="fvm_wait")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: srv
      integer(c_int64_t), value :: request_id
      real(c_double), value :: timeout_s
      integer(c_int), intent(out) :: state
    end function fvm_wait

    integer(c_int) function fvm_fetch_state(srv, request_id, blk, q) bind(c, name="fvm_fetch_state")
      import :: c_int, c_ptr, c_int64_t, c_double
      type(c_ptr), value :: srv
      integer(c_int64_t), value :: request_id
      integer(c_int), value :: blk
      real(c_double), intent(out) :: q(*)
    end function fvm_fetch_state

    integer(c_int) function fvm_release(srv, request_id) bind(c, name="fvm_release")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: srv
      integer(c_int64_t), value :: request_id
    end function fvm_release

    integer(c_int) function fvm_server_stats(srv, active_cells, peak_active_cells, running, queued) &
        bind(c, name="fvm_server_stats")
      import :: c_int, c_ptr, c_int64_t
      type(c_ptr), value :: srv
      integer(c_int64_t), intent(out) :: active_cells, peak_active_cells
      integer(c_int), intent(out) :: running, queued
    end function fvm_server_stats

    integer(c_int) function fvm_server_last_error(srv, buf, n) bind(c, name="fvm_server_last_error")
      import :: c_int, c_ptr, c_char, c_size_t
      type(c_ptr), value :: srv
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_size_t), value :: n
    end function fvm_server_last_error

    integer(c_int) function fvm_server_destroy(srv) bind(c, name="fvm_server_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: srv
    end function fvm_server_destroy

  end interface

end module fvm3d_c
