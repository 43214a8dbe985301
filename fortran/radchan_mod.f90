! radchan_mod.f90 -- Fortran 2003 (iso_c_binding) interface to libradchan.so.
!
! Two ways to call the solver from the channel DNS:
!
!  1. unchanged: the DNS keeps `call mc_gpu(T, zstart, rank)` and
!     `call get_results(Q, sigma, rank)` (src/dns/channel.f:239-256); the
!     compiler resolves them to the symbols mc_gpu_ / get_results_ that the
!     library exports with the reference's arguments and array layouts
!     (src/montecarlo/mc_gpu_noint.cu:660, :876).  The library reads
!     RADCHAN_PARAM_H, RADCHAN_NARROWBAND_H and RADCHAN_PROPERTIES from the
!     environment on the first call, or takes rc_legacy_configure() below.
!
!  2. explicit: use this module, build an rc_params from the same headers,
!     create a context once, and solve / collect every radStep steps.
!
! Array layouts: T(0:imax+1, 0:jmax+1, 0:kmax+1) and Q, sigma
! (0:imax+1, 0:jmax+1, 0:kmax/p_col+1), real(4), Fortran order.
module radchan_mod
  use iso_c_binding
  implicit none
  private

  integer(c_int), parameter, public :: RC_OK = 0
  integer(c_int), parameter, public :: RC_MAX_LEVELS = 9

  ! mirror of struct rc_params (include/radchan.h)
  type, bind(C), public :: rc_params
    integer(c_int) :: imax, jmax, kmax
    real(c_float) :: Lx, Ly, Lz
    real(c_double) :: fact_mesh
    integer(c_int) :: nVar
    integer(c_int) :: photmax
    real(c_double) :: chanHeight
    integer(c_int) :: grid_num
    integer(c_int) :: maxi(RC_MAX_LEVELS), maxj(RC_MAX_LEVELS), maxk(RC_MAX_LEVELS)
    integer(c_int) :: maxs(RC_MAX_LEVELS)
    integer(c_int) :: num_gpu, p_col
    integer(c_int) :: num_streams, blockdim, nblocks
    integer(c_int) :: srt, grey, calcwalls, random, floatpoint
    real(c_float) :: eps(6), Tw(6)
    integer(c_int) :: adiabw, adiabe
    real(c_double) :: stefan
    real(c_float) :: toll, tollS
    integer(c_int) :: bd(6)
    integer(c_int) :: grey_nT, grey_nB
    real(c_float) :: abscoeff, Tmins, wvmax
    integer(c_int) :: nT, nQ, nB
    integer(c_int64_t) :: seed
  end type rc_params

  ! mirror of struct rc_tables (borrowed pointers into a table set)
  type, bind(C), public :: rc_tables
    integer(c_int) :: nT, nB, nQ
    type(c_ptr) :: Tnb, kP, wvl, wvr, wvc, kavg, kq, prob, probg, wq
  end type rc_tables

  ! mirror of struct rc_scattering (borrowed pointers into a particle set)
  type, bind(C), public :: rc_scattering
    integer(c_int) :: nB, nQ, nA
    type(c_ptr) :: ksca, kabs, theta, phase_cdf
  end type rc_scattering

  ! mirror of struct rc_dns_coupling: what the DNS does with a finished
  ! solve (channel.f:249-266, fixvar.f:16-43 and :179-242)
  type, bind(C), public :: rc_dns_coupling
    real(c_double) :: Tin, Height, underrelax, stefan
    integer(c_int) :: nTemp
    type(c_ptr) :: Tnb, kP        ! c_loc of real(8) arrays(nTemp); kP already times Height
    integer(c_int) :: jstart, jend
  end type rc_dns_coupling

  public :: mc_gpu, get_results
  public :: rc_params_from_headers, rc_create, rc_set_tables, rc_tables_read_dir, rc_tables_view
  public :: rc_tables_free, rc_solve_async, rc_collect, rc_destroy, rc_last_error
  public :: rc_legacy_configure, rc_dns_source, rc_legacy_source, c_string
  public :: rc_scattering_read_dir, rc_scattering_view, rc_scattering_free, rc_set_scattering
  public :: rc_slab_range, rc_slab_unique_id, rc_slab_comm_create, rc_slab_solve, rc_slab_last_error
  public :: rc_slab_comm_destroy

  interface
    ! the reference's entry points (mc_gpu_noint.cu:660, :876)
    subroutine mc_gpu(T, zstart, rank) bind(C, name="mc_gpu_")
      import :: c_float, c_int
      real(c_float), intent(in) :: T(*)
      integer(c_int), intent(in) :: zstart, rank
    end subroutine mc_gpu

    subroutine get_results(Q, sigma, rank) bind(C, name="get_results_")
      import :: c_float, c_int
      real(c_float), intent(inout) :: Q(*), sigma(*)
      integer(c_int), intent(in) :: rank
    end subroutine get_results

    integer(c_int) function rc_params_from_headers(param_h, narrowband_h, p) bind(C, name="rc_params_from_headers")
      import :: c_char, c_int, rc_params
      character(kind=c_char), intent(in) :: param_h(*), narrowband_h(*)
      type(rc_params), intent(out) :: p
    end function rc_params_from_headers

    integer(c_int) function rc_create(p, device, ctx) bind(C, name="rc_create")
      import :: c_int, c_ptr, rc_params
      type(rc_params), intent(in) :: p
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: ctx
    end function rc_create

    integer(c_int) function rc_tables_read_dir(dir, nT, nB, nQ, ts) bind(C, name="rc_tables_read_dir")
      import :: c_char, c_int, c_ptr
      character(kind=c_char), intent(in) :: dir(*)
      integer(c_int), value :: nT, nB, nQ
      type(c_ptr), intent(out) :: ts
    end function rc_tables_read_dir

    integer(c_int) function rc_tables_view(ts, view) bind(C, name="rc_tables_view")
      import :: c_int, c_ptr, rc_tables
      type(c_ptr), value :: ts
      type(rc_tables), intent(out) :: view
    end function rc_tables_view

    subroutine rc_tables_free(ts) bind(C, name="rc_tables_free")
      import :: c_ptr
      type(c_ptr), value :: ts
    end subroutine rc_tables_free

    integer(c_int) function rc_set_tables(ctx, t) bind(C, name="rc_set_tables")
      import :: c_int, c_ptr, rc_tables
      type(c_ptr), value :: ctx
      type(rc_tables), intent(in) :: t
    end function rc_set_tables

    ! particles of the table generator's files (particles/NarrBand%d.txt,
    ! particles/prob_scatt.txt) for the context's later solves
    integer(c_int) function rc_scattering_read_dir(dir, nB, nQ, ps) bind(C, name="rc_scattering_read_dir")
      import :: c_char, c_int, c_ptr
      character(kind=c_char), intent(in) :: dir(*)
      integer(c_int), value :: nB, nQ
      type(c_ptr), intent(out) :: ps
    end function rc_scattering_read_dir

    integer(c_int) function rc_scattering_view(ps, view) bind(C, name="rc_scattering_view")
      import :: c_int, c_ptr, rc_scattering
      type(c_ptr), value :: ps
      type(rc_scattering), intent(out) :: view
    end function rc_scattering_view

    subroutine rc_scattering_free(ps) bind(C, name="rc_scattering_free")
      import :: c_ptr
      type(c_ptr), value :: ps
    end subroutine rc_scattering_free

    integer(c_int) function rc_set_scattering(ctx, s) bind(C, name="rc_set_scattering")
      import :: c_int, c_ptr, rc_scattering
      type(c_ptr), value :: ctx
      type(rc_scattering), intent(in) :: s
    end function rc_set_scattering

    integer(c_int) function rc_solve_async(ctx, T, zstart, ticket) bind(C, name="rc_solve_async")
      import :: c_float, c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      real(c_float), intent(in) :: T(*)
      integer(c_int), value :: zstart
      integer(c_int32_t), intent(out) :: ticket
    end function rc_solve_async

    ! q64, var64, qw64, vw64: c_loc of real(8) arrays, or c_null_ptr
    integer(c_int) function rc_collect(ctx, ticket, Q, sigma, q64, var64, qw64, vw64) bind(C, name="rc_collect")
      import :: c_float, c_int, c_int32_t, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ticket
      real(c_float), intent(inout) :: Q(*), sigma(*)
      type(c_ptr), value :: q64, var64, qw64, vw64
    end function rc_collect

    integer(c_int) function rc_destroy(ctx) bind(C, name="rc_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function rc_destroy

    integer(c_int) function rc_last_error(ctx, buf, len) bind(C, name="rc_last_error")
      import :: c_char, c_int, c_ptr, c_size_t
      type(c_ptr), value :: ctx
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_size_t), value :: len
    end function rc_last_error

    ! one solve over several GPUs by z slabs (NCCL inside the library):
    ! rank 0 makes the group id, MPI_Bcast hands its 128 bytes to every
    ! rank, each rank joins with its GPU and solves with a context created
    ! with p_col = nranks; every rank receives the whole solution
    integer(c_int) function rc_slab_range(kmax, nranks, rank, kloc, zstart) bind(C, name="rc_slab_range")
      import :: c_int
      integer(c_int), value :: kmax, nranks, rank
      integer(c_int), intent(out) :: kloc, zstart
    end function rc_slab_range

    integer(c_int) function rc_slab_unique_id(id) bind(C, name="rc_slab_unique_id")
      import :: c_int, c_int8_t
      integer(c_int8_t), intent(out) :: id(128)
    end function rc_slab_unique_id

    integer(c_int) function rc_slab_comm_create(device, nranks, rank, id, timeout_s, comm) &
        bind(C, name="rc_slab_comm_create")
      import :: c_double, c_int, c_int8_t, c_ptr
      integer(c_int), value :: device, nranks, rank
      integer(c_int8_t), intent(in) :: id(128)
      real(c_double), value :: timeout_s
      type(c_ptr), intent(out) :: comm
    end function rc_slab_comm_create

    ! T (whole field, real(4)), q64, var64 (real(8), imax*jmax*kmax), qw64,
    ! vw64 (real(8), 2*jmax*kmax, or c_null_ptr): c_loc of host or device arrays
    integer(c_int) function rc_slab_solve(comm, ctx, T, q64, var64, qw64, vw64) bind(C, name="rc_slab_solve")
      import :: c_int, c_ptr
      type(c_ptr), value :: comm, ctx, T, q64, var64, qw64, vw64
    end function rc_slab_solve

    integer(c_int) function rc_slab_last_error(comm, buf, len) bind(C, name="rc_slab_last_error")
      import :: c_char, c_int, c_ptr, c_size_t
      type(c_ptr), value :: comm
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_size_t), value :: len
    end function rc_slab_last_error

    integer(c_int) function rc_slab_comm_destroy(comm) bind(C, name="rc_slab_comm_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: comm
    end function rc_slab_comm_destroy

    ! tables: c_null_ptr in grey mode, else c_loc of an rc_tables view
    integer(c_int) function rc_legacy_configure(p, tables) bind(C, name="rc_legacy_configure")
      import :: c_int, c_ptr, rc_params
      type(rc_params), intent(in) :: p
      type(c_ptr), value :: tables
    end function rc_legacy_configure

    ! GET_RESULTS + fix_rad + fix_kappa + the Gnew loop for a ticket:
    ! T1(0:i1, 0:jn+1, 0:kloc+1) real(8) nondimensional; Qnew, Varnew, Knew,
    ! Gnew(0:i1, jn, kloc) real(8); n_clamped: c_loc of an integer(8) or c_null_ptr
    integer(c_int) function rc_dns_source(ctx, ticket, cfg, T1, Qnew, Varnew, Knew, Gnew, n_clamped) &
        bind(C, name="rc_dns_source")
      import :: c_double, c_int, c_int32_t, c_ptr, rc_dns_coupling
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: ticket
      type(rc_dns_coupling), intent(in) :: cfg
      real(c_double), intent(in) :: T1(*)
      real(c_double), intent(inout) :: Qnew(*), Varnew(*), Knew(*), Gnew(*)
      type(c_ptr), value :: n_clamped
    end function rc_dns_source

    ! the same for the pending mc_gpu launch (replaces channel.f:252-266)
    integer(c_int) function rc_legacy_source(cfg, T1, Qnew, Varnew, Knew, Gnew, n_clamped) &
        bind(C, name="rc_legacy_source")
      import :: c_double, c_int, c_ptr, rc_dns_coupling
      type(rc_dns_coupling), intent(in) :: cfg
      real(c_double), intent(in) :: T1(*)
      real(c_double), intent(inout) :: Qnew(*), Varnew(*), Knew(*), Gnew(*)
      type(c_ptr), value :: n_clamped
    end function rc_legacy_source
  end interface

contains

  ! NUL-terminated copy of a Fortran string for the char* arguments
  function c_string(s) result(cs)
    character(len=*), intent(in) :: s
    character(kind=c_char) :: cs(len_trim(s) + 1)
    integer :: i
    do i = 1, len_trim(s)
      cs(i) = s(i:i)
    end do
    cs(len_trim(s) + 1) = c_null_char
  end function c_string

end module radchan_mod
