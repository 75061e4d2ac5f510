! yspec_gpu.f90 -- Fortran 2003 (ISO_C_BINDING) interface to the C-ABI of
! include/yspec_gpu.h, for a yspec host that keeps the reference's Fortran
! (yspec.f90 with module_model and module_spline) and hands the hot path,
! yspec.f90:250-486, to the B200 engine.
!
! Compile beside the reference's sources and link the engine:
!     gfortran -c yspec_gpu.f90
!     gfortran ... yspec.f90 yspec_gpu.o -L<repo>/yspec_b200/lib -lyspec_b200
! The derived types mirror the C structs field by field (bind(C) keeps the
! C layout); arrays are passed by address, scalars by value where the C
! prototype takes a value.  complex(dpc) arrays map to interleaved
! (re, im) doubles, so they can be passed directly as complex(c_double_complex).
module yspec_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: YSG_OK = 0, YSG_ERR_ARG = 1, YSG_ERR_CUDA = 2, &
       YSG_ERR_NO_MODEL = 3, YSG_ERR_NO_SPECTRA = 4, YSG_ERR_DEVICE_WAIT = 5, &
       YSG_ERR_NO_DEVICE = 6, YSG_ERR_LIMIT = 7, YSG_ERR_UNSUPPORTED = 8

  ! module_model.f90:118-160 after read_model: pointers to nknot doubles each;
  ! val/cs: rho, acon, ccon, fcon, lcon, ncon, kappa, mu, qkappa, qmu, grav,
  ! xlam, xa2 and their spline second derivatives
  type, bind(C) :: ysg_model
     integer(c_int) :: nknot, nic, noc, nsl, ocean, fic
     real(c_double) :: tref, pibigg, fre_norm
     type(c_ptr)    :: r
     type(c_ptr)    :: val(13), cs(13)
     type(c_ptr)    :: alpha, beta
  end type ysg_model

  ! one event's spectral problem (yspec.f90:176-261, normalised)
  type, bind(C) :: ysg_event
     integer(c_int) :: lmin, lmax, nw, is, ir, ats, grav, out, cor, nr, jofs, jstride
     real(c_double) :: wmin, dw, ep, rs, rr, mm(6)
     type(c_ptr)    :: delta, azst
  end type ysg_event

  ! the time-series stage (module_fourier.f90:362-397 outputs, yspec.f90:432-486)
  type, bind(C) :: ysg_time
     integer(c_int) :: nt, i1, i2, nr
     real(c_double) :: df, dt, ep, tout, f11, f12, f21, f22, t_norm, amp_norm
     type(c_ptr)    :: azep
  end type ysg_time

  interface
     integer(c_int) function ysg_create(h, device) bind(C, name="ysg_create")
       import :: c_int, c_ptr
       type(c_ptr), intent(out) :: h
       integer(c_int), value :: device
     end function ysg_create

     subroutine ysg_destroy(h) bind(C, name="ysg_destroy")
       import :: c_ptr
       type(c_ptr), value :: h
     end subroutine ysg_destroy

     integer(c_int) function ysg_model_upload(h, m) bind(C, name="ysg_model_upload")
       import :: c_int, c_ptr, ysg_model
       type(c_ptr), value :: h
       type(ysg_model), intent(in) :: m
     end function ysg_model_upload

     ! yspec.f90:250-486: out(nout, 4, nr) = t, Z, N, E
     integer(c_int) function ysg_event_run(h, ev, tm, out, nout) bind(C, name="ysg_event_run")
       import :: c_int, c_ptr, c_double, ysg_event, ysg_time
       type(c_ptr), value :: h
       type(ysg_event), intent(in) :: ev
       type(ysg_time), intent(in) :: tm
       real(c_double), intent(out) :: out(*)
       integer(c_int), intent(out) :: nout
     end function ysg_event_run

     ! yspec.f90:250-426: ur, ut, up(nw, nr)
     integer(c_int) function ysg_event_spectra(h, ev, ur, ut, up) bind(C, name="ysg_event_spectra")
       import :: c_int, c_ptr, c_double_complex, ysg_event
       type(c_ptr), value :: h
       type(ysg_event), intent(in) :: ev
       complex(c_double_complex), intent(out) :: ur(*), ut(*), up(*)
     end function ysg_event_spectra

     ! yspec.f90:432-486 on the last spectra
     integer(c_int) function ysg_event_traces(h, tm, out, nout) bind(C, name="ysg_event_traces")
       import :: c_int, c_ptr, c_double, ysg_time
       type(c_ptr), value :: h
       type(ysg_time), intent(in) :: tm
       real(c_double), intent(out) :: out(*)
       integer(c_int), intent(out) :: nout
     end function ysg_event_traces

     integer(c_int) function ysg_trace_rows(tm) bind(C, name="ysg_trace_rows")
       import :: c_int, ysg_time
       type(ysg_time), intent(in) :: tm
     end function ysg_trace_rows

     ! several events as one batch: outs(e) = c_loc of event e's out array
     integer(c_int) function ysg_batch_run(h, nev, evs, tms, outs, nouts) &
          bind(C, name="ysg_batch_run")
       import :: c_int, c_ptr, ysg_event, ysg_time
       type(c_ptr), value :: h
       integer(c_int), value :: nev
       type(ysg_event), intent(in) :: evs(*)
       type(ysg_time), intent(in) :: tms(*)
       type(c_ptr), intent(in) :: outs(*)
       integer(c_int), intent(out) :: nouts(*)
     end function ysg_batch_run

     ! potential traces: out(nout, 2, nr) = t, potential; tm%amp_norm the
     ! potential's normalisation for the output type
     integer(c_int) function ysg_event_potential(h, ev, tm, out, nout) &
          bind(C, name="ysg_event_potential")
       import :: c_int, c_ptr, c_double, ysg_event, ysg_time
       type(c_ptr), value :: h
       type(ysg_event), intent(in) :: ev
       type(ysg_time), intent(in) :: tm
       real(c_double), intent(out) :: out(*)
       integer(c_int), intent(out) :: nout
     end function ysg_event_potential

     ! dL/dval(p, i), dL/dcs(p, i) of L = sum gout * traces (reverse mode):
     ! gout(nout, 4, nr) as ysg_event_run's out; gval, gcs (nknot, 13)
     integer(c_int) function ysg_event_gradient(h, ev, tm, gout, gval, gcs) &
          bind(C, name="ysg_event_gradient")
       import :: c_int, c_ptr, c_double, ysg_event, ysg_time
       type(c_ptr), value :: h
       type(ysg_event), intent(in) :: ev
       type(ysg_time), intent(in) :: tm
       real(c_double), intent(in) :: gout(*)
       real(c_double), intent(out) :: gval(*), gcs(*)
     end function ysg_event_gradient

     ! 0 plain, 1 batched persistent (default), 2 tangent-linear
     integer(c_int) function ysg_set_solver(h, which) bind(C, name="ysg_set_solver")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: which
     end function ysg_set_solver

     ! stage times of the last run (ms): Legendre, solve, l-sum, time series
     integer(c_int) function ysg_last_timings(h, ms) bind(C, name="ysg_last_timings")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       real(c_float), intent(out) :: ms(4)
     end function ysg_last_timings

     ! message of a status (the reference's stop text where one exists)
     type(c_ptr) function ysg_status_string(status) bind(C, name="ysg_status_string")
       import :: c_ptr, c_int
       integer(c_int), value :: status
     end function ysg_status_string

     type(c_ptr) function ysg_last_cuda_error() bind(C, name="ysg_last_cuda_error")
       import :: c_ptr
     end function ysg_last_cuda_error
  end interface

contains

  ! The NUL-terminated C string behind p as a Fortran string.
  function ysg_c_string(p) result(s)
    type(c_ptr), intent(in) :: p
    character(len=:), allocatable :: s
    character(kind=c_char), pointer :: c(:)
    integer :: n
    interface
       integer(c_size_t) function c_strlen(q) bind(C, name="strlen")
         import :: c_ptr, c_size_t
         type(c_ptr), value :: q
       end function c_strlen
    end interface
    if (.not. c_associated(p)) then
       s = ''
       return
    end if
    n = int(c_strlen(p))
    call c_f_pointer(p, c, [n])
    allocate(character(len=n) :: s)
    s = transfer(c(1:n), s)
  end function ysg_c_string

end module yspec_gpu
