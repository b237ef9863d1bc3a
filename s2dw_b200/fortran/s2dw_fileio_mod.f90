!------------------------------------------------------------------------------
! s2dw_fileio_mod -- drop-in replacement of the reference module of the same
! name (src/mod/s2dw_fileio_mod.f90): FITS and Matlab wavelet coefficient
! files, written and read by libs2dw_cuda (C ABI: include/s2dw_cuda.h,
! s2dwc_fileio_*), without CFITSIO.
!
! Same generic names, arguments and allocation behaviour: the readers
! allocate wav / wavdyn and scoeff; on a non-zero status every routine calls
! the reference's s2dw_error, which prints and halts.
!
! Build status: no Fortran compiler exists on the build machine, so this
! file has not been compiled there; the C entry points it binds are tested
! from Python/ctypes.
!------------------------------------------------------------------------------
module s2dw_fileio_mod

  use, intrinsic :: iso_c_binding
  use s2dw_types_mod
  use s2dw_error_mod
  use s2dw_core_mod

  implicit none

  private

  public :: &
       s2dw_fileio_matlab_wav_write, &
       s2dw_fileio_matlab_wav_read, &
       s2dw_fileio_fits_wav_write, &
       s2dw_fileio_fits_wav_read

  interface s2dw_fileio_matlab_wav_write
     module procedure matlab_write_static, matlab_write_dynamic
  end interface s2dw_fileio_matlab_wav_write

  interface s2dw_fileio_matlab_wav_read
     module procedure matlab_read_static, matlab_read_dynamic
  end interface s2dw_fileio_matlab_wav_read

  interface s2dw_fileio_fits_wav_write
     module procedure fits_write_static, fits_write_dynamic
  end interface s2dw_fileio_fits_wav_write

  interface s2dw_fileio_fits_wav_read
     module procedure fits_read_static, fits_read_dynamic
  end interface s2dw_fileio_fits_wav_read

  interface
     integer(c_int) function c_fits_write_dyn(ptrs, scoeff, J, B, N, bl_scoeff, alpha, filename, comment) &
          bind(C, name='s2dwc_fileio_fits_wav_write_dynamic')
       import :: c_int, c_double, c_double_complex, c_ptr, c_char
       type(c_ptr), intent(in) :: ptrs(*)
       complex(c_double_complex), intent(in) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
       character(kind=c_char), intent(in) :: filename(*), comment(*)
     end function c_fits_write_dyn

     integer(c_int) function c_fits_write_static(wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment) &
          bind(C, name='s2dwc_fileio_fits_wav_write_static')
       import :: c_int, c_double, c_double_complex, c_char
       real(c_double), intent(in) :: wav(*)
       complex(c_double_complex), intent(in) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
       character(kind=c_char), intent(in) :: filename(*), comment(*)
     end function c_fits_write_static

     integer(c_int) function c_fits_read_header(filename, J, B, N, bl_scoeff, alpha) &
          bind(C, name='s2dwc_fileio_fits_wav_read_header')
       import :: c_int, c_double, c_char
       character(kind=c_char), intent(in) :: filename(*)
       integer(c_int), intent(out) :: J, B, N, bl_scoeff
       real(c_double), intent(out) :: alpha
     end function c_fits_read_header

     integer(c_int) function c_fits_read_dyn(ptrs, scoeff, J, B, N, bl_scoeff, filename) &
          bind(C, name='s2dwc_fileio_fits_wav_read_dynamic')
       import :: c_int, c_double_complex, c_ptr, c_char
       type(c_ptr), intent(in) :: ptrs(*)
       complex(c_double_complex), intent(out) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       character(kind=c_char), intent(in) :: filename(*)
     end function c_fits_read_dyn

     integer(c_int) function c_fits_read_static(wav, scoeff, J, B, N, bl_scoeff, filename) &
          bind(C, name='s2dwc_fileio_fits_wav_read_static')
       import :: c_int, c_double, c_double_complex, c_char
       real(c_double), intent(out) :: wav(*)
       complex(c_double_complex), intent(out) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       character(kind=c_char), intent(in) :: filename(*)
     end function c_fits_read_static

     integer(c_int) function c_mat_write_dyn(ptrs, scoeff, J, B, N, bl_scoeff, alpha, filename, comment) &
          bind(C, name='s2dwc_fileio_matlab_wav_write_dynamic')
       import :: c_int, c_double, c_double_complex, c_ptr, c_char
       type(c_ptr), intent(in) :: ptrs(*)
       complex(c_double_complex), intent(in) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
       character(kind=c_char), intent(in) :: filename(*), comment(*)
     end function c_mat_write_dyn

     integer(c_int) function c_mat_write_static(wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment) &
          bind(C, name='s2dwc_fileio_matlab_wav_write_static')
       import :: c_int, c_double, c_double_complex, c_char
       real(c_double), intent(in) :: wav(*)
       complex(c_double_complex), intent(in) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
       character(kind=c_char), intent(in) :: filename(*), comment(*)
     end function c_mat_write_static

     integer(c_int) function c_mat_read_header(filename, J, B, N, bl_scoeff, alpha) &
          bind(C, name='s2dwc_fileio_matlab_wav_read_header')
       import :: c_int, c_double, c_char
       character(kind=c_char), intent(in) :: filename(*)
       integer(c_int), intent(out) :: J, B, N, bl_scoeff
       real(c_double), intent(out) :: alpha
     end function c_mat_read_header

     integer(c_int) function c_mat_read_dyn(ptrs, scoeff, J, B, N, bl_scoeff, filename) &
          bind(C, name='s2dwc_fileio_matlab_wav_read_dynamic')
       import :: c_int, c_double_complex, c_ptr, c_char
       type(c_ptr), intent(in) :: ptrs(*)
       complex(c_double_complex), intent(out) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       character(kind=c_char), intent(in) :: filename(*)
     end function c_mat_read_dyn

     integer(c_int) function c_mat_read_static(wav, scoeff, J, B, N, bl_scoeff, filename) &
          bind(C, name='s2dwc_fileio_matlab_wav_read_static')
       import :: c_int, c_double, c_double_complex, c_char
       real(c_double), intent(out) :: wav(*)
       complex(c_double_complex), intent(out) :: scoeff(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       character(kind=c_char), intent(in) :: filename(*)
     end function c_mat_read_static

     integer(c_int) function c_band_limits(jj, B, alpha, bl_hi, bl_lo) bind(C, name='s2dwc_band_limits')
       import :: c_int, c_double
       integer(c_int), value :: jj, B
       real(c_double), value :: alpha
       integer(c_int), intent(out) :: bl_hi, bl_lo
     end function c_band_limits
  end interface

contains

  subroutine check(status, proc)
    integer(c_int), intent(in) :: status
    character(len=*), intent(in) :: proc
    if (status /= 0) call s2dw_error(int(status), proc)
  end subroutine check

  function cstr(s) result(c)
    character(len=*), intent(in) :: s
    character(kind=c_char, len=len_trim(s)+1) :: c
    c = trim(s) // c_null_char
  end function cstr

  function ccomment(comment) result(c)
    character(len=*), intent(in), optional :: comment
    character(kind=c_char, len=:), allocatable :: c
    if (present(comment)) then
       c = trim(comment) // c_null_char
    else
       c = c_null_char  ! empty: no comment in the file
    end if
  end function ccomment

  ! per-scale pointers of wavdyn, allocating it first when `alloc`
  subroutine scale_ptrs(wavdyn, ptrs, J, B, N, alpha, alloc, proc)
    type(s2dw_wav_abg), allocatable, target, intent(inout) :: wavdyn(:)
    type(c_ptr), intent(out) :: ptrs(0:J)
    integer, intent(in) :: J, B, N
    real(dp), intent(in) :: alpha
    logical, intent(in) :: alloc
    character(len=*), intent(in) :: proc
    integer :: jj, fail
    integer(c_int) :: bl_hi, bl_lo
    if (alloc) then
       allocate(wavdyn(0:J), stat=fail)
       if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, proc)
    end if
    do jj = 0, J
       if (alloc) then
          call check(c_band_limits(jj, B, alpha, bl_hi, bl_lo), proc)
          allocate(wavdyn(jj)%coeff(0:2*bl_hi-2, 0:2*bl_hi-1, 0:N-1), stat=fail)
          if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, proc)
       end if
       ptrs(jj) = c_loc(wavdyn(jj)%coeff)
    end do
  end subroutine scale_ptrs

  ! ---- FITS ----------------------------------------------------------------

  subroutine fits_write_static(wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    real(dp), intent(in) :: wav(0:J, 0:2*B-2, 0:2*B-1, 0:N-1)
    complex(dpc), intent(in) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    character(len=*), intent(in) :: filename
    character(len=*), intent(in), optional :: comment
    call check(c_fits_write_static(wav, scoeff, J, B, N, bl_scoeff, alpha, cstr(filename), ccomment(comment)), &
         's2dw_fileio_fits_wav_write_static')
  end subroutine fits_write_static

  subroutine fits_write_dynamic(wavdyn, scoeff, J, B, N, bl_scoeff, alpha, filename, comment)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    type(s2dw_wav_abg), intent(inout), allocatable, target :: wavdyn(:)
    complex(dpc), intent(in) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    character(len=*), intent(in) :: filename
    character(len=*), intent(in), optional :: comment
    type(c_ptr) :: ptrs(0:J)
    call scale_ptrs(wavdyn, ptrs, J, B, N, alpha, .false., 's2dw_fileio_fits_wav_write_dynamic')
    call check(c_fits_write_dyn(ptrs, scoeff, J, B, N, bl_scoeff, alpha, cstr(filename), ccomment(comment)), &
         's2dw_fileio_fits_wav_write_dynamic')
  end subroutine fits_write_dynamic

  subroutine fits_read_static(wav, scoeff, J, B, N, bl_scoeff, alpha, filename)
    integer, intent(out) :: J, B, N, bl_scoeff
    real(dp), intent(out) :: alpha
    real(dp), allocatable, intent(out) :: wav(:,:,:,:)
    complex(dpc), allocatable, intent(out) :: scoeff(:,:)
    character(len=*), intent(in) :: filename
    integer :: fail
    call check(c_fits_read_header(cstr(filename), J, B, N, bl_scoeff, alpha), 's2dw_fileio_fits_wav_read_static')
    allocate(wav(0:J, 0:2*B-2, 0:2*B-1, 0:N-1), scoeff(0:bl_scoeff-1, 0:bl_scoeff-1), stat=fail)
    if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, 's2dw_fileio_fits_wav_read_static')
    call check(c_fits_read_static(wav, scoeff, J, B, N, bl_scoeff, cstr(filename)), &
         's2dw_fileio_fits_wav_read_static')
  end subroutine fits_read_static

  subroutine fits_read_dynamic(wavdyn, scoeff, J, B, N, bl_scoeff, alpha, filename)
    integer, intent(out) :: J, B, N, bl_scoeff
    real(dp), intent(out) :: alpha
    type(s2dw_wav_abg), intent(out), allocatable, target :: wavdyn(:)
    complex(dpc), allocatable, intent(out) :: scoeff(:,:)
    character(len=*), intent(in) :: filename
    type(c_ptr), allocatable :: ptrs(:)
    integer :: fail
    call check(c_fits_read_header(cstr(filename), J, B, N, bl_scoeff, alpha), 's2dw_fileio_fits_wav_read_dynamic')
    allocate(ptrs(0:J), scoeff(0:bl_scoeff-1, 0:bl_scoeff-1), stat=fail)
    if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, 's2dw_fileio_fits_wav_read_dynamic')
    call scale_ptrs(wavdyn, ptrs, J, B, N, alpha, .true., 's2dw_fileio_fits_wav_read_dynamic')
    call check(c_fits_read_dyn(ptrs, scoeff, J, B, N, bl_scoeff, cstr(filename)), &
         's2dw_fileio_fits_wav_read_dynamic')
  end subroutine fits_read_dynamic

  ! ---- Matlab --------------------------------------------------------------

  subroutine matlab_write_static(wav, scoeff, J, B, N, bl_scoeff, alpha, filename, comment)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    real(dp), intent(in) :: wav(0:J, 0:2*B-2, 0:2*B-1, 0:N-1)
    complex(dpc), intent(in) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    character(len=*), intent(in) :: filename
    character(len=*), intent(in), optional :: comment
    call check(c_mat_write_static(wav, scoeff, J, B, N, bl_scoeff, alpha, cstr(filename), ccomment(comment)), &
         's2dw_fileio_matlab_wav_write_static')
  end subroutine matlab_write_static

  subroutine matlab_write_dynamic(wavdyn, scoeff, J, B, N, bl_scoeff, alpha, filename, comment)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    type(s2dw_wav_abg), intent(inout), allocatable, target :: wavdyn(:)
    complex(dpc), intent(in) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    character(len=*), intent(in) :: filename
    character(len=*), intent(in), optional :: comment
    type(c_ptr) :: ptrs(0:J)
    call scale_ptrs(wavdyn, ptrs, J, B, N, alpha, .false., 's2dw_fileio_matlab_wav_write_dynamic')
    call check(c_mat_write_dyn(ptrs, scoeff, J, B, N, bl_scoeff, alpha, cstr(filename), ccomment(comment)), &
         's2dw_fileio_matlab_wav_write_dynamic')
  end subroutine matlab_write_dynamic

  subroutine matlab_read_static(wav, scoeff, J, B, N, bl_scoeff, alpha, filename)
    integer, intent(out) :: J, B, N, bl_scoeff
    real(dp), intent(out) :: alpha
    real(dp), allocatable, intent(out) :: wav(:,:,:,:)
    complex(dpc), allocatable, intent(out) :: scoeff(:,:)
    character(len=*), intent(in) :: filename
    integer :: fail
    call check(c_mat_read_header(cstr(filename), J, B, N, bl_scoeff, alpha), 's2dw_fileio_matlab_wav_read_static')
    allocate(wav(0:J, 0:2*B-2, 0:2*B-1, 0:N-1), scoeff(0:bl_scoeff-1, 0:bl_scoeff-1), stat=fail)
    if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, 's2dw_fileio_matlab_wav_read_static')
    call check(c_mat_read_static(wav, scoeff, J, B, N, bl_scoeff, cstr(filename)), &
         's2dw_fileio_matlab_wav_read_static')
  end subroutine matlab_read_static

  subroutine matlab_read_dynamic(wavdyn, scoeff, J, B, N, bl_scoeff, alpha, filename)
    integer, intent(out) :: J, B, N, bl_scoeff
    real(dp), intent(out) :: alpha
    type(s2dw_wav_abg), intent(out), allocatable, target :: wavdyn(:)
    complex(dpc), allocatable, intent(out) :: scoeff(:,:)
    character(len=*), intent(in) :: filename
    type(c_ptr), allocatable :: ptrs(:)
    integer :: fail
    call check(c_mat_read_header(cstr(filename), J, B, N, bl_scoeff, alpha), 's2dw_fileio_matlab_wav_read_dynamic')
    allocate(ptrs(0:J), scoeff(0:bl_scoeff-1, 0:bl_scoeff-1), stat=fail)
    if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, 's2dw_fileio_matlab_wav_read_dynamic')
    call scale_ptrs(wavdyn, ptrs, J, B, N, alpha, .true., 's2dw_fileio_matlab_wav_read_dynamic')
    call check(c_mat_read_dyn(ptrs, scoeff, J, B, N, bl_scoeff, cstr(filename)), &
         's2dw_fileio_matlab_wav_read_dynamic')
  end subroutine matlab_read_dynamic

end module s2dw_fileio_mod
