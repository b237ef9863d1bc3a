!------------------------------------------------------------------------------
! s2dw_core_mod -- drop-in replacement of the reference module of the same
! name (src/mod/s2dw_core_mod.f90) whose transforms run on the GPU through
! libs2dw_cuda (C ABI: include/s2dw_cuda.h).
!
! Same public names, arguments, array shapes and halting behaviour: every
! routine calls the C entry point and, on a non-zero status, reports it with
! the reference's s2dw_error (which prints and halts for fatal codes).
! Fortran callers (s2dw_test, s2dw_analysis, s2dw_synthesis, s2dw_wstats,
! s2dw_maskgen, ...) only relink:
!
!   gfortran -c s2dw_core_mod.f90 -I<s2dw include dir>
!   ... -L<dir of libs2dw_cuda.so> -ls2dw_cuda
!
! Build status: no Fortran compiler exists on the build machine, so this
! file has not been compiled there; the C entry points it binds are tested
! from Python/ctypes.
!------------------------------------------------------------------------------
module s2dw_core_mod

  use, intrinsic :: iso_c_binding
  use s2dw_types_mod
  use s2dw_error_mod

  implicit none

  private

  public :: &
       s2dw_core_init_kernels, &
       s2dw_core_init_directionality, &
       s2dw_core_comp_Jmax, &
       s2dw_core_admiss, &
       s2dw_core_analysis_flm2wav, &
       s2dw_core_analysis_flm2wav_dynamic, &
       s2dw_core_synthesis_wav2flm, &
       s2dw_core_synthesis_wav2flm_dynamic, &
       s2dw_core_free_wavdyn, &
       s2dw_core_assimilate_int

  !! Per-scale wavelet coefficients (reference: s2dw_core_mod.f90:56-58).
  type, public :: s2dw_wav_abg
     real(dp), allocatable :: coeff(:,:,:)
  end type s2dw_wav_abg

  interface
     integer(c_int) function c_init_kernels(K_gamma, Phi2, bl_scoeff, J, B, alpha) &
          bind(C, name='s2dwc_init_kernels')
       import :: c_int, c_double
       real(c_double), intent(out) :: K_gamma(*), Phi2(*)
       integer(c_int), intent(out) :: bl_scoeff
       integer(c_int), value :: J, B
       real(c_double), value :: alpha
     end function c_init_kernels

     integer(c_int) function c_init_directionality(Slm, B, N) &
          bind(C, name='s2dwc_init_directionality')
       import :: c_int, c_double_complex
       complex(c_double_complex), intent(out) :: Slm(*)
       integer(c_int), value :: B, N
     end function c_init_directionality

     integer(c_int) function c_comp_jmax(B, alpha) bind(C, name='s2dwc_comp_jmax')
       import :: c_int, c_double
       integer(c_int), value :: B
       real(c_double), value :: alpha
     end function c_comp_jmax

     integer(c_int) function c_assimilate_int(x, y) bind(C, name='s2dwc_assimilate_int')
       import :: c_int, c_double
       real(c_double), value :: x
       integer(c_int) :: y
     end function c_assimilate_int

     integer(c_int) function c_admiss(admiss, K_gamma, Phi2, B, J, pass) &
          bind(C, name='s2dwc_admiss')
       import :: c_int, c_double
       real(c_double), intent(out) :: admiss(*)
       real(c_double), intent(in) :: K_gamma(*), Phi2(*)
       integer(c_int), value :: B, J
       integer(c_int), intent(out) :: pass
     end function c_admiss

     integer(c_int) function c_analysis(wav, scoeff, flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha) &
          bind(C, name='s2dwc_analysis_flm2wav')
       import :: c_int, c_double, c_double_complex
       real(c_double), intent(inout) :: wav(*)
       real(c_double), intent(in) :: K_gamma(*)
       complex(c_double_complex), intent(out) :: scoeff(*)
       complex(c_double_complex), intent(in) :: flm(*), Slm(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
     end function c_analysis

     integer(c_int) function c_analysis_dyn(wav_scales, scoeff, flm, K_gamma, Slm, J, B, N, &
          bl_scoeff, alpha) bind(C, name='s2dwc_analysis_flm2wav_dynamic')
       import :: c_int, c_double, c_double_complex, c_ptr
       type(c_ptr), intent(in) :: wav_scales(*)
       real(c_double), intent(in) :: K_gamma(*)
       complex(c_double_complex), intent(out) :: scoeff(*)
       complex(c_double_complex), intent(in) :: flm(*), Slm(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
     end function c_analysis_dyn

     integer(c_int) function c_synthesis(flm, wav, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, &
          alpha) bind(C, name='s2dwc_synthesis_wav2flm')
       import :: c_int, c_double, c_double_complex
       complex(c_double_complex), intent(out) :: flm(*)
       complex(c_double_complex), intent(in) :: scoeff(*), Slm(*)
       real(c_double), intent(in) :: wav(*), K_gamma(*), Phi2(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
     end function c_synthesis

     integer(c_int) function c_synthesis_dyn(flm, wav_scales, scoeff, K_gamma, Phi2, Slm, J, B, N, &
          bl_scoeff, alpha) bind(C, name='s2dwc_synthesis_wav2flm_dynamic')
       import :: c_int, c_double, c_double_complex, c_ptr
       complex(c_double_complex), intent(out) :: flm(*)
       complex(c_double_complex), intent(in) :: scoeff(*), Slm(*)
       type(c_ptr), intent(in) :: wav_scales(*)
       real(c_double), intent(in) :: K_gamma(*), Phi2(*)
       integer(c_int), value :: J, B, N, bl_scoeff
       real(c_double), value :: alpha
     end function c_synthesis_dyn

     integer(c_int) function c_band_limits(jj, B, alpha, bl_hi, bl_lo) &
          bind(C, name='s2dwc_band_limits')
       import :: c_int, c_double
       integer(c_int), value :: jj, B
       real(c_double), value :: alpha
       integer(c_int) :: bl_hi, bl_lo
     end function c_band_limits
  end interface

contains

  subroutine check(status, proc)
    integer(c_int), intent(in) :: status
    character(len=*), intent(in) :: proc
    ! Codes 0..14 are the reference's S2DW_ERROR_*; 15 (CUDA runtime
    ! error) is reported as an initialisation failure.
    if (status /= 0) then
       if (status <= 14) then
          call s2dw_error(int(status), proc)
       else
          call s2dw_error(S2DW_ERROR_INIT_FAIL, proc, comment_add='CUDA runtime error')
       end if
    end if
  end subroutine check

  subroutine s2dw_core_init_kernels(K_gamma, Phi2, bl_scoeff, J, B, alpha)
    integer, intent(in) :: J, B
    real(dp), intent(in) :: alpha
    real(dp), intent(out) :: K_gamma(0:J,0:B-1)
    real(dp), intent(out) :: Phi2(0:B-1)
    integer, intent(out) :: bl_scoeff
    integer(c_int) :: bs
    call check(c_init_kernels(K_gamma, Phi2, bs, J, B, alpha), 's2dw_core_init_kernels')
    bl_scoeff = bs
  end subroutine s2dw_core_init_kernels

  subroutine s2dw_core_init_directionality(Slm, B, N)
    integer, intent(in) :: B, N
    complex(dpc), intent(out) :: Slm(0:B-1,0:N-1)
    call check(c_init_directionality(Slm, B, N), 's2dw_core_init_directionality')
  end subroutine s2dw_core_init_directionality

  function s2dw_core_comp_Jmax(B, alpha) result(J_max)
    integer, intent(in) :: B
    real(dp), intent(in) :: alpha
    integer :: J_max
    J_max = c_comp_jmax(B, alpha)
  end function s2dw_core_comp_Jmax

  function s2dw_core_assimilate_int(x, y) result(assimilated)
    real(dp), intent(in) :: x
    integer, intent(out) :: y
    logical :: assimilated
    integer(c_int) :: yy
    assimilated = c_assimilate_int(x, yy) /= 0
    y = yy
  end function s2dw_core_assimilate_int

  function s2dw_core_admiss(admiss, K_gamma, Phi2, B, J) result(pass)
    integer, intent(in) :: J, B
    real(dp), intent(in) :: K_gamma(0:J,0:B-1)
    real(dp), intent(in) :: Phi2(0:B-1)
    real(dp), intent(out) :: admiss(0:B-1)
    logical :: pass
    integer(c_int) :: ok
    call check(c_admiss(admiss, K_gamma, Phi2, B, J, ok), 's2dw_core_admiss')
    pass = ok /= 0
  end function s2dw_core_admiss

  subroutine s2dw_core_analysis_flm2wav(wav, scoeff, flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    real(dp), intent(out) :: wav(0:J, 0:2*B-2, 0:2*B-1, 0:N-1)
    complex(dpc), intent(out) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    complex(dpc), intent(in) :: flm(0:B-1, 0:B-1)
    real(dp), intent(in) :: K_gamma(0:J, 0:B-1)
    complex(dpc), intent(in) :: Slm(0:B-1, 0:N-1)
    call check(c_analysis(wav, scoeff, flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha), &
         's2dw_core_analysis_flm2wav')
  end subroutine s2dw_core_analysis_flm2wav

  subroutine s2dw_core_analysis_flm2wav_dynamic(wavdyn, scoeff, flm, K_gamma, Slm, J, B, N, &
       bl_scoeff, alpha)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    type(s2dw_wav_abg), intent(out), allocatable, target :: wavdyn(:)
    complex(dpc), intent(out) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    complex(dpc), intent(in) :: flm(0:B-1, 0:B-1)
    real(dp), intent(in) :: K_gamma(0:J, 0:B-1)
    complex(dpc), intent(in) :: Slm(0:B-1, 0:N-1)
    type(c_ptr) :: ptrs(0:J)
    integer :: jj, fail
    integer(c_int) :: bl_hi, bl_lo
    ! allocation as at s2dw_core_mod.f90:599 and :746
    allocate(wavdyn(0:J), stat=fail)
    if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, 's2dw_core_analysis_flm2wav_dynamic')
    do jj = 0, J
       call check(c_band_limits(jj, B, alpha, bl_hi, bl_lo), 's2dw_core_analysis_flm2wav_dynamic')
       allocate(wavdyn(jj)%coeff(0:2*bl_hi-2, 0:2*bl_hi-1, 0:N-1), stat=fail)
       if (fail /= 0) call s2dw_error(S2DW_ERROR_MEM_ALLOC_FAIL, 's2dw_core_analysis_flm2wav_dynamic')
       ptrs(jj) = c_loc(wavdyn(jj)%coeff)
    end do
    call check(c_analysis_dyn(ptrs, scoeff, flm, K_gamma, Slm, J, B, N, bl_scoeff, alpha), &
         's2dw_core_analysis_flm2wav_dynamic')
  end subroutine s2dw_core_analysis_flm2wav_dynamic

  subroutine s2dw_core_synthesis_wav2flm(flm, wav, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, alpha)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    real(dp), intent(in) :: wav(0:J, 0:2*B-2, 0:2*B-1, 0:N-1)
    complex(dpc), intent(in) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    complex(dpc), intent(out) :: flm(0:B-1, 0:B-1)
    real(dp), intent(in) :: K_gamma(0:J, 0:B-1)
    real(dp), intent(in) :: Phi2(0:B-1)
    complex(dpc), intent(in) :: Slm(0:B-1, 0:N-1)
    call check(c_synthesis(flm, wav, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, alpha), &
         's2dw_core_synthesis_wav2flm')
  end subroutine s2dw_core_synthesis_wav2flm

  subroutine s2dw_core_synthesis_wav2flm_dynamic(flm, wavdyn, scoeff, K_gamma, Phi2, Slm, J, B, N, &
       bl_scoeff, alpha)
    integer, intent(in) :: J, B, N, bl_scoeff
    real(dp), intent(in) :: alpha
    type(s2dw_wav_abg), intent(inout), allocatable, target :: wavdyn(:)
    complex(dpc), intent(in) :: scoeff(0:bl_scoeff-1, 0:bl_scoeff-1)
    complex(dpc), intent(out) :: flm(0:B-1, 0:B-1)
    real(dp), intent(in) :: K_gamma(0:J, 0:B-1)
    real(dp), intent(in) :: Phi2(0:B-1)
    complex(dpc), intent(in) :: Slm(0:B-1, 0:N-1)
    type(c_ptr) :: ptrs(0:J)
    integer :: jj
    do jj = 0, J
       ptrs(jj) = c_loc(wavdyn(jj)%coeff)
    end do
    call check(c_synthesis_dyn(flm, ptrs, scoeff, K_gamma, Phi2, Slm, J, B, N, bl_scoeff, alpha), &
         's2dw_core_synthesis_wav2flm_dynamic')
    ! the reference destroys and frees the wavelet coefficients
    ! (s2dw_core_mod.f90:1130, :1264)
    call s2dw_core_free_wavdyn(wavdyn)
  end subroutine s2dw_core_synthesis_wav2flm_dynamic

  subroutine s2dw_core_free_wavdyn(wavdyn)
    type(s2dw_wav_abg), intent(inout), allocatable :: wavdyn(:)
    integer :: jj
    do jj = 0, size(wavdyn) - 1
       if (allocated(wavdyn(jj)%coeff)) deallocate(wavdyn(jj)%coeff)
    end do
    deallocate(wavdyn)
  end subroutine s2dw_core_free_wavdyn

end module s2dw_core_mod
