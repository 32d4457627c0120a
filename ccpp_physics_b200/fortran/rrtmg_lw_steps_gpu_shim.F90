!> \file rrtmg_lw_steps_gpu_shim.F90
!! Drop-in module rrtmg_lw_post for a CCPP host: the public
!! rrtmg_lw_post_run keeps the dummy arguments of
!! physics/Radiation/RRTMG/rrtmg_lw_post.F90:13-34 and forwards to
!! rrtmg_lw_gpu_post (include/rrtmg_lw_gpu.h) through ISO_C_BINDING, host
!! memory, synchronous.  Build it in place of rrtmg_lw_post.F90.  Arrays are
!! passed by address; sfcflw_type records are four contiguous reals, the
!! layout the C ABI expects.
module rrtmg_lw_steps_gpu_c
  use iso_c_binding
  implicit none
  private
  public :: c_lw_exec, c_lw_post_args, c_rrtmg_lw_gpu_post

  type, bind(c) :: c_lw_exec
    integer(c_int32_t) :: precision, memory
    type(c_ptr) :: stream = c_null_ptr
    integer(c_int32_t) :: sync, reserved
    type(c_ptr) :: kernel_ms = c_null_ptr
  end type

  type, bind(c) :: c_lw_post_args
    integer(c_int32_t) :: im, levs, ltp, lm, kd, lslwr, lwhtr
    type(c_ptr) :: tsfa = c_null_ptr, htlwc = c_null_ptr, htlw0 = c_null_ptr, sfcflw = c_null_ptr
    type(c_ptr) :: tsflw = c_null_ptr, sfcdlw = c_null_ptr, htrlw = c_null_ptr, lwhc = c_null_ptr
  end type

  interface
    integer(c_int) function c_rrtmg_lw_gpu_post(args, exec, errmsg, errmsg_len) bind(c, name="rrtmg_lw_gpu_post")
      import :: c_lw_post_args, c_lw_exec, c_int, c_char, c_int32_t
      type(c_lw_post_args), intent(in) :: args
      type(c_lw_exec), intent(in) :: exec
      character(kind=c_char), dimension(*), intent(out) :: errmsg
      integer(c_int32_t), value :: errmsg_len
    end function
  end interface
end module rrtmg_lw_steps_gpu_c


module rrtmg_lw_post
  use iso_c_binding
  use machine, only: kind_phys
  use module_radlw_parameters, only: sfcflw_type
  use rrtmg_lw_steps_gpu_c
  implicit none
  private
  public :: rrtmg_lw_post_run

contains

  !> rrtmg_lw_post_run (rrtmg_lw_post.F90:13-15): same dummy arguments.
  subroutine rrtmg_lw_post_run(im, levs, ltp, lm, kd, lslwr, lwhtr, tsfa, htlwc, htlw0, sfcflw, tsflw, sfcdlw, &
                               htrlw, lwhc, errmsg, errflg)
    integer, intent(in) :: im, levs, ltp, lm, kd
    logical, intent(in) :: lslwr, lwhtr
    real(kind=kind_phys), dimension(im), intent(in), target :: tsfa
    real(kind=kind_phys), dimension(im, lm+ltp), intent(in), target :: htlwc, htlw0
    type(sfcflw_type), dimension(im), intent(in), target :: sfcflw
    real(kind=kind_phys), dimension(im), intent(inout), target :: tsflw, sfcdlw
    real(kind=kind_phys), dimension(im, levs), intent(inout), target :: htrlw, lwhc
    character(len=*), intent(out) :: errmsg
    integer, intent(out) :: errflg
    type(c_lw_post_args) :: a
    type(c_lw_exec) :: x
    character(kind=c_char) :: cmsg(512)
    integer :: i

    errmsg = ''; errflg = 0
    if (.not. lslwr .or. im <= 0) return               ! rrtmg_lw_post.F90:42; c_loc needs nonzero sizes
    a%im = im; a%levs = levs; a%ltp = ltp; a%lm = lm; a%kd = kd
    a%lslwr = 1; a%lwhtr = merge(1_c_int32_t, 0_c_int32_t, lwhtr)
    a%tsfa = c_loc(tsfa); a%sfcflw = c_loc(sfcflw)     ! records of 4 real(kind_phys)
    a%tsflw = c_loc(tsflw); a%sfcdlw = c_loc(sfcdlw)
    if (levs > 0 .and. lm + ltp > 0) then
      a%htlwc = c_loc(htlwc); a%htrlw = c_loc(htrlw)
      if (lwhtr) then
        a%htlw0 = c_loc(htlw0); a%lwhc = c_loc(lwhc)
      end if
    end if
    x%precision = 0; x%memory = 0; x%sync = 1; x%reserved = 0
    errflg = c_rrtmg_lw_gpu_post(a, x, cmsg, size(cmsg, kind=c_int32_t))
    errmsg = ''
    do i = 1, min(size(cmsg), len(errmsg))
      if (cmsg(i) == c_null_char) exit
      errmsg(i:i) = cmsg(i)
    end do
  end subroutine rrtmg_lw_post_run
end module rrtmg_lw_post
