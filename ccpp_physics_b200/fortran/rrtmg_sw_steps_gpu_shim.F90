!> \file rrtmg_sw_steps_gpu_shim.F90
!! Drop-in modules rad_sw_pre and rrtmg_sw_post for a CCPP host: the public
!! rad_sw_pre_run (physics/Radiation/RRTMG/rad_sw_pre.F90:14-51) and
!! rrtmg_sw_post_run (physics/Radiation/RRTMG/rrtmg_sw_post.F90:13-129) keep
!! the reference's dummy arguments and forward to the C ABI of
!! librrtmg_lw_gpu.so (rrtmg_sw_gpu_pre, rrtmg_sw_gpu_post in
!! include/rrtmg_sw_gpu.h) through ISO_C_BINDING, host memory, synchronous.
!! Build them in place of rad_sw_pre.F90 and rrtmg_sw_post.F90.  Arrays are
!! passed by address; the derived-type records are contiguous reals, the
!! layout the C ABI expects.
module rrtmg_sw_steps_gpu_c
  use iso_c_binding
  implicit none
  private
  public :: c_sw_exec, c_sw_pre_args, c_sw_post_args, c_rrtmg_sw_gpu_pre, c_rrtmg_sw_gpu_post, host_exec, &
            c2f, lg

  type, bind(c) :: c_sw_exec
    integer(c_int32_t) :: precision, memory
    type(c_ptr) :: stream = c_null_ptr
    integer(c_int32_t) :: sync, reserved
    type(c_ptr) :: kernel_ms = c_null_ptr
  end type

  type, bind(c) :: c_sw_pre_args
    integer(c_int32_t) :: im, lsswr
    type(c_ptr) :: coszen = c_null_ptr, nday = c_null_ptr, idxday = c_null_ptr
  end type

  type, bind(c) :: c_sw_post_args
    integer(c_int32_t) :: im, levr, levs, ltp, nday, lm, kd, lsswr, swhtr
    type(c_ptr) :: sfcalb1 = c_null_ptr, sfcalb2 = c_null_ptr, sfcalb3 = c_null_ptr, sfcalb4 = c_null_ptr
    type(c_ptr) :: htswc = c_null_ptr, htsw0 = c_null_ptr
    type(c_ptr) :: nirbmdi = c_null_ptr, nirdfdi = c_null_ptr, visbmdi = c_null_ptr, visdfdi = c_null_ptr
    type(c_ptr) :: nirbmui = c_null_ptr, nirdfui = c_null_ptr, visbmui = c_null_ptr, visdfui = c_null_ptr
    type(c_ptr) :: sfcdsw = c_null_ptr, sfcnsw = c_null_ptr, htrsw = c_null_ptr, swhc = c_null_ptr
    type(c_ptr) :: scmpsw = c_null_ptr, sfcfsw = c_null_ptr, topfsw = c_null_ptr
  end type

  interface
    integer(c_int) function c_rrtmg_sw_gpu_pre(args, exec, errmsg, errmsg_len) bind(c, name="rrtmg_sw_gpu_pre")
      import :: c_sw_pre_args, c_sw_exec, c_int, c_char, c_int32_t
      type(c_sw_pre_args), intent(in) :: args
      type(c_sw_exec), intent(in) :: exec
      character(kind=c_char), dimension(*), intent(out) :: errmsg
      integer(c_int32_t), value :: errmsg_len
    end function
    integer(c_int) function c_rrtmg_sw_gpu_post(args, exec, errmsg, errmsg_len) bind(c, name="rrtmg_sw_gpu_post")
      import :: c_sw_post_args, c_sw_exec, c_int, c_char, c_int32_t
      type(c_sw_post_args), intent(in) :: args
      type(c_sw_exec), intent(in) :: exec
      character(kind=c_char), dimension(*), intent(out) :: errmsg
      integer(c_int32_t), value :: errmsg_len
    end function
  end interface

contains

  !> FP64, host pointers, synchronous, the calling thread's stream.
  type(c_sw_exec) function host_exec()
    host_exec%precision = 0
    host_exec%memory = 0
    host_exec%stream = c_null_ptr
    host_exec%sync = 1
    host_exec%reserved = 0
    host_exec%kernel_ms = c_null_ptr
  end function host_exec

  subroutine c2f(cmsg, fmsg)
    character(kind=c_char), dimension(:), intent(in) :: cmsg
    character(len=*), intent(out) :: fmsg
    integer :: i
    fmsg = ''
    do i = 1, min(size(cmsg), len(fmsg))
      if (cmsg(i) == c_null_char) exit
      fmsg(i:i) = cmsg(i)
    end do
  end subroutine c2f

  integer(c_int32_t) function lg(l)
    logical, intent(in) :: l
    lg = merge(1_c_int32_t, 0_c_int32_t, l)
  end function lg
end module rrtmg_sw_steps_gpu_c


module rad_sw_pre
  use iso_c_binding
  use machine, only: kind_phys
  use rrtmg_sw_steps_gpu_c
  implicit none
  private
  public :: rad_sw_pre_run

contains

  !> rad_sw_pre_run (rad_sw_pre.F90:14): same dummy arguments.
  subroutine rad_sw_pre_run(im, lsswr, coszen, nday, idxday, errmsg, errflg)
    integer, intent(in) :: im
    logical, intent(in) :: lsswr
    real(kind_phys), dimension(:), intent(in), target, contiguous :: coszen
    integer, intent(out) :: nday
    integer, dimension(:), intent(out), target, contiguous :: idxday
    character(len=*), intent(out) :: errmsg
    integer, intent(out) :: errflg
    type(c_sw_pre_args) :: a
    character(kind=c_char) :: cmsg(512)
    integer(c_int32_t), target :: nd

    nday = 0; errmsg = ''; errflg = 0
    if (im <= 0 .or. size(idxday) == 0) return      ! c_loc needs arrays of nonzero size
    a%im = im; a%lsswr = lg(lsswr)
    a%nday = c_loc(nd); a%idxday = c_loc(idxday)
    if (size(coszen) > 0) a%coszen = c_loc(coszen)
    errflg = c_rrtmg_sw_gpu_pre(a, host_exec(), cmsg, size(cmsg, kind=c_int32_t))
    nday = nd
    call c2f(cmsg, errmsg)
  end subroutine rad_sw_pre_run
end module rad_sw_pre


module rrtmg_sw_post
  use iso_c_binding
  use machine, only: kind_phys
  use module_radsw_parameters, only: topfsw_type, sfcfsw_type, cmpfsw_type
  use rrtmg_sw_steps_gpu_c
  implicit none
  private
  public :: rrtmg_sw_post_run

contains

  !> rrtmg_sw_post_run (rrtmg_sw_post.F90:13-17): same dummy arguments.
  subroutine rrtmg_sw_post_run(im, levr, levs, ltp, nday, lm, kd, lsswr, swhtr, sfcalb1, sfcalb2, sfcalb3, &
                               sfcalb4, htswc, htsw0, nirbmdi, nirdfdi, visbmdi, visdfdi, nirbmui, nirdfui, &
                               visbmui, visdfui, sfcdsw, sfcnsw, htrsw, swhc, scmpsw, sfcfsw, topfsw, errmsg, errflg)
    integer, intent(in) :: im, levr, levs, ltp, nday, lm, kd
    logical, intent(in) :: lsswr, swhtr
    real(kind_phys), dimension(:), intent(in), target, contiguous :: sfcalb1, sfcalb2, sfcalb3, sfcalb4
    real(kind_phys), dimension(:,:), intent(in), target, contiguous :: htswc, htsw0
    real(kind_phys), dimension(:), intent(inout), target, contiguous :: nirbmdi, nirdfdi, visbmdi, visdfdi, &
         nirbmui, nirdfui, visbmui, visdfui, sfcdsw, sfcnsw
    real(kind_phys), dimension(:,:), intent(inout), target, contiguous :: htrsw, swhc
    type(cmpfsw_type), dimension(:), intent(inout), target :: scmpsw
    type(sfcfsw_type), dimension(:), intent(inout), target :: sfcfsw
    type(topfsw_type), dimension(:), intent(inout), target :: topfsw
    character(len=*), intent(out) :: errmsg
    integer, intent(out) :: errflg
    type(c_sw_post_args) :: a
    character(kind=c_char) :: cmsg(512)

    errmsg = ''; errflg = 0
    if (.not. lsswr .or. im <= 0) return               ! rrtmg_sw_post.F90:52; c_loc needs nonzero sizes
    a%im = im; a%levr = levr; a%levs = levs; a%ltp = ltp; a%nday = nday; a%lm = lm; a%kd = kd
    a%lsswr = lg(lsswr); a%swhtr = lg(swhtr)
    a%sfcalb1 = c_loc(sfcalb1); a%sfcalb2 = c_loc(sfcalb2); a%sfcalb3 = c_loc(sfcalb3)
    a%sfcalb4 = c_loc(sfcalb4)
    if (size(htswc) > 0) a%htswc = c_loc(htswc)
    if (swhtr .and. size(htsw0) > 0) a%htsw0 = c_loc(htsw0)
    a%nirbmdi = c_loc(nirbmdi); a%nirdfdi = c_loc(nirdfdi); a%visbmdi = c_loc(visbmdi)
    a%visdfdi = c_loc(visdfdi); a%nirbmui = c_loc(nirbmui); a%nirdfui = c_loc(nirdfui)
    a%visbmui = c_loc(visbmui); a%visdfui = c_loc(visdfui)
    a%sfcdsw = c_loc(sfcdsw); a%sfcnsw = c_loc(sfcnsw)
    if (size(htrsw) > 0) a%htrsw = c_loc(htrsw)
    if (swhtr .and. size(swhc) > 0) a%swhc = c_loc(swhc)
    a%scmpsw = c_loc(scmpsw)       ! records of 6 real(kind_phys)
    a%sfcfsw = c_loc(sfcfsw)       ! records of 4 real(kind_phys)
    a%topfsw = c_loc(topfsw)       ! records of 3 real(kind_phys)
    errflg = c_rrtmg_sw_gpu_post(a, host_exec(), cmsg, size(cmsg, kind=c_int32_t))
    call c2f(cmsg, errmsg)
  end subroutine rrtmg_sw_post_run
end module rrtmg_sw_post
