!> \file rrtmg_lw_gpu_shim.F90
!! Drop-in module rrtmg_lw for a CCPP host: the public rlwinit and
!! rrtmg_lw_run keep the interfaces of physics/Radiation/RRTMG/radlw_main.F90
!! (rrtmg_lw_run :419-434 with the declarations :609-656, rlwinit
!! :1322-1324) and forward to the C ABI of librrtmg_lw_gpu.so
!! (include/rrtmg_lw_gpu.h) through ISO_C_BINDING.  Build it in place of
!! radlw_main.F90 and link the shared library.  Arrays are passed by address
!! (no copies when the actual arguments are contiguous, which CCPP's
!! (horizontal_loop_extent, ...) arrays are); optional arguments that are
!! absent become NULL.  Host memory is staged to the GPU inside the library.
module rrtmg_lw_gpu_c
  use iso_c_binding
  implicit none
  private
  public :: c_init_args, c_run_args, c_rrtmg_lw_gpu_init, c_rrtmg_lw_gpu_run

  type, bind(c) :: c_init_args
    integer(c_int32_t) :: me, rad_hr_units, inc_minor_gas, ilwcliq, isubclw
    integer(c_int32_t) :: iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp, iovr_exprand
    integer(c_int32_t) :: device
  end type

  type, bind(c) :: c_run_args
    integer(c_int32_t) :: npts, nlay, nlp1, ldim, lprnt, lslwr, top_at_1, inc_minor_gas
    integer(c_int32_t) :: iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp, iovr_exprand
    integer(c_int32_t) :: ilwcliq, ilwcice, isubclw
    type(c_ptr) :: plyr = c_null_ptr, plvl = c_null_ptr, tlyr = c_null_ptr, tlvl = c_null_ptr
    type(c_ptr) :: qlyr = c_null_ptr, olyr = c_null_ptr
    type(c_ptr) :: gasvmr_co2 = c_null_ptr, gasvmr_n2o = c_null_ptr, gasvmr_ch4 = c_null_ptr
    type(c_ptr) :: gasvmr_o2 = c_null_ptr, gasvmr_co = c_null_ptr, gasvmr_cfc11 = c_null_ptr
    type(c_ptr) :: gasvmr_cfc12 = c_null_ptr, gasvmr_cfc22 = c_null_ptr, gasvmr_ccl4 = c_null_ptr
    type(c_ptr) :: icseed = c_null_ptr, aeraod = c_null_ptr, aerssa = c_null_ptr
    type(c_ptr) :: sfemis = c_null_ptr, sfgtmp = c_null_ptr, dzlyr = c_null_ptr, delpin = c_null_ptr
    type(c_ptr) :: de_lgth = c_null_ptr, alpha = c_null_ptr, cld_cf = c_null_ptr
    type(c_ptr) :: cld_lwp = c_null_ptr, cld_ref_liq = c_null_ptr, cld_iwp = c_null_ptr
    type(c_ptr) :: cld_ref_ice = c_null_ptr, cld_rwp = c_null_ptr, cld_ref_rain = c_null_ptr
    type(c_ptr) :: cld_swp = c_null_ptr, cld_ref_snow = c_null_ptr, cld_od = c_null_ptr
    type(c_ptr) :: hlwc = c_null_ptr, topflx = c_null_ptr, sfcflx = c_null_ptr, cldtau = c_null_ptr
    type(c_ptr) :: hlw0 = c_null_ptr, hlwb = c_null_ptr, flxprf = c_null_ptr
  end type

  interface
    integer(c_int) function c_rrtmg_lw_gpu_init(args, errmsg, errmsg_len) bind(c, name="rrtmg_lw_gpu_init")
      import :: c_init_args, c_int, c_char, c_int32_t
      type(c_init_args), intent(in) :: args
      character(kind=c_char), dimension(*), intent(out) :: errmsg
      integer(c_int32_t), value :: errmsg_len
    end function
    integer(c_int) function c_rrtmg_lw_gpu_run(args, errmsg, errmsg_len) bind(c, name="rrtmg_lw_gpu_run")
      import :: c_run_args, c_int, c_char, c_int32_t
      type(c_run_args), intent(in) :: args
      character(kind=c_char), dimension(*), intent(out) :: errmsg
      integer(c_int32_t), value :: errmsg_len
    end function
  end interface
end module rrtmg_lw_gpu_c


module rrtmg_lw
  use iso_c_binding
  use machine, only: kind_phys
  use module_radlw_parameters, only: topflw_type, sfcflw_type, proflw_type
  use rrtmg_lw_gpu_c
  implicit none
  private
  public :: rrtmg_lw_run, rlwinit

contains

  ! copy a NUL-terminated C message into a Fortran string
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

  !> rlwinit (radlw_main.F90:1322): same arguments; the GPU device is the
  !! one current for the calling MPI rank.
  subroutine rlwinit(me, rad_hr_units, inc_minor_gas, ilwcliq, isubclw, iovr, iovr_rand, iovr_maxrand, &
                     iovr_max, iovr_dcorr, iovr_exp, iovr_exprand, errflg, errmsg)
    integer, intent(in) :: me, rad_hr_units, ilwcliq, isubclw, iovr, iovr_rand, iovr_maxrand, iovr_max, &
                           iovr_dcorr, iovr_exp, iovr_exprand
    logical, intent(in) :: inc_minor_gas
    character(len=*), intent(out) :: errmsg
    integer, intent(out) :: errflg
    type(c_init_args) :: a
    character(kind=c_char) :: cmsg(512)
    a = c_init_args(me, rad_hr_units, lg(inc_minor_gas), ilwcliq, isubclw, iovr, iovr_rand, iovr_maxrand, &
                    iovr_max, iovr_dcorr, iovr_exp, iovr_exprand, 0)
    errflg = c_rrtmg_lw_gpu_init(a, cmsg, size(cmsg, kind=c_int32_t))
    call c2f(cmsg, errmsg)
  end subroutine rlwinit

  !> rrtmg_lw_run (radlw_main.F90:419-434): same dummy arguments.
  subroutine rrtmg_lw_run(plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr_co2, gasvmr_n2o, gasvmr_ch4, gasvmr_o2, &
                          gasvmr_co, gasvmr_cfc11, gasvmr_cfc12, gasvmr_cfc22, gasvmr_ccl4, icseed, aeraod, aerssa, &
                          sfemis, sfgtmp, dzlyr, delpin, de_lgth, alpha, npts, nlay, nlp1, lprnt, cld_cf, lslwr, &
                          top_at_1, iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp, iovr_exprand, &
                          inc_minor_gas, ilwcliq, ilwcice, isubclw, hlwc, topflx, sfcflx, cldtau, hlw0, hlwb, flxprf, &
                          cld_lwp, cld_ref_liq, cld_iwp, cld_ref_ice, cld_rwp, cld_ref_rain, cld_swp, cld_ref_snow, &
                          cld_od, errmsg, errflg)
    integer, intent(in) :: npts, nlay, nlp1, ilwcliq, ilwcice, isubclw, iovr, iovr_dcorr, iovr_exp, &
                           iovr_exprand, iovr_rand, iovr_maxrand, iovr_max
    integer, intent(in), target :: icseed(npts)
    logical, intent(in) :: lprnt, inc_minor_gas, lslwr, top_at_1
    real(kind_phys), dimension(:,:), intent(in), target, contiguous :: plvl, tlvl, plyr, tlyr, qlyr, olyr, &
         dzlyr, delpin, gasvmr_co2, gasvmr_n2o, gasvmr_ch4, gasvmr_o2, gasvmr_co, gasvmr_cfc11, gasvmr_cfc12, &
         gasvmr_cfc22, gasvmr_ccl4, cld_cf
    real(kind_phys), dimension(:,:), intent(in), target, contiguous, optional :: cld_lwp, cld_ref_liq, &
         cld_iwp, cld_ref_ice, cld_rwp, cld_ref_rain, cld_swp, cld_ref_snow, cld_od
    real(kind_phys), dimension(:), intent(in), target, contiguous :: sfemis, sfgtmp, de_lgth
    real(kind_phys), dimension(npts,nlay), intent(in), target :: alpha
    real(kind_phys), dimension(:,:,:), intent(in), target, contiguous :: aeraod, aerssa
    real(kind_phys), dimension(:,:), intent(inout), target, contiguous :: hlwc, cldtau
    type(topflw_type), dimension(:), intent(inout), target :: topflx
    type(sfcflw_type), dimension(:), intent(inout), target :: sfcflx
    real(kind_phys), dimension(:,:,:), optional, intent(inout), target, contiguous :: hlwb
    real(kind_phys), dimension(:,:), optional, intent(inout), target, contiguous :: hlw0
    type(proflw_type), dimension(:,:), optional, intent(inout), target :: flxprf
    character(len=*), intent(out) :: errmsg
    integer, intent(out) :: errflg
    type(c_run_args) :: a
    character(kind=c_char) :: cmsg(512)

    a%npts = npts; a%nlay = nlay; a%nlp1 = nlp1; a%ldim = size(plyr, 1)
    a%lprnt = lg(lprnt); a%lslwr = lg(lslwr); a%top_at_1 = lg(top_at_1); a%inc_minor_gas = lg(inc_minor_gas)
    a%iovr = iovr; a%iovr_rand = iovr_rand; a%iovr_maxrand = iovr_maxrand; a%iovr_max = iovr_max
    a%iovr_dcorr = iovr_dcorr; a%iovr_exp = iovr_exp; a%iovr_exprand = iovr_exprand
    a%ilwcliq = ilwcliq; a%ilwcice = ilwcice; a%isubclw = isubclw
    a%plyr = c_loc(plyr); a%plvl = c_loc(plvl); a%tlyr = c_loc(tlyr); a%tlvl = c_loc(tlvl)
    a%qlyr = c_loc(qlyr); a%olyr = c_loc(olyr)
    a%gasvmr_co2 = c_loc(gasvmr_co2); a%gasvmr_n2o = c_loc(gasvmr_n2o); a%gasvmr_ch4 = c_loc(gasvmr_ch4)
    a%gasvmr_o2 = c_loc(gasvmr_o2); a%gasvmr_co = c_loc(gasvmr_co); a%gasvmr_cfc11 = c_loc(gasvmr_cfc11)
    a%gasvmr_cfc12 = c_loc(gasvmr_cfc12); a%gasvmr_cfc22 = c_loc(gasvmr_cfc22)
    a%gasvmr_ccl4 = c_loc(gasvmr_ccl4)
    a%icseed = c_loc(icseed); a%aeraod = c_loc(aeraod); a%aerssa = c_loc(aerssa)
    a%sfemis = c_loc(sfemis); a%sfgtmp = c_loc(sfgtmp); a%dzlyr = c_loc(dzlyr); a%delpin = c_loc(delpin)
    a%de_lgth = c_loc(de_lgth); a%alpha = c_loc(alpha); a%cld_cf = c_loc(cld_cf)
    if (present(cld_lwp)) a%cld_lwp = c_loc(cld_lwp)
    if (present(cld_ref_liq)) a%cld_ref_liq = c_loc(cld_ref_liq)
    if (present(cld_iwp)) a%cld_iwp = c_loc(cld_iwp)
    if (present(cld_ref_ice)) a%cld_ref_ice = c_loc(cld_ref_ice)
    if (present(cld_rwp)) a%cld_rwp = c_loc(cld_rwp)
    if (present(cld_ref_rain)) a%cld_ref_rain = c_loc(cld_ref_rain)
    if (present(cld_swp)) a%cld_swp = c_loc(cld_swp)
    if (present(cld_ref_snow)) a%cld_ref_snow = c_loc(cld_ref_snow)
    if (present(cld_od)) a%cld_od = c_loc(cld_od)
    a%hlwc = c_loc(hlwc); a%cldtau = c_loc(cldtau)
    a%topflx = c_loc(topflx); a%sfcflx = c_loc(sfcflx)     ! records of 2 / 4 real(kind_phys)
    if (present(hlw0)) a%hlw0 = c_loc(hlw0)
    if (present(hlwb)) a%hlwb = c_loc(hlwb)
    if (present(flxprf)) a%flxprf = c_loc(flxprf)          ! records of 4 real(kind_phys)
    errflg = c_rrtmg_lw_gpu_run(a, cmsg, size(cmsg, kind=c_int32_t))
    call c2f(cmsg, errmsg)
  end subroutine rrtmg_lw_run

end module rrtmg_lw
