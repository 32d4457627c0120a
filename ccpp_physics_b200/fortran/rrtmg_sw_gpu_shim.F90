!> \file rrtmg_sw_gpu_shim.F90
!! Drop-in module rrtmg_sw for a CCPP host: the public rswinit and
!! rrtmg_sw_run keep the interfaces of physics/Radiation/RRTMG/radsw_main.F90
!! (rrtmg_sw_run :493-510 with the declarations :515-600, rswinit
!! :1388-1390) and forward to the C ABI of librrtmg_lw_gpu.so
!! (include/rrtmg_sw_gpu.h) through ISO_C_BINDING.  Build it in place of
!! radsw_main.F90 and link the shared library.  Arrays are passed by address
!! (no copies when the actual arguments are contiguous); optional arguments
!! that are absent become NULL.  Host memory is staged to the GPU inside the
!! library.
module rrtmg_sw_gpu_c
  use iso_c_binding
  implicit none
  private
  public :: c_sw_init_args, c_sw_run_args, c_rrtmg_sw_gpu_init, c_rrtmg_sw_gpu_run

  type, bind(c) :: c_sw_init_args
    integer(c_int32_t) :: me, rad_hr_units, inc_minor_gas, iswcliq, isubcsw
    integer(c_int32_t) :: iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp, iovr_exprand
    integer(c_int32_t) :: iswmode, device
  end type

  type, bind(c) :: c_sw_run_args
    integer(c_int32_t) :: npts, nlay, nlp1, ldim, nday, lprnt, lsswr, top_at_1, inc_minor_gas
    integer(c_int32_t) :: iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp, iovr_exprand
    integer(c_int32_t) :: iswcliq, iswcice, isubcsw, iswmode
    real(c_double) :: solcon
    type(c_ptr) :: plyr = c_null_ptr, plvl = c_null_ptr, tlyr = c_null_ptr, tlvl = c_null_ptr
    type(c_ptr) :: qlyr = c_null_ptr, olyr = c_null_ptr
    type(c_ptr) :: gasvmr_co2 = c_null_ptr, gasvmr_n2o = c_null_ptr, gasvmr_ch4 = c_null_ptr
    type(c_ptr) :: gasvmr_o2 = c_null_ptr, gasvmr_co = c_null_ptr, gasvmr_cfc11 = c_null_ptr
    type(c_ptr) :: gasvmr_cfc12 = c_null_ptr, gasvmr_cfc22 = c_null_ptr, gasvmr_ccl4 = c_null_ptr
    type(c_ptr) :: icseed = c_null_ptr, idxday = c_null_ptr
    type(c_ptr) :: aeraod = c_null_ptr, aerssa = c_null_ptr, aerasy = c_null_ptr
    type(c_ptr) :: sfcalb_nir_dir = c_null_ptr, sfcalb_nir_dif = c_null_ptr
    type(c_ptr) :: sfcalb_uvis_dir = c_null_ptr, sfcalb_uvis_dif = c_null_ptr
    type(c_ptr) :: dzlyr = c_null_ptr, delpin = c_null_ptr, de_lgth = c_null_ptr, alpha = c_null_ptr
    type(c_ptr) :: cosz = c_null_ptr, cld_cf = c_null_ptr
    type(c_ptr) :: cld_lwp = c_null_ptr, cld_ref_liq = c_null_ptr, cld_iwp = c_null_ptr
    type(c_ptr) :: cld_ref_ice = c_null_ptr, cld_rwp = c_null_ptr, cld_ref_rain = c_null_ptr
    type(c_ptr) :: cld_swp = c_null_ptr, cld_ref_snow = c_null_ptr, cld_od = c_null_ptr
    type(c_ptr) :: cld_ssa = c_null_ptr, cld_asy = c_null_ptr
    type(c_ptr) :: hswc = c_null_ptr, topflx = c_null_ptr, sfcflx = c_null_ptr, cldtau = c_null_ptr
    type(c_ptr) :: hsw0 = c_null_ptr, hswb = c_null_ptr, flxprf = c_null_ptr, fdncmp = c_null_ptr
  end type

  interface
    integer(c_int) function c_rrtmg_sw_gpu_init(args, errmsg, errmsg_len) bind(c, name="rrtmg_sw_gpu_init")
      import :: c_sw_init_args, c_int, c_char, c_int32_t
      type(c_sw_init_args), intent(in) :: args
      character(kind=c_char), dimension(*), intent(out) :: errmsg
      integer(c_int32_t), value :: errmsg_len
    end function
    integer(c_int) function c_rrtmg_sw_gpu_run(args, errmsg, errmsg_len) bind(c, name="rrtmg_sw_gpu_run")
      import :: c_sw_run_args, c_int, c_char, c_int32_t
      type(c_sw_run_args), intent(in) :: args
      character(kind=c_char), dimension(*), intent(out) :: errmsg
      integer(c_int32_t), value :: errmsg_len
    end function
  end interface
end module rrtmg_sw_gpu_c


module rrtmg_sw
  use iso_c_binding
  use machine, only: kind_phys
  use module_radsw_parameters, only: topfsw_type, sfcfsw_type, profsw_type, cmpfsw_type
  use rrtmg_sw_gpu_c
  implicit none
  private
  public :: rrtmg_sw_run, rswinit

contains

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

  !> rswinit (radsw_main.F90:1388): same arguments; the GPU device is the
  !! one current for the calling MPI rank.
  subroutine rswinit(me, rad_hr_units, inc_minor_gas, iswcliq, isubcsw, iovr, iovr_rand, iovr_maxrand, &
                     iovr_max, iovr_dcorr, iovr_exp, iovr_exprand, iswmode, errflg, errmsg)
    integer, intent(in) :: me, rad_hr_units, iswcliq, isubcsw, iovr, iswmode, iovr_rand, iovr_maxrand, &
                           iovr_max, iovr_dcorr, iovr_exp, iovr_exprand
    logical, intent(in) :: inc_minor_gas
    character(len=*), intent(out) :: errmsg
    integer, intent(out) :: errflg
    type(c_sw_init_args) :: a
    character(kind=c_char) :: cmsg(512)
    a = c_sw_init_args(me, rad_hr_units, lg(inc_minor_gas), iswcliq, isubcsw, iovr, iovr_rand, iovr_maxrand, &
                       iovr_max, iovr_dcorr, iovr_exp, iovr_exprand, iswmode, 0)
    errflg = c_rrtmg_sw_gpu_init(a, cmsg, size(cmsg, kind=c_int32_t))
    call c2f(cmsg, errmsg)
  end subroutine rswinit

  !> rrtmg_sw_run (radsw_main.F90:493-510): same dummy arguments.
  subroutine rrtmg_sw_run(plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr_co2, gasvmr_n2o, gasvmr_ch4, gasvmr_o2, &
                          gasvmr_co, gasvmr_cfc11, gasvmr_cfc12, gasvmr_cfc22, gasvmr_ccl4, icseed, aeraod, aerssa, &
                          aerasy, sfcalb_nir_dir, sfcalb_nir_dif, sfcalb_uvis_dir, sfcalb_uvis_dif, dzlyr, delpin, &
                          de_lgth, alpha, cosz, solcon, NDAY, idxday, npts, nlay, nlp1, lprnt, inc_minor_gas, &
                          iswcliq, iswcice, isubcsw, iovr, top_at_1, iswmode, cld_cf, lsswr, iovr_rand, &
                          iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp, iovr_exprand, hswc, topflx, sfcflx, cldtau, &
                          HSW0, HSWB, FLXPRF, FDNCMP, cld_lwp, cld_ref_liq, cld_iwp, cld_ref_ice, cld_rwp, &
                          cld_ref_rain, cld_swp, cld_ref_snow, cld_od, cld_ssa, cld_asy, errmsg, errflg)
    integer, intent(in) :: npts, nlay, nlp1, NDAY, iswcliq, iswcice, isubcsw, iovr, iswmode, iovr_dcorr, &
                           iovr_exp, iovr_exprand, iovr_rand, iovr_maxrand, iovr_max
    integer, dimension(:), intent(in), target, contiguous :: idxday, icseed
    logical, intent(in) :: lprnt, lsswr, inc_minor_gas, top_at_1
    real(kind_phys), dimension(:,:), intent(in), target, contiguous :: plvl, tlvl, plyr, tlyr, qlyr, olyr, &
         dzlyr, delpin, gasvmr_co2, gasvmr_n2o, gasvmr_ch4, gasvmr_o2, gasvmr_co, gasvmr_cfc11, gasvmr_cfc12, &
         gasvmr_cfc22, gasvmr_ccl4, cld_cf
    real(kind_phys), dimension(:), intent(in), target, contiguous :: sfcalb_nir_dir, sfcalb_nir_dif, &
         sfcalb_uvis_dir, sfcalb_uvis_dif
    real(kind_phys), dimension(:,:), intent(in), target, contiguous, optional :: cld_lwp, cld_ref_liq, &
         cld_iwp, cld_ref_ice, cld_rwp, cld_ref_rain, cld_swp, cld_ref_snow, cld_od, cld_ssa, cld_asy
    real(kind_phys), dimension(:,:,:), intent(in), target, contiguous :: aeraod, aerssa, aerasy
    real(kind_phys), intent(in), target :: cosz(npts), de_lgth(npts)
    real(kind_phys), intent(in) :: solcon
    real(kind_phys), dimension(npts,nlay), intent(in), target :: alpha
    real(kind_phys), dimension(:,:), intent(inout), target, contiguous :: hswc, cldtau
    type(topfsw_type), dimension(:), intent(inout), target :: topflx
    type(sfcfsw_type), dimension(:), intent(inout), target :: sfcflx
    real(kind_phys), dimension(:,:,:), optional, intent(inout), target, contiguous :: hswb
    real(kind_phys), dimension(:,:), optional, intent(inout), target, contiguous :: hsw0
    type(profsw_type), dimension(:,:), optional, intent(inout), target :: flxprf
    type(cmpfsw_type), dimension(:), optional, intent(inout), target :: fdncmp
    character(len=*), intent(out) :: errmsg
    integer, intent(out) :: errflg
    type(c_sw_run_args) :: a
    character(kind=c_char) :: cmsg(512)

    a%npts = npts; a%nlay = nlay; a%nlp1 = nlp1; a%ldim = size(plyr, 1); a%nday = NDAY
    a%lprnt = lg(lprnt); a%lsswr = lg(lsswr); a%top_at_1 = lg(top_at_1); a%inc_minor_gas = lg(inc_minor_gas)
    a%iovr = iovr; a%iovr_rand = iovr_rand; a%iovr_maxrand = iovr_maxrand; a%iovr_max = iovr_max
    a%iovr_dcorr = iovr_dcorr; a%iovr_exp = iovr_exp; a%iovr_exprand = iovr_exprand
    a%iswcliq = iswcliq; a%iswcice = iswcice; a%isubcsw = isubcsw; a%iswmode = iswmode
    a%solcon = solcon
    a%plyr = c_loc(plyr); a%plvl = c_loc(plvl); a%tlyr = c_loc(tlyr); a%tlvl = c_loc(tlvl)
    a%qlyr = c_loc(qlyr); a%olyr = c_loc(olyr)
    a%gasvmr_co2 = c_loc(gasvmr_co2); a%gasvmr_n2o = c_loc(gasvmr_n2o); a%gasvmr_ch4 = c_loc(gasvmr_ch4)
    a%gasvmr_o2 = c_loc(gasvmr_o2); a%gasvmr_co = c_loc(gasvmr_co); a%gasvmr_cfc11 = c_loc(gasvmr_cfc11)
    a%gasvmr_cfc12 = c_loc(gasvmr_cfc12); a%gasvmr_cfc22 = c_loc(gasvmr_cfc22)
    a%gasvmr_ccl4 = c_loc(gasvmr_ccl4)
    a%icseed = c_loc(icseed); a%idxday = c_loc(idxday)
    a%aeraod = c_loc(aeraod); a%aerssa = c_loc(aerssa); a%aerasy = c_loc(aerasy)
    a%sfcalb_nir_dir = c_loc(sfcalb_nir_dir); a%sfcalb_nir_dif = c_loc(sfcalb_nir_dif)
    a%sfcalb_uvis_dir = c_loc(sfcalb_uvis_dir); a%sfcalb_uvis_dif = c_loc(sfcalb_uvis_dif)
    a%dzlyr = c_loc(dzlyr); a%delpin = c_loc(delpin); a%de_lgth = c_loc(de_lgth); a%alpha = c_loc(alpha)
    a%cosz = c_loc(cosz); a%cld_cf = c_loc(cld_cf)
    if (present(cld_lwp)) a%cld_lwp = c_loc(cld_lwp)
    if (present(cld_ref_liq)) a%cld_ref_liq = c_loc(cld_ref_liq)
    if (present(cld_iwp)) a%cld_iwp = c_loc(cld_iwp)
    if (present(cld_ref_ice)) a%cld_ref_ice = c_loc(cld_ref_ice)
    if (present(cld_rwp)) a%cld_rwp = c_loc(cld_rwp)
    if (present(cld_ref_rain)) a%cld_ref_rain = c_loc(cld_ref_rain)
    if (present(cld_swp)) a%cld_swp = c_loc(cld_swp)
    if (present(cld_ref_snow)) a%cld_ref_snow = c_loc(cld_ref_snow)
    if (present(cld_od)) a%cld_od = c_loc(cld_od)
    if (present(cld_ssa)) a%cld_ssa = c_loc(cld_ssa)
    if (present(cld_asy)) a%cld_asy = c_loc(cld_asy)
    a%hswc = c_loc(hswc); a%cldtau = c_loc(cldtau)
    a%topflx = c_loc(topflx); a%sfcflx = c_loc(sfcflx)     ! records of 3 / 4 real(kind_phys)
    if (present(hsw0)) a%hsw0 = c_loc(hsw0)
    if (present(hswb)) a%hswb = c_loc(hswb)
    if (present(flxprf)) a%flxprf = c_loc(flxprf)          ! records of 4 real(kind_phys)
    if (present(fdncmp)) a%fdncmp = c_loc(fdncmp)          ! records of 6 real(kind_phys)
    errflg = c_rrtmg_sw_gpu_run(a, cmsg, size(cmsg, kind=c_int32_t))
    call c2f(cmsg, errmsg)
  end subroutine rrtmg_sw_run

end module rrtmg_sw
