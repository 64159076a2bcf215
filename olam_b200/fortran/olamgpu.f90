!===============================================================================
! olamgpu.f90 -- ISO_C_BINDING side of the B200 library for OLAM.
!
! Module olamgpu_c declares the C-ABI of include/olamgpu.h (bind(C) types in
! the same member order, interfaces of the entry points).  Module
! olamgpu_shim fills those types from OLAM's own modules and is what the
! replacement wrtv_rk / scalar_transport modules (olamgpu_modules.f90) call.
!
! OLAM's per-point tables are arrays of derived types (itab_w(iw)%iv(7) ...),
! so the shim packs them once into contiguous (7, mwa) / (2, mva) / (3, mma)
! integer and real arrays kept here for the life of the run; every other
! array is passed in place, by address.
!
! This file is source for the OLAM build; it is not compiled in this
! repository (no Fortran compiler in the build image).
!===============================================================================
module olamgpu_c

  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: OLAMGPU_OK = 0
  integer(c_int), parameter :: OLAMGPU_SYNC_EACH_CALL = 0, OLAMGPU_RESIDENT = 1
  integer(c_int), parameter :: OLAMGPU_F_RHO = 1, OLAMGPU_F_PRESS = 2, OLAMGPU_F_THIL = 4, &
                               OLAMGPU_F_WC = 8, OLAMGPU_F_WMC = 16, OLAMGPU_F_VXE = 32,   &
                               OLAMGPU_F_VMC = 64, OLAMGPU_F_VC = 128, OLAMGPU_F_VMASC = 256, &
                               OLAMGPU_F_WMASC = 512, OLAMGPU_F_TEND = 1024,                &
                               OLAMGPU_F_FACS = 2048, OLAMGPU_F_SCALARS = 4096,            &
                               OLAMGPU_F_SCALAR_TEND = 8192, OLAMGPU_F_EDDY = 16384,       &
                               OLAMGPU_F_ALL = 65535
  integer(c_int), parameter :: OLAMGPU_TS_GRAPH = 1, OLAMGPU_TS_HORIZ_K = 2, &
                               OLAMGPU_TS_MAXMIN = 4, OLAMGPU_TS_MASS = 8
  integer(c_int), parameter :: OLAMGPU_WIN_HOST = 1, OLAMGPU_WIN_LEAN = 2

  type, bind(C) :: olamgpu_grid
     integer(c_int) :: mza, mwa, mva, mma
     integer(c_int) :: nw_prog;  type(c_ptr) :: jtw_prog
     integer(c_int) :: nw_wadj;  type(c_ptr) :: jtw_wadj
     integer(c_int) :: nv_prog;  type(c_ptr) :: jtv_prog
     integer(c_int) :: nv_wadj;  type(c_ptr) :: jtv_wadj
     integer(c_int) :: nm_prog;  type(c_ptr) :: jtm_prog
     type(c_ptr) :: npoly, itab_w_iv, itab_w_iw, itab_w_im, itab_w_dirv
     type(c_ptr) :: ecvec_vx, ecvec_vy, ecvec_vz, iwglobe
     type(c_ptr) :: itab_v_iw, itab_v_im, dxps, dyps
     type(c_ptr) :: itab_m_iv, itab_m_iw, itab_m_im
     type(c_ptr) :: lpw, lpv, lpm, lve2
     type(c_ptr) :: zm, zt, dzm, dzt, dzim, dzit, dzt_top, dzt_bot, zfacit
     type(c_ptr) :: zwgt_top8, zwgt_bot8, gdz_wgtm8, gdz_wgtp8, gdz_wgtm, gdz_wgtp
     type(c_ptr) :: wnx, wny, wnz, wnxo2, wnyo2, wnzo2, vnx, vny, vnz
     type(c_ptr) :: dnu, dniu, dnv, dniv, arw0, arm0
     type(c_ptr) :: arv, arw, volt, volti, volwi, volvi
     type(c_ptr) :: gxps_coef, gyps_coef, a_w, a_wu, xy_h, xy_hu
     type(c_ptr) :: xx0_v, xy0_v, yy0_v, xx0_vu, xy0_vu, yy0_vu, xx_yy, xx_yy_m
  end type olamgpu_grid

  type, bind(C) :: olamgpu_opts
     real(c_double) :: dtlm, dtsm
     integer(c_int) :: nacoust, nrk_wrtv, nrk_scal
     integer(c_int) :: thil_horiz_adv_order, wind_horiz_adv_order, scal_horiz_adv_order
     integer(c_int) :: ithil_monot, iwind_monot, iscal_monot
     real(c_float)  :: divh_damp_fact;  integer(c_int) :: divh_damp_level, divh_damp_short
     real(c_float)  :: vort_damp_fact;  integer(c_int) :: vort_damp_level, vort_damp_short
     real(c_float)  :: fcoriol
     integer(c_int) :: mdomain
     integer(c_int) :: krayf_bot
     type(c_ptr)    :: rayf_cof, dn01d, th01d, vc03d
     integer(c_int) :: krayfw_bot
     type(c_ptr)    :: rayf_cofw
     integer(c_int) :: initial
  end type olamgpu_opts

  type, bind(C) :: olamgpu_state
     type(c_ptr) :: rho, press, thil, wc, wmc, vxe, vye, vze, vmc, vc, vmasc, wmasc
     type(c_ptr) :: alpha_press, pwfac, pvfac, thilt, vmxet, vmyet, vmzet, vmt
  end type olamgpu_state

  type, bind(C) :: olamgpu_halo
     integer(c_int) :: nnb
     type(c_ptr)    :: rank, nsend, send_cols, nrecv, recv_cols
     integer(c_int) :: host_staged
     type(c_funptr) :: exchange     ! int f(user, nnb, rank, sendbuf, sendcount, recvbuf, recvcount, stream)
     type(c_ptr)    :: user
     type(c_ptr)    :: nsend_v, send_v, nrecv_v, recv_v, nsend_m, send_m, nrecv_m, recv_m
  end type olamgpu_halo

  type, bind(C) :: olamgpu_eddy
     type(c_ptr) :: vkm, vkh, agamma, akm_sfc, sfluxt, kmtop, khtop, kpblh, theta, tair
     type(c_ptr) :: akmodx, akhodx, kmtopv, khtopv, lsw
     integer(c_int) :: nsw_max
     type(c_ptr) :: mrlw, mrlv
     integer(c_int) :: mrls
     type(c_ptr) :: idiffk, akmin
     integer(c_int) :: test_case
     real(c_float) :: cp
     integer(c_int) :: krayfmix_bot
     type(c_ptr) :: rayf_cofmix
  end type olamgpu_eddy

  interface
     integer(c_int) function olamgpu_init(grid, opts, state) bind(C, name="olamgpu_init")
       import :: c_int, olamgpu_grid, olamgpu_opts, olamgpu_state
       type(olamgpu_grid),  intent(in) :: grid
       type(olamgpu_opts),  intent(in) :: opts
       type(olamgpu_state), intent(in) :: state
     end function
     integer(c_int) function olamgpu_register_scalars(n, var_p, var_t, pdef, sgsmix) &
          bind(C, name="olamgpu_register_scalars")
       import :: c_int, c_ptr
       integer(c_int), value :: n
       type(c_ptr), intent(in) :: var_p(*), var_t(*)
       integer(c_int), intent(in) :: pdef(*), sgsmix(*)
     end function
     integer(c_int) function olamgpu_set_coherence(mode) bind(C, name="olamgpu_set_coherence")
       import :: c_int
       integer(c_int), value :: mode
     end function
     integer(c_int) function olamgpu_sync_to_device(mask) bind(C, name="olamgpu_sync_to_device")
       import :: c_int
       integer(c_int), value :: mask
     end function
     integer(c_int) function olamgpu_sync_to_host(mask) bind(C, name="olamgpu_sync_to_host")
       import :: c_int
       integer(c_int), value :: mask
     end function
     integer(c_int) function olamgpu_scalar_transport_rk(rho_old, diag) &
          bind(C, name="olamgpu_scalar_transport_rk")
       import :: c_int, c_float, c_ptr
       real(c_float), intent(in) :: rho_old(*)
       type(c_ptr), value :: diag
     end function
     ! lam(n) / lam_sct(n): c_loc of tracer n's (mza,mwa) adjoint arrays
     integer(c_int) function olamgpu_scalar_transport_rk_adjoint(rho_old, lam, lam_sct) &
          bind(C, name="olamgpu_scalar_transport_rk_adjoint")
       import :: c_int, c_float, c_ptr
       real(c_float), intent(in) :: rho_old(*)
       type(c_ptr), intent(in) :: lam(*)
       type(c_ptr), intent(in) :: lam_sct(*)
     end function
     integer(c_int) function olamgpu_prog_wrtv_rk(istp) bind(C, name="olamgpu_prog_wrtv_rk")
       import :: c_int
       integer(c_int), value :: istp
     end function
     integer(c_int) function olamgpu_tend0(rho_old) bind(C, name="olamgpu_tend0")
       import :: c_int, c_float
       real(c_float), intent(out) :: rho_old(*)
     end function
     integer(c_int) function olamgpu_timeavg_momsc() bind(C, name="olamgpu_timeavg_momsc")
       import :: c_int
     end function
     integer(c_int) function olamgpu_set_eddy(eddy) bind(C, name="olamgpu_set_eddy")
       import :: c_int, olamgpu_eddy
       type(olamgpu_eddy), intent(in) :: eddy
     end function
     integer(c_int) function olamgpu_comp_horiz_k() bind(C, name="olamgpu_comp_horiz_k")
       import :: c_int
     end function
     integer(c_int) function olamgpu_set_halo(halo) bind(C, name="olamgpu_set_halo")
       import :: c_int, olamgpu_halo
       type(olamgpu_halo), intent(in) :: halo
     end function
     integer(c_int) function olamgpu_timestep(flags, nmass, mass_ids) bind(C, name="olamgpu_timestep")
       import :: c_int
       integer(c_int), value :: flags, nmass
       integer(c_int), intent(in) :: mass_ids(*)
     end function
     ! emis(n): c_loc of scalar n's (mwa) surface source, or c_null_ptr
     integer(c_int) function olamgpu_set_surface_emission(emis) bind(C, name="olamgpu_set_surface_emission")
       import :: c_int, c_ptr
       type(c_ptr), intent(in) :: emis(*)
     end function
     integer(c_int) function olamgpu_window_forward(nsteps, nchk, flags) bind(C, name="olamgpu_window_forward")
       import :: c_int
       integer(c_int), value :: nsteps, nchk, flags
     end function
     integer(c_int) function olamgpu_window_adjoint(lam, lam_sct) bind(C, name="olamgpu_window_adjoint")
       import :: c_int, c_ptr
       type(c_ptr), intent(in) :: lam(*)
       type(c_ptr), intent(in) :: lam_sct(*)
     end function
     integer(c_int) function olamgpu_window_memory(flags, segment_steps, nsteps, nchk) &
         bind(C, name="olamgpu_window_memory")
       import :: c_int
       integer(c_int), value :: flags, segment_steps, nsteps, nchk
     end function
     integer(c_int) function olamgpu_window_rewind() bind(C, name="olamgpu_window_rewind")
       import :: c_int
     end function
     integer(c_int) function olamgpu_set_tile_shape(t, g, ks, ord) bind(C, name="olamgpu_set_tile_shape")
       import :: c_int
       integer(c_int), value :: t, g, ks, ord
     end function
     integer(c_int) function olamgpu_tile_shape(shape, nmax, cand, ms) bind(C, name="olamgpu_tile_shape")
       import :: c_int, c_float
       integer(c_int), intent(out) :: shape(4)
       integer(c_int), value :: nmax
       integer(c_int), intent(out) :: cand(*)
       real(c_float), intent(out) :: ms(*)
     end function
     integer(c_int) function olamgpu_finalize() bind(C, name="olamgpu_finalize")
       import :: c_int
     end function
     type(c_ptr) function olamgpu_strerror(status) bind(C, name="olamgpu_strerror")
       import :: c_int, c_ptr
       integer(c_int), value :: status
     end function
  end interface

contains

  ! address of an array argument (passed by reference, without a copy)
  function addr_i4(a) result(p)
    integer(c_int), target, intent(in) :: a(*)
    type(c_ptr) :: p
    p = c_loc(a)
  end function addr_i4

  function addr_r4(a) result(p)
    real(c_float), target, intent(in) :: a(*)
    type(c_ptr) :: p
    p = c_loc(a)
  end function addr_r4

  function addr_r8(a) result(p)
    real(c_double), target, intent(in) :: a(*)
    type(c_ptr) :: p
    p = c_loc(a)
  end function addr_r8

  ! OLAM stops with the library's message on any non-zero status
  subroutine olamgpu_check(rc, where)
    integer(c_int), intent(in) :: rc
    character(*),   intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    character(len=256) :: text
    integer :: i
    if (rc == OLAMGPU_OK) return
    call c_f_pointer(olamgpu_strerror(rc), msg, [256])
    text = ' '
    do i = 1, 256
       if (msg(i) == c_null_char) exit
       text(i:i) = msg(i)
    enddo
    write(*,'(3a)') 'olamgpu: ', where, ': ' // trim(text)
    stop 'olamgpu'
  end subroutine olamgpu_check

end module olamgpu_c

!===============================================================================
module olamgpu_shim

  use, intrinsic :: iso_c_binding
  use olamgpu_c
  implicit none

  private
  public :: olamgpu_shim_init, olamgpu_shim_scalars, olamgpu_shim_eddy

  ! packed copies of OLAM's derived-type tables (kept for the run)
  integer(c_int), allocatable, target, save :: npoly_p(:), iwglobe_p(:)
  integer(c_int), allocatable, target, save :: w_iv(:,:), w_iw(:,:), w_im(:,:)
  real(c_float),  allocatable, target, save :: w_dirv(:,:), w_ecx(:,:), w_ecy(:,:), w_ecz(:,:)
  integer(c_int), allocatable, target, save :: v_iw(:,:), v_im(:,:)
  real(c_float),  allocatable, target, save :: v_dxps(:,:), v_dyps(:,:)
  integer(c_int), allocatable, target, save :: m_iv(:,:), m_iw(:,:), m_im(:,:)
  integer(c_int), allocatable, target, save :: jtw_p(:), jtw_a(:), jtv_p(:), jtv_a(:), jtm_p(:)
  type(c_ptr),    allocatable, target, save :: vp(:), vt(:)
  integer(c_int), allocatable, target, save :: pdef_p(:), sgs_p(:)
  integer(c_int), allocatable, target, save :: mrlw_p(:), mrlv_p(:), idiffk_p(:)
  real(c_float),  allocatable, target, save :: akmin_p(:)

contains

  subroutine olamgpu_shim_init()
    use mem_ijtabs,  only: itab_w, itab_v, itab_m, jtab_w, jtab_v, jtab_m, &
                           jtw_prog, jtw_wadj, jtv_prog, jtv_wadj, jtm_prog
    use mem_grid,    only: mza, mwa, mva, mma, lpw, lpv, lpm, lve2, zm, zt, dzm, dzt, &
                           dzim, dzit, dzt_top, dzt_bot, zfacit, zwgt_top8, zwgt_bot8, &
                           gdz_wgtm8, gdz_wgtp8, gdz_wgtm, gdz_wgtp, wnx, wny, wnz,      &
                           wnxo2, wnyo2, wnzo2, vnx, vny, vnz, dnu, dniu, dnv, dniv,     &
                           arw0, arm0, arv, arw, volt, volti, volwi, volvi,              &
                           gxps_coef, gyps_coef
    use mem_adv,     only: a_w, a_wu, xy_h, xy_hu, xx0_v, xy0_v, yy0_v, &
                           xx0_vu, xy0_vu, yy0_vu, xx_yy, xx_yy_m
    use mem_basic,   only: rho, press, thil, wc, wmc, vxe, vye, vze, vmc, vc, vmasc, wmasc, &
                           alpha_press, pwfac, pvfac
    use mem_tend,    only: thilt, vmxet, vmyet, vmzet, vmt
    use misc_coms,   only: dtlm, dtsm, nacoust, mdomain, initial
    use oname_coms,  only: nl
    use consts_coms, only: fcoriol
    use mem_rayf,    only: rayf_cof, rayf_cofw, krayf_bot, krayfw_bot, dn01d, th01d, vc03d

    type(olamgpu_grid),  save :: g
    type(olamgpu_opts),  save :: o
    type(olamgpu_state), save :: s
    integer :: iw, iv, im

    allocate(npoly_p(mwa), iwglobe_p(mwa), w_iv(7,mwa), w_iw(7,mwa), w_im(7,mwa))
    allocate(w_dirv(7,mwa), w_ecx(7,mwa), w_ecy(7,mwa), w_ecz(7,mwa))
    allocate(v_iw(2,mva), v_im(2,mva), v_dxps(2,mva), v_dyps(2,mva))
    allocate(m_iv(3,mma), m_iw(3,mma), m_im(3,mma))
    do iw = 1, mwa
       npoly_p(iw) = itab_w(iw)%npoly;  iwglobe_p(iw) = itab_w(iw)%iwglobe
       w_iv(:,iw) = itab_w(iw)%iv;  w_iw(:,iw) = itab_w(iw)%iw;  w_im(:,iw) = itab_w(iw)%im
       w_dirv(:,iw) = itab_w(iw)%dirv
       w_ecx(:,iw) = itab_w(iw)%ecvec_vx; w_ecy(:,iw) = itab_w(iw)%ecvec_vy; w_ecz(:,iw) = itab_w(iw)%ecvec_vz
    enddo
    do iv = 1, mva
       v_iw(:,iv) = itab_v(iv)%iw;  v_im(:,iv) = itab_v(iv)%im
       v_dxps(:,iv) = itab_v(iv)%dxps;  v_dyps(:,iv) = itab_v(iv)%dyps
    enddo
    do im = 1, mma
       m_iv(:,im) = itab_m(im)%iv;  m_iw(:,im) = itab_m(im)%iw;  m_im(:,im) = itab_m(im)%im
    enddo
    jtw_p = jtab_w(jtw_prog)%iw(1:jtab_w(jtw_prog)%jend)
    jtw_a = jtab_w(jtw_wadj)%iw(1:jtab_w(jtw_wadj)%jend)
    jtv_p = jtab_v(jtv_prog)%iv(1:jtab_v(jtv_prog)%jend)
    jtv_a = jtab_v(jtv_wadj)%iv(1:jtab_v(jtv_wadj)%jend)
    jtm_p = jtab_m(jtm_prog)%im(1:jtab_m(jtm_prog)%jend)

    g%mza = mza; g%mwa = mwa; g%mva = mva; g%mma = mma
    g%nw_prog = size(jtw_p); g%jtw_prog = c_loc(jtw_p)
    g%nw_wadj = size(jtw_a); g%jtw_wadj = c_loc(jtw_a)
    g%nv_prog = size(jtv_p); g%jtv_prog = c_loc(jtv_p)
    g%nv_wadj = size(jtv_a); g%jtv_wadj = c_loc(jtv_a)
    g%nm_prog = size(jtm_p); g%jtm_prog = c_loc(jtm_p)
    g%npoly = c_loc(npoly_p); g%itab_w_iv = c_loc(w_iv); g%itab_w_iw = c_loc(w_iw)
    g%itab_w_im = c_loc(w_im); g%itab_w_dirv = c_loc(w_dirv)
    g%ecvec_vx = c_loc(w_ecx); g%ecvec_vy = c_loc(w_ecy); g%ecvec_vz = c_loc(w_ecz)
    g%iwglobe = c_loc(iwglobe_p)
    g%itab_v_iw = c_loc(v_iw); g%itab_v_im = c_loc(v_im); g%dxps = c_loc(v_dxps); g%dyps = c_loc(v_dyps)
    g%itab_m_iv = c_loc(m_iv); g%itab_m_iw = c_loc(m_iw); g%itab_m_im = c_loc(m_im)
    g%lpw = addr_i4(lpw); g%lpv = addr_i4(lpv); g%lpm = addr_i4(lpm); g%lve2 = addr_i4(lve2)
    g%zm = addr_r4(zm); g%zt = addr_r4(zt); g%dzm = addr_r4(dzm); g%dzt = addr_r4(dzt)
    g%dzim = addr_r4(dzim); g%dzit = addr_r4(dzit)
    g%dzt_top = addr_r4(dzt_top); g%dzt_bot = addr_r4(dzt_bot); g%zfacit = addr_r4(zfacit)
    g%zwgt_top8 = addr_r8(zwgt_top8); g%zwgt_bot8 = addr_r8(zwgt_bot8)
    g%gdz_wgtm8 = addr_r8(gdz_wgtm8); g%gdz_wgtp8 = addr_r8(gdz_wgtp8)
    g%gdz_wgtm = addr_r4(gdz_wgtm); g%gdz_wgtp = addr_r4(gdz_wgtp)
    g%wnx = addr_r4(wnx); g%wny = addr_r4(wny); g%wnz = addr_r4(wnz)
    g%wnxo2 = addr_r4(wnxo2); g%wnyo2 = addr_r4(wnyo2); g%wnzo2 = addr_r4(wnzo2)
    g%vnx = addr_r4(vnx); g%vny = addr_r4(vny); g%vnz = addr_r4(vnz)
    g%dnu = addr_r4(dnu); g%dniu = addr_r4(dniu); g%dnv = addr_r4(dnv); g%dniv = addr_r4(dniv)
    g%arw0 = addr_r4(arw0); g%arm0 = addr_r4(arm0)
    g%arv = addr_r4(arv); g%arw = addr_r4(arw); g%volt = addr_r8(volt)
    g%volti = addr_r4(volti); g%volwi = addr_r4(volwi); g%volvi = addr_r4(volvi)
    g%gxps_coef = addr_r4(gxps_coef); g%gyps_coef = addr_r4(gyps_coef)
    g%a_w = addr_r4(a_w); g%a_wu = addr_r4(a_wu); g%xy_h = addr_r4(xy_h); g%xy_hu = addr_r4(xy_hu)
    g%xx0_v = addr_r4(xx0_v); g%xy0_v = addr_r4(xy0_v); g%yy0_v = addr_r4(yy0_v)
    g%xx0_vu = addr_r4(xx0_vu); g%xy0_vu = addr_r4(xy0_vu); g%yy0_vu = addr_r4(yy0_vu)
    g%xx_yy = addr_r4(xx_yy); g%xx_yy_m = addr_r4(xx_yy_m)

    o%dtlm = dtlm(1); o%dtsm = dtsm(1); o%nacoust = nacoust(1)
    o%nrk_wrtv = nl%acoust_timestep_level; o%nrk_scal = nl%scalar_timestep_level
    o%thil_horiz_adv_order = nl%thil_horiz_adv_order
    o%wind_horiz_adv_order = nl%wind_horiz_adv_order
    o%scal_horiz_adv_order = nl%scal_horiz_adv_order
    o%ithil_monot = nl%ithil_monot; o%iwind_monot = nl%iwind_monot; o%iscal_monot = nl%iscal_monot
    o%divh_damp_fact = nl%divh_damp_fact; o%divh_damp_level = nl%divh_damp_level
    o%divh_damp_short = merge(1, 0, nl%divh_damp_short)
    o%vort_damp_fact = nl%vort_damp_fact; o%vort_damp_level = nl%vort_damp_level
    o%vort_damp_short = merge(1, 0, nl%vort_damp_short)
    o%fcoriol = fcoriol; o%mdomain = mdomain; o%initial = initial
    o%krayf_bot = krayf_bot; o%krayfw_bot = krayfw_bot
    o%rayf_cof = c_null_ptr; o%rayf_cofw = c_null_ptr
    o%dn01d = c_null_ptr; o%th01d = c_null_ptr; o%vc03d = c_null_ptr
    if (allocated(rayf_cof))  o%rayf_cof  = addr_r4(rayf_cof)
    if (allocated(rayf_cofw)) o%rayf_cofw = addr_r4(rayf_cofw)
    if (allocated(dn01d))     o%dn01d     = addr_r4(dn01d)
    if (allocated(th01d))     o%th01d     = addr_r4(th01d)
    if (allocated(vc03d))     o%vc03d     = addr_r4(vc03d)

    s%rho = addr_r8(rho); s%press = addr_r8(press)
    s%thil = addr_r4(thil); s%wc = addr_r4(wc); s%wmc = addr_r4(wmc)
    s%vxe = addr_r4(vxe); s%vye = addr_r4(vye); s%vze = addr_r4(vze)
    s%vmc = addr_r4(vmc); s%vc = addr_r4(vc); s%vmasc = addr_r4(vmasc); s%wmasc = addr_r4(wmasc)
    s%alpha_press = addr_r4(alpha_press); s%pwfac = addr_r4(pwfac); s%pvfac = addr_r4(pvfac)
    s%thilt = addr_r4(thilt); s%vmxet = addr_r4(vmxet); s%vmyet = addr_r4(vmyet)
    s%vmzet = addr_r4(vmzet); s%vmt = addr_r4(vmt)

    call olamgpu_check(olamgpu_init(g, o, s), 'init')
  end subroutine olamgpu_shim_init

  ! scalar_tab(1:num_scalar) as OLAM registered it (var_tables.f90:53-69);
  ! the first call registers, later calls return
  subroutine olamgpu_shim_scalars()
    use var_tables, only: scalar_tab, num_scalar
    integer :: n
    if (allocated(vp)) return
    allocate(vp(num_scalar), vt(num_scalar), pdef_p(num_scalar), sgs_p(num_scalar))
    do n = 1, num_scalar
       vp(n) = addr_r4(scalar_tab(n)%var_p)
       vt(n) = addr_r4(scalar_tab(n)%var_t)
       pdef_p(n) = merge(1, 0, scalar_tab(n)%pdef)
       sgs_p(n)  = merge(1, 0, scalar_tab(n)%do_sgsmix)
    enddo
    call olamgpu_check(olamgpu_register_scalars(int(num_scalar, c_int), vp, vt, pdef_p, sgs_p), &
                       'register_scalars')
  end subroutine olamgpu_shim_scalars

  ! eddy diffusion inside the acoustic step: mem_turb's PBL arrays and
  ! comp_horiz_k outputs, the refinement levels of itab_w / itab_v, and the
  ! namelist values solve_eddy_diff_heat / _vxe and rayf_mix_top_vxe read
  ! (pbl_driver.f90:136-238, 519-742; mem_rayf.f90:177-220).  Call once
  ! after the PBL arrays are allocated; with the RESIDENT coherence, sync
  ! OLAMGPU_F_EDDY to the device after each PBL update.
  subroutine olamgpu_shim_eddy()
    use mem_turb,    only: vkm, vkh, agamma, akm_sfc, sfluxt, kmtop, khtop, kpblh, &
                           akmodx, akhodx, kmtopv, khtopv
    use mem_basic,   only: theta, tair
    use mem_grid,    only: mwa, mva, lsw, nsw_max
    use mem_ijtabs,  only: itab_w, itab_v, mrls
    use misc_coms,   only: akmin
    use oname_coms,  only: nl
    use consts_coms, only: cp
    use mem_rayf,    only: rayf_cofmix, krayfmix_bot, dorayfmix

    type(olamgpu_eddy), save :: e
    integer :: iw, iv

    allocate(mrlw_p(mwa), mrlv_p(mva), idiffk_p(mrls), akmin_p(mrls))
    do iw = 1, mwa
       mrlw_p(iw) = max(1, itab_w(iw)%mrlw)
    enddo
    do iv = 1, mva
       mrlv_p(iv) = max(1, itab_v(iv)%mrlv)
    enddo
    idiffk_p = nl%idiffk(1:mrls)
    akmin_p = akmin(1:mrls)
    e%vkm = addr_r4(vkm); e%vkh = addr_r4(vkh); e%agamma = addr_r4(agamma)
    e%akm_sfc = addr_r4(akm_sfc); e%sfluxt = addr_r4(sfluxt)
    e%kmtop = addr_i4(kmtop); e%khtop = addr_i4(khtop); e%kpblh = addr_i4(kpblh)
    e%theta = addr_r4(theta); e%tair = addr_r4(tair)
    e%akmodx = addr_r4(akmodx); e%akhodx = addr_r4(akhodx)
    e%kmtopv = addr_i4(kmtopv); e%khtopv = addr_i4(khtopv)
    e%lsw = addr_i4(lsw); e%nsw_max = nsw_max
    e%mrlw = c_loc(mrlw_p); e%mrlv = c_loc(mrlv_p); e%mrls = mrls
    e%idiffk = c_loc(idiffk_p); e%akmin = c_loc(akmin_p)
    e%test_case = nl%test_case; e%cp = cp
    e%krayfmix_bot = krayfmix_bot
    e%rayf_cofmix = c_null_ptr
    if (dorayfmix) e%rayf_cofmix = addr_r4(rayf_cofmix)
    call olamgpu_check(olamgpu_set_eddy(e), 'set_eddy')
  end subroutine olamgpu_shim_eddy

end module olamgpu_shim
