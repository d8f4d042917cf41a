! ISO_C_BINDING interface of libfinflo_gpu.so for a FINFLO host (Fortran 2003).
!
! The derived types match include/finflo_types.h field for field (bind(C)
! gives them the C layout); the interfaces bind the C-ABI of
! include/finflo_gpu.h under their own names.  Every function returns 0 or
! an FF_ERR_* code (the reference STOPs instead, e.g. ns3c.f:2209-2217).
!
! Two ways to call the library from a FINFLO host:
!  * the stage functions below (ff_statim, ff_residi, ff_imps, ff_fin,
!    ff_boundi, ff_transf, ff_forcfu, ff_addres, ff_interp, or ff_cycles for
!    whole cycles), with a context and block ids;
!  * the external subroutines statim_, residi_, impsdi_, fin_ and boundi_
!    the library also exports: linked in place of the CPU routines, the
!    existing CALL STATIM(1,N,0,.TRUE.), CALL RESIDI(1,N,1,IPRINT), CALL
!    IMPSDI(1,N,1,AMGDIVL), CALL FIN(...) and CALL BOUNDI(1) of CYCLES
!    (ns3c.f:1450, 1484, 1497, 1517, 556) reach the device unchanged once
!    ff_fortran_bind and ff_fortran_block have been called.
!
! Slots (enum ff_slot) are 0-based indices; the named constants below give
! the ones a host uploads and downloads.
module finflo_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: FF_ABI_VERSION = 7
  integer(c_int), parameter :: FF_OK = 0, FF_ERR_CUDA = 1, FF_ERR_ARG = 2, &
                               FF_ERR_TIMEOUT = 3, FF_ERR_SIZE = 4
  integer(c_int), parameter :: FF_BC_CON = 1, FF_BC_INL = 3, FF_BC_MIR = 4, &
                               FF_BC_OUT = 5, FF_BC_SOL = 8
  ! ff_params%flux (enum ff_flux): a host with IFLUX sets
  ! flux = merge(FF_FLUX_ROE, merge(FF_FLUX_VANLEER, IFLUX, IFLUX == 0), IFLUX == 1)
  integer(c_int), parameter :: FF_FLUX_ROE = 0, FF_FLUX_VANLEER = 1, FF_FLUX_WPS = 2, &
                               FF_FLUX_AUSM = 3, FF_FLUX_KT = 7, FF_FLUX_HCUSP = 8

  ! ICON(IC9,L) columns of one patch (charac.f:182) and its boundary values
  type, bind(C) :: ff_patch
    integer(c_int) :: ityp, iface
    integer(c_int) :: r1a, r1b, r2a, r2b
    integer(c_int) :: ibtype, iheat
    integer(c_int) :: nface, iori
    integer(c_int) :: n1a, n2a
    real(c_double) :: bounr, bounu, bounv, bounw, bount, bounp, bounpd
    real(c_double) :: bounrk, bounep
  end type ff_patch

  ! flow, gas and solver constants (main.f:5234-5440, 3499)
  type, bind(C) :: ff_params
    real(c_double) :: gamma, rgas, pr, prt
    real(c_double) :: visu0, expsu, tsu0
    real(c_double) :: e0ref, t0ref
    real(c_double) :: frsden, frspre, frsvel, frsvis, frstem
    real(c_double) :: cfl, cfll
    real(c_double) :: theta
    real(c_double) :: cdiff
    real(c_double) :: pvisc
    real(c_double) :: tlolim, tuplim
    real(c_double) :: cmgk, cmgeps
    real(c_double) :: rklim, epslim
    real(c_double) :: turlim
    real(c_double) :: csimps
    real(c_double) :: re
    integer(c_int) :: interi, interj, interk
    integer(c_int) :: entropy_fix
    integer(c_int) :: iturb
    integer(c_int) :: fullns
    integer(c_int) :: idi1, idi2, idi3
    integer(c_int) :: coarse_inter
    integer(c_int) :: lusgs_fp32
    integer(c_int) :: ddadi
    integer(c_int) :: timel
    integer(c_int) :: flux
    real(c_double) :: dt
    integer(c_int) :: predgs_full
    integer(c_int) :: res_fp32
    integer(c_int) :: xxtral
    real(c_double) :: rjk2, rjk4
  end type ff_params

  ! slot indices (enum ff_slot, include/finflo_types.h)
  integer(c_int), parameter :: FF_RO = 0, FF_RM = 1, FF_RN = 2, FF_RW = 3, FF_E = 4, &
    FF_P = 5, FF_PDIFF = 6, FF_U = 7, FF_V = 8, FF_W = 9, FF_C = 10, FF_TEMP = 11, &
    FF_VIS = 12, FF_CH = 13, FF_CP = 14, FF_DRDP = 15, FF_DRDH = 16, FF_EPS2 = 17, &
    FF_VIST = 18, FF_DRO = 19, FF_DM = 20, FF_DN = 21, FF_DW = 22, FF_DE = 23, &
    FF_DRK = 24, FF_DEPS = 25, FF_DTL = 26, FF_TOLD = 27, FF_UOLD = 28, FF_VOLD = 29, &
    FF_WOLD = 30, FF_POLD = 31, FF_A1 = 32, FF_VOL = 44, FF_XC = 45, FF_D1 = 48, &
    FF_RK = 75, FF_REPS = 76, FF_DISTW = 77, FF_RKOLD = 88, FF_EPSOLD = 89, &
    FF_ROLE2 = 94, FF_ROLE3 = 101, FF_SCALEJ = 108, FF_NSLOTS = 109

  interface
    integer(c_int) function ff_abi_version() bind(C, name="ff_abi_version")
      import :: c_int
    end function
    integer(c_int) function ff_create(ctx, device) bind(C, name="ff_create")
      import :: c_int, c_ptr
      type(c_ptr), intent(out) :: ctx
      integer(c_int), value :: device
    end function
    integer(c_int) function ff_destroy(ctx) bind(C, name="ff_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ff_block_add(ctx, imax, jmax, kmax, npatch, patches, prm) &
        bind(C, name="ff_block_add")
      import :: c_int, c_ptr, ff_patch, ff_params
      type(c_ptr), value :: ctx
      integer(c_int), value :: imax, jmax, kmax, npatch
      type(ff_patch), intent(in) :: patches(*)
      type(ff_params), intent(in) :: prm
    end function
    integer(c_int) function ff_block_params(ctx, blk, prm) bind(C, name="ff_block_params")
      import :: c_int, c_ptr, ff_params
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
      type(ff_params), intent(in) :: prm
    end function
    integer(c_int) function ff_mg_link(ctx, fine, coarse) bind(C, name="ff_mg_link")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: fine, coarse
    end function
    ! one slot of a block: NTOT = (IMAX+4)(JMAX+4)(KMAX+4) values, e.g. TEMP(IG1)
    integer(c_int) function ff_upload(ctx, blk, slot, host) bind(C, name="ff_upload")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, slot
      real(c_double), intent(in) :: host(*)
    end function
    integer(c_int) function ff_download(ctx, blk, slot, host) bind(C, name="ff_download")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, slot
      real(c_double), intent(out) :: host(*)
    end function
    integer(c_int) function ff_synchronize(ctx) bind(C, name="ff_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ff_statim(ctx, blk) bind(C, name="ff_statim")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
    end function
    integer(c_int) function ff_boundi(ctx, blk) bind(C, name="ff_boundi")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
    end function
    integer(c_int) function ff_boundi_all(ctx) bind(C, name="ff_boundi_all")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ff_residu(ctx, blk, level, icycle) bind(C, name="ff_residu")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, level, icycle
    end function
    integer(c_int) function ff_residi(ctx, blk, m2, icycle) bind(C, name="ff_residi")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, m2, icycle
    end function
    integer(c_int) function ff_resl2(ctx, blk, out5) bind(C, name="ff_resl2")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
      real(c_double), intent(out) :: out5(5)
    end function
    integer(c_int) function ff_imps(ctx, blk, level) bind(C, name="ff_imps")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, level
    end function
    integer(c_int) function ff_fin(ctx, blk, dromax) bind(C, name="ff_fin")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
      real(c_double), intent(out) :: dromax
    end function
    integer(c_int) function ff_transf(ctx, fine, coarse) bind(C, name="ff_transf")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: fine, coarse
    end function
    integer(c_int) function ff_forcfu(ctx, blk) bind(C, name="ff_forcfu")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
    end function
    integer(c_int) function ff_addres(ctx, blk) bind(C, name="ff_addres")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk
    end function
    integer(c_int) function ff_interp(ctx, coarse, fine) bind(C, name="ff_interp")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: coarse, fine
    end function
    integer(c_int) function ff_cycles(ctx, blk, ncycles, icycle0, hist, use_graph) &
        bind(C, name="ff_cycles")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, ncycles, icycle0, use_graph
      real(c_double), intent(out) :: hist(6, *)
    end function
    integer(c_int) function ff_cycles_all(ctx, ncycles, icycle0, hist, use_graph) &
        bind(C, name="ff_cycles_all")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ncycles, icycle0, use_graph
      real(c_double), intent(out) :: hist(6, *)
    end function
    integer(c_int) function ff_time_levels(ctx, blk, mode) bind(C, name="ff_time_levels")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: blk, mode
    end function
    ! the table the gfortran-named wrappers (statim_, residi_, impsdi_,
    ! fin_, boundi_) use
    integer(c_int) function ff_fortran_bind(ctx) bind(C, name="ff_fortran_bind")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function ff_fortran_block(m, n, ngl, blk) bind(C, name="ff_fortran_block")
      import :: c_int
      integer(c_int), value :: m, n, ngl, blk
    end function
    integer(c_int) function ff_fortran_cycle(icycle) bind(C, name="ff_fortran_cycle")
      import :: c_int
      integer(c_int), value :: icycle
    end function
    integer(c_int) function ff_fortran_ierr() bind(C, name="ff_fortran_ierr")
      import :: c_int
    end function
  end interface
end module finflo_gpu
