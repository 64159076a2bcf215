!===============================================================================
! olamgpu_modules.f90 -- drop-in replacements for OLAM's wrtv_rk and
! scalar_transport modules (omodel/prog_wrtv_rk.f90:29-30,
! omodel/scalar_transport_rk.F90:23-24): same module names, same public
! procedures and arguments, bodies that call the B200 library.  Compile
! these instead of omodel/prog_wrtv_rk.f90 and omodel/scalar_transport_rk.F90
! and link libolamgpu.so.  The calls in timestep.f90 (:205, :254) and
! olam_run.f90 (:566) stay as they are.
!
! Source for the OLAM build; not compiled in this repository (no Fortran
! compiler in the build image).
!===============================================================================
module wrtv_rk

  use, intrinsic :: iso_c_binding
  use olamgpu_c
  implicit none

  private
  public :: init_wrtv_rk, prog_wrtv_rk

contains

  ! omodel/prog_wrtv_rk.f90:36-54; called once at olam_run.f90:566
  subroutine init_wrtv_rk()
    use olamgpu_shim, only: olamgpu_shim_init
    call olamgpu_shim_init()
  end subroutine init_wrtv_rk

  ! omodel/prog_wrtv_rk.f90:58-488; called nacoust times per long step
  subroutine prog_wrtv_rk()
    use mem_ijtabs,   only: istp
    use olamgpu_shim, only: olamgpu_shim_scalars
    call olamgpu_shim_scalars()   ! var_tables is complete once the model runs
    call olamgpu_check(olamgpu_prog_wrtv_rk(int(istp, c_int)), 'prog_wrtv_rk')
  end subroutine prog_wrtv_rk

end module wrtv_rk

!===============================================================================
module scalar_transport

  use, intrinsic :: iso_c_binding
  use olamgpu_c
  implicit none

  private
  public :: scalar_transport_rk

contains

  ! omodel/scalar_transport_rk.F90:30-385
  subroutine scalar_transport_rk(rho_old)
    use mem_grid,     only: mza, mwa
    use olamgpu_shim, only: olamgpu_shim_scalars
    real, intent(in) :: rho_old(mza,mwa)
    call olamgpu_shim_scalars()
    call olamgpu_check(olamgpu_scalar_transport_rk(rho_old, c_null_ptr), 'scalar_transport_rk')
  end subroutine scalar_transport_rk

end module scalar_transport
