! tiger_chem_gpu.f90 -- ISO_C_BINDING interface to libtiger_chem.so and a drop-in GPU
! replacement for the finite-rate chemistry substep of the host solver.
!
! Replaces finitechem_source_chemistry(RHO_, SC_) (combustion/finitechem.f90:962-1071). To use
! it, link libtiger_chem.so, call tiger_chem_gpu_init once after finitechem_init (which has
! found isc_sc and the H2O/CO/CO2 indices, finitechem.f90:218-251) and call
! finitechem_source_chemistry_gpu where combustion_source_scalar_full calls
! finitechem_source_chemistry (combustion.f90:1047-1049). The mechanism is chosen by name at
! run time instead of by the linked *F.f90 file (combustion/Makefile:3-5).
! The mixture-property routines around the substep have drop-ins too: finitechem_density_gpu
! (for finitechem_density, combustion.f90:1098 and :1149), finitechem_viscosity_gpu
! (:1197) and finitechem_diffusivity_gpu (:1305), or finitechem_transport_gpu for both.
module tiger_chem_gpu
  use iso_c_binding
  implicit none
  private
  public :: tiger_chem_gpu_init, finitechem_source_chemistry_gpu, tiger_chem_gpu_finalize
  public :: finitechem_density_gpu, finitechem_viscosity_gpu, finitechem_diffusivity_gpu, finitechem_transport_gpu
  public :: tng_cfg, tng_extent, tng_default_cfg, tng_chem_create, tng_chem_destroy, tng_chem_substep
  public :: tng_prodrates_batch, tng_last_error

  integer(c_int), parameter, public :: TNG_OK = 0, TNG_DEVICE_PTRS = 0, TNG_HOST_PTRS = 1
  integer(c_int), parameter, public :: TNG_FP64 = 0, TNG_MIXED = 1, TNG_LIT_REF = 0, TNG_LIT_F64 = 1

  type, bind(C) :: tng_cfg
    integer(c_int) :: precision, literal_mode, device
    real(c_double) :: rtol, atol
    integer(c_int) :: max_steps, max_newton, block_size, rate_variant
    integer(c_int) :: solver_warps, pass_budget, max_passes
    integer(c_int) :: solver_occupancy
    integer(c_int) :: reserved(3)
  end type tng_cfg

  type, bind(C) :: tng_extent
    integer(c_int) :: imino, imaxo, jmino, jmaxo, kmino, kmaxo
    integer(c_int) :: imin, imax, jmin, jmax, kmin, kmax
    integer(c_int) :: nscalar, isc_sc, isc_T
    integer(c_int) :: isc_H2O, isc_CO, isc_CO2
  end type tng_extent

  interface
    subroutine tng_default_cfg(cfg) bind(C, name='tng_default_cfg')
      import :: tng_cfg
      type(tng_cfg), intent(out) :: cfg
    end subroutine tng_default_cfg

    integer(c_int) function tng_chem_create(mechanism, cfg, h) bind(C, name='tng_chem_create')
      import :: c_int, c_char, c_ptr, tng_cfg
      character(kind=c_char), dimension(*), intent(in) :: mechanism
      type(tng_cfg), intent(in) :: cfg
      type(c_ptr), intent(out) :: h
    end function tng_chem_create

    integer(c_int) function tng_chem_destroy(h) bind(C, name='tng_chem_destroy')
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function tng_chem_destroy

    integer(c_int) function tng_chem_substep(h, rho, sc, mask, ext, dt, p_mid, hr, chemsrc, flags, stats) &
         bind(C, name='tng_chem_substep')
      import :: c_int, c_double, c_ptr, tng_extent
      type(c_ptr), value :: h
      real(c_double), dimension(*), intent(in) :: rho
      real(c_double), dimension(*), intent(inout) :: sc
      ! mask, hr and chemsrc may be left out: an absent optional argument of a bind(C)
      ! interface is passed as a null pointer (Fortran 2018), which the C side reads as
      ! "no mask" / "no diagnostics"
      integer(c_int), dimension(*), intent(in), optional :: mask
      type(tng_extent), intent(in) :: ext
      real(c_double), value :: dt, p_mid
      real(c_double), dimension(*), intent(inout), optional :: hr, chemsrc
      integer(c_int), value :: flags
      type(c_ptr), value :: stats
    end function tng_chem_substep

    integer(c_int) function tng_chem_density(h, rho, wmix, sc, mask, ext, p_thermo, flags) &
         bind(C, name='tng_chem_density')
      import :: c_int, c_double, c_ptr, tng_extent
      type(c_ptr), value :: h, rho, wmix
      real(c_double), dimension(*), intent(in) :: sc
      integer(c_int), dimension(*), intent(in), optional :: mask  ! absent: no mask (null)
      type(tng_extent), intent(in) :: ext
      real(c_double), value :: p_thermo
      integer(c_int), value :: flags
    end function tng_chem_density

    integer(c_int) function tng_chem_transport(h, visc, diff, sc, mask, ext, lewis, isc_zmix, flags) &
         bind(C, name='tng_chem_transport')
      import :: c_int, c_double, c_ptr, tng_extent
      type(c_ptr), value :: h, visc, diff
      real(c_double), dimension(*), intent(in) :: sc
      integer(c_int), dimension(*), intent(in), optional :: mask  ! absent: no mask (null)
      type(tng_extent), intent(in) :: ext
      type(c_ptr), value :: lewis
      integer(c_int), value :: isc_zmix, flags
    end function tng_chem_transport

    integer(c_int) function tng_prodrates_batch(h, sol, rhs, ncells, ld, p, flags) bind(C, name='tng_prodrates_batch')
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      real(c_double), dimension(*), intent(in) :: sol
      real(c_double), dimension(*), intent(out) :: rhs
      integer(c_int64_t), value :: ncells, ld
      real(c_double), value :: p
      integer(c_int), value :: flags
    end function tng_prodrates_batch

    integer(c_int) function tng_last_error(buf, length) bind(C, name='tng_last_error')
      import :: c_int, c_char
      character(kind=c_char), dimension(*) :: buf
      integer(c_int), value :: length
    end function tng_last_error
  end interface

  type(c_ptr), save :: handle = c_null_ptr

contains

  ! Create the GPU handle for the mechanism (e.g. 'grimech30') with the finitechem
  ! tolerances ('Finitechem rel. tol.' / 'abs. tol.', finitechem.f90:266-267).
  subroutine tiger_chem_gpu_init(mechanism, rtol, atol, device)
    character(len=*), intent(in) :: mechanism
    real(c_double), intent(in) :: rtol, atol
    integer, intent(in) :: device
    type(tng_cfg) :: cfg
    integer(c_int) :: rc
    call tng_default_cfg(cfg)
    cfg%rtol = rtol
    cfg%atol = atol
    cfg%device = device
    rc = tng_chem_create(trim(mechanism)//c_null_char, cfg, handle)
    if (rc /= TNG_OK) call report('tng_chem_create')
  end subroutine tiger_chem_gpu_init

  subroutine tiger_chem_gpu_finalize()
    integer(c_int) :: rc
    if (c_associated(handle)) rc = tng_chem_destroy(handle)
    handle = c_null_ptr
  end subroutine tiger_chem_gpu_finalize

  ! Same arguments and effect as finitechem_source_chemistry (finitechem.f90:962-1071),
  ! including HR_gp and chemsrc_gp; 'Cold flow' is honoured as in the reference (:983-984).
  subroutine finitechem_source_chemistry_gpu(RHO_, SC_)
    use finitechem
    use time_info
    use masks
    use parser
    real(WP), dimension(imino_:imaxo_, jmino_:jmaxo_, kmino_:kmaxo_), intent(inout) :: RHO_
    real(WP), dimension(imino_:imaxo_, jmino_:jmaxo_, kmino_:kmaxo_, nscalar), intent(inout) :: SC_
    type(tng_extent) :: ext
    integer(c_int) :: rc
    call parser_read('Cold flow', coldflow, .false.)
    if (coldflow) return
    ext = tng_extent(imino_, imaxo_, jmino_, jmaxo_, kmino_, kmaxo_, imin_, imax_, jmin_, jmax_, kmin_, kmax_, &
         nscalar, isc_sc, isc_T, isc_H2O, isc_CO, isc_CO2)
    ! mask is allocated on the global index range (geometry/masks.f90:55); pass this rank's part
    rc = tng_chem_substep(handle, RHO_, SC_, mask(imino_:imaxo_, jmino_:jmaxo_), ext, dt, &
         0.5_WP * (P_thermo + P_thermo_old), HR_gp, chemsrc_gp, TNG_HOST_PTRS, c_null_ptr)
    if (rc /= TNG_OK) call report('tng_chem_substep')
  end subroutine finitechem_source_chemistry_gpu

  ! The padded block of this rank with the species / temperature columns of SC.
  function block_extent() result(ext)
    use finitechem
    type(tng_extent) :: ext
    ext = tng_extent(imino_, imaxo_, jmino_, jmaxo_, kmino_, kmaxo_, imin_, imax_, jmin_, jmax_, kmin_, kmax_, &
         nscalar, isc_sc, isc_T, 0, 0, 0)
  end function block_extent

  ! Same effect as finitechem_density (finitechem.f90:324-345): RHO of every unmasked cell of
  ! the padded block from the equation of state.
  subroutine finitechem_density_gpu
    use finitechem
    use masks
    integer(c_int) :: rc
    rc = tng_chem_density(handle, c_loc(RHO), c_null_ptr, SC, mask(imino_:imaxo_, jmino_:jmaxo_), block_extent(), &
         P_thermo, TNG_HOST_PTRS)
    if (rc /= TNG_OK) call report('tng_chem_density')
  end subroutine finitechem_density_gpu

  ! Same effect as finitechem_viscosity (finitechem.f90:351-406), border update included.
  subroutine finitechem_viscosity_gpu
    use finitechem
    use masks
    integer(c_int) :: rc
    rc = tng_chem_transport(handle, c_loc(VISC), c_null_ptr, SC, mask(imino_:imaxo_, jmino_:jmaxo_), block_extent(), &
         c_loc(Lewis), 0_c_int, TNG_HOST_PTRS)
    if (rc /= TNG_OK) call report('tng_chem_transport')
    call boundary_update_border(VISC, '+', 'ym')
  end subroutine finitechem_viscosity_gpu

  ! Same effect as finitechem_diffusivity (finitechem.f90:412-461), border update included.
  subroutine finitechem_diffusivity_gpu
    use finitechem
    use masks
    integer(c_int) :: rc
    rc = tng_chem_transport(handle, c_null_ptr, c_loc(DIFF), SC, mask(imino_:imaxo_, jmino_:jmaxo_), block_extent(), &
         c_loc(Lewis), int(isc_ZMIX, c_int), TNG_HOST_PTRS)
    if (rc /= TNG_OK) call report('tng_chem_transport')
    call boundary_update_border(DIFF, '+', 'ym')
  end subroutine finitechem_diffusivity_gpu

  ! Both of the above in one pass over SC (combustion_prestep calls them back to back,
  ! combustion.f90:686-687).
  subroutine finitechem_transport_gpu
    use finitechem
    use masks
    integer(c_int) :: rc
    rc = tng_chem_transport(handle, c_loc(VISC), c_loc(DIFF), SC, mask(imino_:imaxo_, jmino_:jmaxo_), &
         block_extent(), c_loc(Lewis), int(isc_ZMIX, c_int), TNG_HOST_PTRS)
    if (rc /= TNG_OK) call report('tng_chem_transport')
    call boundary_update_border(VISC, '+', 'ym')
    call boundary_update_border(DIFF, '+', 'ym')
  end subroutine finitechem_transport_gpu

  subroutine report(what)
    character(len=*), intent(in) :: what
    character(kind=c_char) :: buf(512)
    character(len=512) :: msg
    integer(c_int) :: n
    integer :: i
    n = tng_last_error(buf, 512_c_int)
    msg = ''
    do i = 1, min(int(n), 511)
      msg(i:i) = buf(i)
    end do
    call die(what // ': ' // trim(msg))
  end subroutine report

end module tiger_chem_gpu
