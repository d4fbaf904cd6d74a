!-- gfx_fluid_genasis.f90 -- the GenASiS-side wrapper of the B200 fluid step:
!   a type that owns one brick's handle and offers the reference's call
!   surface on device-resident StorageForm objects,
!     ComputeIncrement  = IncrementDivergence_FV_Form % Compute
!                         ( Increment, TimeStep, Weight_RK )
!                         (IncrementDivergence_FV__Form.f90:344-412),
!     ComputeStep       = Step_RK_C_ASC_Template % Compute ( Time, TimeStep )
!                         (Step_RK_C_ASC__Template.f90:504-542),
!     ComputeTimeStep   = the integrator's ComputeTimeStepLocal
!                         (Integrator_C_PS__Form.f90:146-147, 444-459).
!   The storages hold the conserved fields D, S1, S2, S3, G, DS in that order
!   on the device (AllocateDevice, Storage_Form.f90:300-335); their
!   D_Selected ( 1 ) is the base the C functions take.  Errors are shown and
!   abort the program, as the reference does (IncrementDivergence_FV__Form.f90:
!   442-445).
!
!   Compiled with the GenASiS sources (it uses their Basics module); no
!   Fortran compiler is available to this repository, so tests/test_abi.py
!   checks its calls against include/gfx_fluid.h instead.

module GFX_FluidBox_Form

  use iso_c_binding
  use Basics
  use GFX_Fluid_C

  implicit none
  private

  type, public :: GFX_FluidBoxForm
    type ( c_ptr ) :: &
      Handle = c_null_ptr, &
      Stream = c_null_ptr
    type ( GFX_FluidConfig ) :: &
      Config
  contains
    procedure, public, pass :: &
      Initialize
    procedure, public, pass :: &
      ComputeIncrement
    procedure, public, pass :: &
      ComputeStep
    procedure, public, pass :: &
      ComputeTimeStep
    procedure, public, pass :: &
      Finalize
  end type GFX_FluidBoxForm

contains

  subroutine Initialize ( FB, Config )

    class ( GFX_FluidBoxForm ), intent ( inout ) :: &
      FB
    type ( GFX_FluidConfig ), intent ( in ) :: &
      Config

    FB % Config = Config
    call CheckStatus ( gfx_fluid_create ( FB % Config, FB % Handle ), &
                       'gfx_fluid_create' )

  end subroutine Initialize


  subroutine ComputeIncrement ( FB, Solution, Increment, TimeStep, Weight_RK )

    class ( GFX_FluidBoxForm ), intent ( inout ) :: &
      FB
    type ( StorageForm ), intent ( in ) :: &
      Solution
    type ( StorageForm ), intent ( inout ) :: &
      Increment  !-- assumed cleared, as the reference assumes
    real ( KDR ), intent ( in ) :: &
      TimeStep, &
      Weight_RK

    call CheckStatus &
           ( gfx_fluid_increment &
               ( FB % Handle, Solution % D_Selected ( 1 ), &
                 Increment % D_Selected ( 1 ), real ( TimeStep, c_double ), &
                 real ( Weight_RK, c_double ), c_null_ptr, FB % Stream ), &
             'gfx_fluid_increment' )

  end subroutine ComputeIncrement


  subroutine ComputeStep ( FB, Solution, Time, TimeStep )

    class ( GFX_FluidBoxForm ), intent ( inout ) :: &
      FB
    type ( StorageForm ), intent ( inout ) :: &
      Solution
    real ( KDR ), intent ( in ) :: &
      Time, &
      TimeStep

    !-- the RK2 stages of this fluid do not depend on Time
    call CheckStatus &
           ( gfx_fluid_step &
               ( FB % Handle, Solution % D_Selected ( 1 ), &
                 real ( TimeStep, c_double ), c_null_ptr, FB % Stream ), &
             'gfx_fluid_step' )

  end subroutine ComputeStep


  subroutine ComputeTimeStep ( FB, Solution, iCycle, TimeStep )

    class ( GFX_FluidBoxForm ), intent ( inout ) :: &
      FB
    type ( StorageForm ), intent ( in ) :: &
      Solution
    integer ( KDI ), intent ( in ) :: &
      iCycle
    real ( KDR ), intent ( out ) :: &
      TimeStep

    real ( c_double ) :: &
      dt

    call CheckStatus &
           ( gfx_fluid_timestep &
               ( FB % Handle, Solution % D_Selected ( 1 ), int ( iCycle, c_int ), &
                 dt, FB % Stream ), &
             'gfx_fluid_timestep' )
    TimeStep = dt

  end subroutine ComputeTimeStep


  subroutine Finalize ( FB )

    class ( GFX_FluidBoxForm ), intent ( inout ) :: &
      FB

    if ( c_associated ( FB % Handle ) ) &
      call CheckStatus ( gfx_fluid_destroy ( FB % Handle ), 'gfx_fluid_destroy' )
    FB % Handle = c_null_ptr

  end subroutine Finalize


  subroutine CheckStatus ( Status, Where )

    integer ( c_int ), intent ( in ) :: &
      Status
    character ( * ), intent ( in ) :: &
      Where

    character ( kind = c_char ) :: &
      Message ( 512 )
    character ( 512 ) :: &
      Text
    integer ( c_int ) :: &
      Ignore
    integer :: &
      iC

    if ( Status == GFX_OK ) &
      return
    Ignore = gfx_fluid_last_error ( Message, 512_c_size_t )
    Text = ''
    do iC = 1, 512
      if ( Message ( iC ) == c_null_char ) &
        exit
      Text ( iC : iC ) = Message ( iC )
    end do
    call Show ( trim ( Text ), Where, CONSOLE % ERROR )
    call PROGRAM_HEADER % Abort ( )

  end subroutine CheckStatus

end module GFX_FluidBox_Form
