!-- gfx_fluid_f.f90 -- ISO_C_BINDING interfaces to include/gfx_fluid.h, for
!   the GenASiS side of the drop-in (Fortran 2008).  Every function returns
!   the C status (GFX_OK = 0, negative on error); pointers are type ( c_ptr )
!   passed by value: device pointers for *_dev arguments (for a StorageForm
!   on the device, its D_Selected ( 1 ): Storage_Form.f90:300-335), host
!   pointers for *_host (c_loc of a contiguous array).  `stream` is a
!   cudaStream_t or c_null_ptr for the default stream.
!
!   Not compiled in this repository (no Fortran compiler is available to it);
!   it is checked against the C header by tests/test_abi.py (names, argument
!   counts and the layout of gfx_fluid_config).

module GFX_Fluid_C

  use iso_c_binding

  implicit none
  private

  integer ( c_int ), parameter, public :: &
    GFX_OK = 0, &
    GFX_ERR_ARGUMENT = -1, &
    GFX_ERR_CUDA = -2, &
    GFX_ERR_UNSUPPORTED = -3, &
    GFX_ERR_STATE = -4, &
    GFX_ERR_TIMEOUT = -5, &
    GFX_ERR_NO_MEMORY = -6, &
    GFX_BC_OUTFLOW = 0, &
    GFX_BC_REFLECTING = 1, &
    GFX_BC_PERIODIC = 2, &
    GFX_RIEMANN_HLL = 0, &
    GFX_RIEMANN_HLLC = 1, &
    GFX_RECONSTRUCTION_LINEAR = 0, &
    GFX_RECONSTRUCTION_PARABOLIC = 1

  !-- gfx_fluid_config; Boundary ( iSide, iDimension ) is the C
  !   boundary[iDimension][iSide] (row-major there, column-major here)
  type, bind ( c ), public :: GFX_FluidConfig
    integer ( c_int ) :: nCells ( 3 )
    integer ( c_int ) :: nGhostLayers
    real ( c_double ) :: MinCoordinate ( 3 )
    real ( c_double ) :: MaxCoordinate ( 3 )
    integer ( c_int ) :: Boundary ( 2, 3 )
    integer ( c_int ) :: RiemannSolver
    integer ( c_int ) :: UseLimiter
    real ( c_double ) :: LimiterParameter
    real ( c_double ) :: AdiabaticIndex
    real ( c_double ) :: ShockThreshold
    real ( c_double ) :: CourantFactor
    real ( c_double ) :: BaryonDensityMin
    real ( c_double ) :: UniformAcceleration
    integer ( c_int ) :: nRampCycles
    integer ( c_int ) :: ReconstructionType  !-- GFX_RECONSTRUCTION_*
  end type GFX_FluidConfig

  public :: &
    gfx_fluid_config_default, gfx_fluid_create, gfx_fluid_destroy, &
    gfx_fluid_n_values, gfx_fluid_geometry, gfx_fluid_from_primitive, &
    gfx_fluid_to_primitive, gfx_fluid_detect_features, &
    gfx_fluid_clear_features, gfx_fluid_get_features, gfx_fluid_increment, &
    gfx_fluid_fluence_face_size, gfx_fluid_step, gfx_fluid_step_sources, &
    gfx_fluid_step_host, &
    gfx_fluid_timestep, gfx_fluid_evolve, gfx_fluid_evolve_timed, gfx_fluid_step_timed, &
    gfx_fluid_kernel_launches, gfx_fluid_step_adjoint, gfx_fluid_step_branches, &
    gfx_fluid_set_tuning, gfx_fluid_batch_create, gfx_fluid_batch_destroy, &
    gfx_fluid_batch_set_clocks, gfx_fluid_batch_evolve, &
    gfx_fluid_batch_clocks, gfx_fluid_batch_kernel_launches, &
    gfx_fluid_step_noalloc, gfx_fluid_check_state, gfx_fluid_totals, &
    gfx_fluid_resume, gfx_fluid_chart_create, gfx_fluid_chart_destroy, &
    gfx_fluid_chart_n_bricks, gfx_fluid_chart_brick, gfx_fluid_chart_bind, &
    gfx_fluid_chart_from_primitive, gfx_fluid_chart_set_conserved, &
    gfx_fluid_chart_timestep, gfx_fluid_chart_step, gfx_fluid_chart_evolve, &
    gfx_fluid_chart_kernel_launches, gfx_fluid_last_error, &
    gfx_fluid_debug_fail_allocation

  interface

    integer ( c_int ) function gfx_fluid_config_default ( Config ) &
      bind ( c, name = 'gfx_fluid_config_default' )
      import
      type ( GFX_FluidConfig ), intent ( out ) :: Config
    end function gfx_fluid_config_default

    integer ( c_int ) function gfx_fluid_create ( Config, Handle ) &
      bind ( c, name = 'gfx_fluid_create' )
      import
      type ( GFX_FluidConfig ), intent ( in ) :: Config
      type ( c_ptr ), intent ( out ) :: Handle
    end function gfx_fluid_create

    integer ( c_int ) function gfx_fluid_destroy ( Handle ) &
      bind ( c, name = 'gfx_fluid_destroy' )
      import
      type ( c_ptr ), value :: Handle
    end function gfx_fluid_destroy

    integer ( c_int ) function gfx_fluid_n_values ( Handle, nValues ) &
      bind ( c, name = 'gfx_fluid_n_values' )
      import
      type ( c_ptr ), value :: Handle
      integer ( c_size_t ), intent ( out ) :: nValues
    end function gfx_fluid_n_values

    integer ( c_int ) function gfx_fluid_geometry &
      ( Handle, iDimension, Center_host, WidthLeft_host, WidthRight_host ) &
      bind ( c, name = 'gfx_fluid_geometry' )
      import
      type ( c_ptr ), value :: Handle, Center_host, WidthLeft_host, WidthRight_host
      integer ( c_int ), value :: iDimension  !-- 0, 1, 2
    end function gfx_fluid_geometry

    integer ( c_int ) function gfx_fluid_from_primitive &
      ( Handle, Primitive_dev, Conserved_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_from_primitive' )
      import
      type ( c_ptr ), value :: Handle, Primitive_dev, Conserved_dev, Stream
    end function gfx_fluid_from_primitive

    integer ( c_int ) function gfx_fluid_to_primitive &
      ( Handle, Conserved_dev, Primitive_dev, Auxiliary_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_to_primitive' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Primitive_dev, Auxiliary_dev, Stream
    end function gfx_fluid_to_primitive

    integer ( c_int ) function gfx_fluid_detect_features &
      ( Handle, Conserved_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_detect_features' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Stream
    end function gfx_fluid_detect_features

    integer ( c_int ) function gfx_fluid_clear_features ( Handle, Stream ) &
      bind ( c, name = 'gfx_fluid_clear_features' )
      import
      type ( c_ptr ), value :: Handle, Stream
    end function gfx_fluid_clear_features

    integer ( c_int ) function gfx_fluid_get_features ( Handle, Flags_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_get_features' )
      import
      type ( c_ptr ), value :: Handle, Flags_dev, Stream
    end function gfx_fluid_get_features

    integer ( c_int ) function gfx_fluid_increment &
      ( Handle, Conserved_dev, Increment_dev, TimeStep, Weight_RK, Fluence_dev, &
        Stream ) &
      bind ( c, name = 'gfx_fluid_increment' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Increment_dev, Fluence_dev, Stream
      real ( c_double ), value :: TimeStep, Weight_RK
    end function gfx_fluid_increment

    integer ( c_int ) function gfx_fluid_fluence_face_size ( Handle, FaceSize ) &
      bind ( c, name = 'gfx_fluid_fluence_face_size' )
      import
      type ( c_ptr ), value :: Handle
      integer ( c_size_t ), intent ( out ) :: FaceSize
    end function gfx_fluid_fluence_face_size

    integer ( c_int ) function gfx_fluid_step &
      ( Handle, Conserved_dev, TimeStep, Fluence_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_step' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Fluence_dev, Stream
      real ( c_double ), value :: TimeStep
    end function gfx_fluid_step

    integer ( c_int ) function gfx_fluid_step_sources &
      ( Handle, Conserved_dev, TimeStep, Fluence_dev, Sources_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_step_sources' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Fluence_dev, Sources_dev, Stream
      real ( c_double ), value :: TimeStep
    end function gfx_fluid_step_sources

    integer ( c_int ) function gfx_fluid_step_host &
      ( Handle, Conserved_host, TimeStep, Fluence_host ) &
      bind ( c, name = 'gfx_fluid_step_host' )
      import
      type ( c_ptr ), value :: Handle, Conserved_host, Fluence_host
      real ( c_double ), value :: TimeStep
    end function gfx_fluid_step_host

    integer ( c_int ) function gfx_fluid_timestep &
      ( Handle, Conserved_dev, iCycle, TimeStep, Stream ) &
      bind ( c, name = 'gfx_fluid_timestep' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Stream
      integer ( c_int ), value :: iCycle
      real ( c_double ), intent ( out ) :: TimeStep
    end function gfx_fluid_timestep

    integer ( c_int ) function gfx_fluid_evolve &
      ( Handle, Conserved_dev, Time, iCycle, FinishTime, nCyclesMax, TimeOut, &
        iCycleOut, Stream ) &
      bind ( c, name = 'gfx_fluid_evolve' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Stream
      real ( c_double ), value :: Time, FinishTime
      integer ( c_int ), value :: iCycle, nCyclesMax
      real ( c_double ), intent ( out ) :: TimeOut
      integer ( c_int ), intent ( out ) :: iCycleOut
    end function gfx_fluid_evolve

    integer ( c_int ) function gfx_fluid_evolve_timed &
      ( Handle, Conserved_dev, Time, iCycle, FinishTime, nCyclesMax, TimeOut, &
        iCycleOut, DeviceMilliseconds, Stream ) &
      bind ( c, name = 'gfx_fluid_evolve_timed' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Stream
      real ( c_double ), value :: Time, FinishTime
      integer ( c_int ), value :: iCycle, nCyclesMax
      real ( c_double ), intent ( out ) :: TimeOut, DeviceMilliseconds
      integer ( c_int ), intent ( out ) :: iCycleOut
    end function gfx_fluid_evolve_timed

    integer ( c_int ) function gfx_fluid_step_timed &
      ( Handle, Conserved_dev, TimeStep, Fluence_dev, Milliseconds, Stream ) &
      bind ( c, name = 'gfx_fluid_step_timed' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Fluence_dev, Stream
      real ( c_double ), value :: TimeStep
      real ( c_double ), intent ( out ) :: Milliseconds ( 4 )
    end function gfx_fluid_step_timed

    integer ( c_int ) function gfx_fluid_kernel_launches ( Handle, Count ) &
      bind ( c, name = 'gfx_fluid_kernel_launches' )
      import
      type ( c_ptr ), value :: Handle
      integer ( c_long_long ), intent ( out ) :: Count
    end function gfx_fluid_kernel_launches

    integer ( c_int ) function gfx_fluid_step_adjoint &
      ( Handle, Conserved_dev, TimeStep, Adjoint_New_dev, Adjoint_Old_dev, &
        Conserved_New_dev, DetectFeatures, Stream ) &
      bind ( c, name = 'gfx_fluid_step_adjoint' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Adjoint_New_dev, Adjoint_Old_dev, &
                               Conserved_New_dev, Stream
      real ( c_double ), value :: TimeStep
      integer ( c_int ), value :: DetectFeatures
    end function gfx_fluid_step_adjoint

    integer ( c_int ) function gfx_fluid_set_tuning &
      ( Handle, zChunk, AdjointSegment, TileRows ) &
      bind ( c, name = 'gfx_fluid_set_tuning' )
      import
      type ( c_ptr ), value :: Handle
      integer ( c_int ), value :: zChunk, AdjointSegment, TileRows
    end function gfx_fluid_set_tuning

    integer ( c_int ) function gfx_fluid_batch_create ( nBricks, Handles, Conserved_dev, Batch ) &
      bind ( c, name = 'gfx_fluid_batch_create' )
      import
      integer ( c_int ), value :: nBricks
      type ( c_ptr ), intent ( in ) :: Handles ( * ), Conserved_dev ( * )
      type ( c_ptr ), intent ( out ) :: Batch
    end function gfx_fluid_batch_create

    integer ( c_int ) function gfx_fluid_batch_destroy ( Batch ) &
      bind ( c, name = 'gfx_fluid_batch_destroy' )
      import
      type ( c_ptr ), value :: Batch
    end function gfx_fluid_batch_destroy

    integer ( c_int ) function gfx_fluid_batch_set_clocks ( Batch, Time, iCycle ) &
      bind ( c, name = 'gfx_fluid_batch_set_clocks' )
      import
      type ( c_ptr ), value :: Batch
      real ( c_double ), value :: Time
      integer ( c_int ), value :: iCycle
    end function gfx_fluid_batch_set_clocks

    integer ( c_int ) function gfx_fluid_batch_evolve ( Batch, FinishTime, nCycles, Stream ) &
      bind ( c, name = 'gfx_fluid_batch_evolve' )
      import
      type ( c_ptr ), value :: Batch, Stream
      real ( c_double ), value :: FinishTime
      integer ( c_int ), value :: nCycles
    end function gfx_fluid_batch_evolve

    integer ( c_int ) function gfx_fluid_batch_clocks ( Batch, Time_host, Cycle_host, Stream ) &
      bind ( c, name = 'gfx_fluid_batch_clocks' )
      import
      type ( c_ptr ), value :: Batch, Time_host, Cycle_host, Stream
    end function gfx_fluid_batch_clocks

    integer ( c_int ) function gfx_fluid_batch_kernel_launches ( Batch, Count ) &
      bind ( c, name = 'gfx_fluid_batch_kernel_launches' )
      import
      type ( c_ptr ), value :: Batch
      integer ( c_long_long ), intent ( out ) :: Count
    end function gfx_fluid_batch_kernel_launches

    integer ( c_int ) function gfx_fluid_step_branches &
      ( Handle, Conserved_dev, TimeStep, DetectFeatures, Signature, Stream ) &
      bind ( c, name = 'gfx_fluid_step_branches' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Stream
      real ( c_double ), value :: TimeStep
      integer ( c_int ), value :: DetectFeatures
      integer ( c_long_long ), intent ( out ) :: Signature ( 17 )
    end function gfx_fluid_step_branches

    !-- A chart of several bricks on one device (Chart_SLD's bricks)

    integer ( c_int ) function gfx_fluid_chart_create ( Config, nBricks, Chart ) &
      bind ( c, name = 'gfx_fluid_chart_create' )
      import
      type ( GFX_FluidConfig ), intent ( in ) :: Config
      integer ( c_int ), intent ( in ) :: nBricks ( 3 )
      type ( c_ptr ), intent ( out ) :: Chart
    end function gfx_fluid_chart_create

    integer ( c_int ) function gfx_fluid_chart_destroy ( Chart ) &
      bind ( c, name = 'gfx_fluid_chart_destroy' )
      import
      type ( c_ptr ), value :: Chart
    end function gfx_fluid_chart_destroy

    integer ( c_int ) function gfx_fluid_chart_n_bricks ( Chart, nBricks ) &
      bind ( c, name = 'gfx_fluid_chart_n_bricks' )
      import
      type ( c_ptr ), value :: Chart
      integer ( c_int ), intent ( out ) :: nBricks
    end function gfx_fluid_chart_n_bricks

    integer ( c_int ) function gfx_fluid_chart_brick ( Chart, iBrick, Handle, iaBrick ) &
      bind ( c, name = 'gfx_fluid_chart_brick' )
      import
      type ( c_ptr ), value :: Chart
      integer ( c_int ), value :: iBrick
      type ( c_ptr ), intent ( out ) :: Handle
      integer ( c_int ), intent ( out ) :: iaBrick ( 3 )
    end function gfx_fluid_chart_brick

    integer ( c_int ) function gfx_fluid_chart_bind ( Chart, Conserved_dev ) &
      bind ( c, name = 'gfx_fluid_chart_bind' )
      import
      type ( c_ptr ), value :: Chart
      type ( c_ptr ), intent ( in ) :: Conserved_dev ( * )
    end function gfx_fluid_chart_bind

    integer ( c_int ) function gfx_fluid_chart_from_primitive ( Chart, Primitive_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_chart_from_primitive' )
      import
      type ( c_ptr ), value :: Chart, Stream
      type ( c_ptr ), intent ( in ) :: Primitive_dev ( * )
    end function gfx_fluid_chart_from_primitive

    integer ( c_int ) function gfx_fluid_chart_set_conserved ( Chart, Stream ) &
      bind ( c, name = 'gfx_fluid_chart_set_conserved' )
      import
      type ( c_ptr ), value :: Chart, Stream
    end function gfx_fluid_chart_set_conserved

    integer ( c_int ) function gfx_fluid_chart_timestep ( Chart, iCycle, TimeStep, Stream ) &
      bind ( c, name = 'gfx_fluid_chart_timestep' )
      import
      type ( c_ptr ), value :: Chart, Stream
      integer ( c_int ), value :: iCycle
      real ( c_double ), intent ( out ) :: TimeStep
    end function gfx_fluid_chart_timestep

    integer ( c_int ) function gfx_fluid_chart_step ( Chart, TimeStep, Fluence_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_chart_step' )
      import
      type ( c_ptr ), value :: Chart, Stream
      real ( c_double ), value :: TimeStep
      type ( c_ptr ), intent ( in ) :: Fluence_dev ( * )
    end function gfx_fluid_chart_step

    integer ( c_int ) function gfx_fluid_chart_evolve &
      ( Chart, Time, iCycle, FinishTime, nCyclesMax, Time_out, iCycle_out, Stream ) &
      bind ( c, name = 'gfx_fluid_chart_evolve' )
      import
      type ( c_ptr ), value :: Chart, Stream
      real ( c_double ), value :: Time, FinishTime
      integer ( c_int ), value :: iCycle, nCyclesMax
      real ( c_double ), intent ( out ) :: Time_out
      integer ( c_int ), intent ( out ) :: iCycle_out
    end function gfx_fluid_chart_evolve

    integer ( c_int ) function gfx_fluid_chart_kernel_launches ( Chart, Count ) &
      bind ( c, name = 'gfx_fluid_chart_kernel_launches' )
      import
      type ( c_ptr ), value :: Chart
      integer ( c_long_long ), intent ( out ) :: Count
    end function gfx_fluid_chart_kernel_launches

    integer ( c_int ) function gfx_fluid_step_noalloc &
      ( Config, Conserved_dev, TimeStep, DetectFeatures, Fluence_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_step_noalloc' )
      import
      type ( GFX_FluidConfig ), intent ( in ) :: Config
      type ( c_ptr ), value :: Conserved_dev, Fluence_dev, Stream
      real ( c_double ), value :: TimeStep
      integer ( c_int ), value :: DetectFeatures
    end function gfx_fluid_step_noalloc

    integer ( c_int ) function gfx_fluid_check_state ( Handle, Conserved_dev, Stream ) &
      bind ( c, name = 'gfx_fluid_check_state' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Stream
    end function gfx_fluid_check_state

    integer ( c_int ) function gfx_fluid_totals ( Handle, Conserved_dev, Totals, Stream ) &
      bind ( c, name = 'gfx_fluid_totals' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev, Stream
      real ( c_double ), intent ( out ) :: Totals ( 6 )
    end function gfx_fluid_totals

    integer ( c_int ) function gfx_fluid_resume ( Handle, Conserved_dev ) &
      bind ( c, name = 'gfx_fluid_resume' )
      import
      type ( c_ptr ), value :: Handle, Conserved_dev
    end function gfx_fluid_resume

    integer ( c_int ) function gfx_fluid_last_error ( Buffer, Length ) &
      bind ( c, name = 'gfx_fluid_last_error' )
      import
      character ( kind = c_char ), intent ( out ) :: Buffer ( * )
      integer ( c_size_t ), value :: Length
    end function gfx_fluid_last_error

    integer ( c_int ) function gfx_fluid_debug_fail_allocation ( nth ) &
      bind ( c, name = 'gfx_fluid_debug_fail_allocation' )
      import
      integer ( c_int ), value :: nth
    end function gfx_fluid_debug_fail_allocation

  end interface

end module GFX_Fluid_C
