!-----------------------------------------------------------------------------
! Device-backed extensions of LFRic's solver API types, calling liblfx
! (include/lfx.h) through ISO_C_BINDING. Each type-bound procedure is one C
! call; a non-zero status becomes log_event(..., LOG_LEVEL_ERROR), keeping the
! reference's abort-on-error behaviour.
!
! Extends:
!   abstract_vector_type          infrastructure/source/field/vector_mod.F90
!   abstract_linear_operator_type components/science/source/solver/sci_linear_operator_mod.f90
!   abstract_preconditioner_type  components/science/source/solver/sci_preconditioner_mod.f90
!   abstract_iterative_solver_type components/science/source/solver/sci_iterative_solver_mod.f90
!
! Source only in this repository (no Fortran compiler in the build image).
!-----------------------------------------------------------------------------
module lfx_device_mod

  use, intrinsic :: iso_c_binding
  use constants_mod,           only : r_def, i_def, l_def
  use vector_mod,              only : abstract_vector_type
  use sci_linear_operator_mod, only : abstract_linear_operator_type
  use sci_preconditioner_mod,  only : abstract_preconditioner_type
  use log_mod,                 only : log_event, LOG_LEVEL_ERROR

  implicit none
  private

  integer(c_int32_t), parameter, public :: LFX_R64 = 64, LFX_R32 = 32

  ! ------------------------------------------------------------------ C ABI
  interface
    integer(c_int) function lfx_ctx_create(device, ctx) bind(C, name="lfx_ctx_create")
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr)           :: ctx
    end function
    type(c_ptr) function lfx_last_error(ctx) bind(C, name="lfx_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function lfx_vec_create(ctx, nfields, undf, precision, v) &
        bind(C, name="lfx_vec_create")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value        :: ctx
      integer(c_int32_t), value :: nfields, precision
      integer(c_int64_t)        :: undf(*)
      type(c_ptr)               :: v
    end function
    integer(c_int) function lfx_vec_duplicate(src, v) bind(C, name="lfx_vec_duplicate")
      import :: c_int, c_ptr
      type(c_ptr), value :: src
      type(c_ptr)        :: v
    end function
    integer(c_int) function lfx_vec_destroy(v) bind(C, name="lfx_vec_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: v
    end function
    integer(c_int) function lfx_vec_set_scalar(v, s) bind(C, name="lfx_vec_set_scalar")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: v
      real(c_double), value :: s
    end function
    integer(c_int) function lfx_vec_axpy(y, a, x) bind(C, name="lfx_vec_axpy")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: y, x
      real(c_double), value :: a
    end function
    integer(c_int) function lfx_vec_aypx(y, a, x) bind(C, name="lfx_vec_aypx")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: y, x
      real(c_double), value :: a
    end function
    integer(c_int) function lfx_vec_axpby(z, a, x, b, y) bind(C, name="lfx_vec_axpby")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: z, x, y
      real(c_double), value :: a, b
    end function
    integer(c_int) function lfx_vec_norm(v, out) bind(C, name="lfx_vec_norm")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: v
      real(c_double)     :: out
    end function
    integer(c_int) function lfx_vec_field_norm(v, n, out) bind(C, name="lfx_vec_field_norm")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value        :: v
      integer(c_int32_t), value :: n
      real(c_double)            :: out
    end function
    integer(c_int) function lfx_vec_dot(v, x, out) bind(C, name="lfx_vec_dot")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: v, x
      real(c_double)     :: out
    end function
    integer(c_int) function lfx_vec_scale(v, s) bind(C, name="lfx_vec_scale")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: v
      real(c_double), value :: s
    end function
    integer(c_int) function lfx_vec_copy(dst, src) bind(C, name="lfx_vec_copy")
      import :: c_int, c_ptr
      type(c_ptr), value :: dst, src
    end function
    integer(c_int) function lfx_vec_size(v, n) bind(C, name="lfx_vec_size")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: v
      integer(c_int32_t) :: n
    end function
    integer(c_int) function lfx_vec_import_field(v, pos, host, n) &
        bind(C, name="lfx_vec_import_field")
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value        :: v
      integer(c_int32_t), value :: pos
      real(c_double)            :: host(*)
      integer(c_int64_t), value :: n
    end function
    integer(c_int) function lfx_vec_export_field(v, pos, host, n) &
        bind(C, name="lfx_vec_export_field")
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value        :: v
      integer(c_int32_t), value :: pos
      real(c_double)            :: host(*)
      integer(c_int64_t), value :: n
    end function
    integer(c_int) function lfx_lma_create(ctx, ncell_2d, nlayers, ndf_to, ndf_from, map_to, &
        map_from, undf_to, undf_from, local_stencil, ncolours, ncells_per_colour,            &
        cells_in_colour, max_cells, precision, op) bind(C, name="lfx_lma_create")
      import :: c_int, c_int32_t, c_int64_t, c_ptr, c_double
      type(c_ptr), value        :: ctx
      integer(c_int32_t), value :: ncell_2d, nlayers, ndf_to, ndf_from, ncolours, max_cells, &
                                   precision
      integer(c_int32_t)        :: map_to(*), map_from(*), ncells_per_colour(*), cells_in_colour(*)
      integer(c_int64_t), value :: undf_to, undf_from
      real(c_double)            :: local_stencil(*)
      type(c_ptr)               :: op
    end function
    integer(c_int) function lfx_op_apply(op, x, y) bind(C, name="lfx_op_apply")
      import :: c_int, c_ptr
      type(c_ptr), value :: op, x, y
    end function
    integer(c_int) function lfx_prec_apply(p, x, y) bind(C, name="lfx_prec_apply")
      import :: c_int, c_ptr
      type(c_ptr), value :: p, x, y
    end function
  end interface

  ! ------------------------------------------------------------------ types
  type, public, extends(abstract_vector_type) :: device_vector_type
    type(c_ptr) :: h = c_null_ptr
  contains
    procedure, public :: set_scalar => dv_set_scalar
    procedure, public :: axpy       => dv_axpy
    procedure, public :: aypx       => dv_aypx
    procedure, public :: axpby      => dv_axpby
    procedure, public :: norm       => dv_norm
    procedure, public :: field_norm => dv_field_norm
    procedure, public :: dot        => dv_dot
    procedure, public :: scale      => dv_scale
    procedure, public :: duplicate  => dv_duplicate
    procedure, public :: copy       => dv_copy
    procedure, public :: vector_size => dv_size
    final :: dv_destroy
  end type device_vector_type

  type, public, extends(abstract_linear_operator_type) :: device_lma_operator_type
    type(c_ptr) :: h = c_null_ptr
  contains
    procedure, public :: apply => dop_apply
  end type device_lma_operator_type

  type, public, extends(abstract_preconditioner_type) :: device_preconditioner_type
    type(c_ptr) :: h = c_null_ptr
  contains
    procedure, public :: apply => dprec_apply
  end type device_preconditioner_type

  public :: lfx_check

contains

  subroutine lfx_check(rc, what)
    integer(c_int),   intent(in) :: rc
    character(len=*), intent(in) :: what
    if (rc /= 0) call log_event("lfx: "//what//" failed", LOG_LEVEL_ERROR)
  end subroutine lfx_check

  subroutine dv_set_scalar(self, scalar)
    class(device_vector_type), intent(inout) :: self
    real(kind=r_def),          intent(in)    :: scalar
    call lfx_check(lfx_vec_set_scalar(self%h, real(scalar, c_double)), "set_scalar")
  end subroutine

  subroutine dv_axpy(self, alpha, x)
    class(device_vector_type),   intent(inout) :: self
    real(kind=r_def),            intent(in)    :: alpha
    class(abstract_vector_type), intent(inout) :: x
    select type (x)
    type is (device_vector_type)
      call lfx_check(lfx_vec_axpy(self%h, real(alpha, c_double), x%h), "axpy")
    class default
      call log_event("lfx: axpy: x is not a device_vector_type", LOG_LEVEL_ERROR)
    end select
  end subroutine

  subroutine dv_aypx(self, alpha, x)
    class(device_vector_type),   intent(inout) :: self
    real(kind=r_def),            intent(in)    :: alpha
    class(abstract_vector_type), intent(inout) :: x
    select type (x)
    type is (device_vector_type)
      call lfx_check(lfx_vec_aypx(self%h, real(alpha, c_double), x%h), "aypx")
    class default
      call log_event("lfx: aypx: x is not a device_vector_type", LOG_LEVEL_ERROR)
    end select
  end subroutine

  subroutine dv_axpby(self, a, x, b, y)
    class(device_vector_type),   intent(inout) :: self
    real(kind=r_def),            intent(in)    :: a, b
    class(abstract_vector_type), intent(in)    :: x, y
    select type (x)
    type is (device_vector_type)
      select type (y)
      type is (device_vector_type)
        call lfx_check(lfx_vec_axpby(self%h, real(a, c_double), x%h, real(b, c_double), y%h), &
                       "axpby")
      class default
        call log_event("lfx: axpby: y is not a device_vector_type", LOG_LEVEL_ERROR)
      end select
    class default
      call log_event("lfx: axpby: x is not a device_vector_type", LOG_LEVEL_ERROR)
    end select
  end subroutine

  function dv_norm(self) result(normal)
    class(device_vector_type), intent(in) :: self
    real(kind=r_def) :: normal
    real(c_double) :: v
    call lfx_check(lfx_vec_norm(self%h, v), "norm")
    normal = real(v, r_def)
  end function

  function dv_field_norm(self, n) result(normal)
    class(device_vector_type), intent(in) :: self
    integer(kind=i_def),       intent(in) :: n
    real(kind=r_def) :: normal
    real(c_double) :: v
    call lfx_check(lfx_vec_field_norm(self%h, int(n, c_int32_t), v), "field_norm")
    normal = real(v, r_def)
  end function

  function dv_dot(self, x) result(dot_prod)
    class(device_vector_type),   intent(in) :: self
    class(abstract_vector_type), intent(in) :: x
    real(kind=r_def) :: dot_prod
    real(c_double) :: v
    select type (x)
    type is (device_vector_type)
      call lfx_check(lfx_vec_dot(self%h, x%h, v), "dot")
      dot_prod = real(v, r_def)
    class default
      call log_event("lfx: dot: x is not a device_vector_type", LOG_LEVEL_ERROR)
    end select
  end function

  subroutine dv_scale(self, scalar)
    class(device_vector_type), intent(inout) :: self
    real(kind=r_def),          intent(in)    :: scalar
    call lfx_check(lfx_vec_scale(self%h, real(scalar, c_double)), "scale")
  end subroutine

  subroutine dv_duplicate(self, vec)
    class(device_vector_type),                intent(in)    :: self
    class(abstract_vector_type), allocatable, intent(inout) :: vec
    allocate(device_vector_type :: vec)
    select type (vec)
    type is (device_vector_type)
      call lfx_check(lfx_vec_duplicate(self%h, vec%h), "duplicate")
    end select
  end subroutine

  subroutine dv_copy(self, source)
    class(device_vector_type),   intent(out) :: self
    class(abstract_vector_type), intent(in)  :: source
    select type (source)
    type is (device_vector_type)
      if (.not. c_associated(self%h)) call lfx_check(lfx_vec_duplicate(source%h, self%h), "copy")
      call lfx_check(lfx_vec_copy(self%h, source%h), "copy")
    class default
      call log_event("lfx: copy: type mismatch", LOG_LEVEL_ERROR)
    end select
  end subroutine

  function dv_size(self) result(n_fields)
    class(device_vector_type), intent(in) :: self
    integer(kind=i_def) :: n_fields
    integer(c_int32_t) :: n
    call lfx_check(lfx_vec_size(self%h, n), "vector_size")
    n_fields = int(n, i_def)
  end function

  subroutine dv_destroy(self)
    type(device_vector_type), intent(inout) :: self
    integer(c_int) :: rc
    if (c_associated(self%h)) rc = lfx_vec_destroy(self%h)
    self%h = c_null_ptr
  end subroutine

  subroutine dop_apply(self, x, y)
    class(device_lma_operator_type), intent(inout) :: self
    class(abstract_vector_type),     intent(in)    :: x
    class(abstract_vector_type),     intent(inout) :: y
    select type (x)
    type is (device_vector_type)
      select type (y)
      type is (device_vector_type)
        call lfx_check(lfx_op_apply(self%h, x%h, y%h), "operator apply")
      end select
    class default
      call log_event("lfx: operator apply: incorrect vector_type argument", LOG_LEVEL_ERROR)
    end select
  end subroutine

  subroutine dprec_apply(self, x, y)
    class(device_preconditioner_type), intent(inout) :: self
    class(abstract_vector_type),       intent(in)    :: x
    class(abstract_vector_type),       intent(inout) :: y
    select type (x)
    type is (device_vector_type)
      select type (y)
      type is (device_vector_type)
        call lfx_check(lfx_prec_apply(self%h, x%h, y%h), "preconditioner apply")
      end select
    class default
      call log_event("lfx: preconditioner apply: incorrect vector_type argument", LOG_LEVEL_ERROR)
    end select
  end subroutine

end module lfx_device_mod
