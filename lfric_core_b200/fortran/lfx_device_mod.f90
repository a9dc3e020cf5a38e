!-----------------------------------------------------------------------------
! Device-backed extensions of LFRic's solver API types, calling liblfx
! (include/lfx.h) through ISO_C_BINDING. Each type-bound procedure is one C
! call; a non-zero status becomes log_event(..., LOG_LEVEL_ERROR), keeping the
! reference's abort-on-error behaviour (log_mod.F90:423-471), and a vector of
! the wrong dynamic type aborts as the reference's field_vector_type does
! (sci_field_vector_mod.x90:168-181).
!
! Extends:
!   abstract_vector_type           infrastructure/source/field/vector_mod.F90:17-189
!   abstract_linear_operator_type  components/science/source/solver/sci_linear_operator_mod.f90:18-36
!   abstract_preconditioner_type   components/science/source/solver/sci_preconditioner_mod.f90:19-38
!   abstract_iterative_solver_type components/science/source/solver/sci_iterative_solver_mod.f90:38-57
!
! Objects are set up by *_init subroutines (not function results, so that no
! compiler-made temporary of a finalizable type ever destroys a device
! handle) on the module's device context (lfx_device_init). As in the
! reference, a solver keeps pointers to its operator and preconditioner: both
! must outlive it.
!
! Source only in this repository (no Fortran compiler in the build image).
!-----------------------------------------------------------------------------
module lfx_device_mod

  use, intrinsic :: iso_c_binding
  use constants_mod,            only : r_def, i_def, l_def
  use vector_mod,               only : abstract_vector_type
  use sci_linear_operator_mod,  only : abstract_linear_operator_type
  use sci_preconditioner_mod,   only : abstract_preconditioner_type
  use sci_iterative_solver_mod, only : abstract_iterative_solver_type
  use log_mod,                  only : log_event, LOG_LEVEL_ERROR

  implicit none
  private

  integer(c_int32_t), parameter, public :: LFX_R64 = 64, LFX_R32 = 32
  integer(c_int32_t), parameter, public :: LFX_SOLVER_CG = 1, LFX_SOLVER_BICGSTAB = 2, &
                                           LFX_SOLVER_GMRES = 3, LFX_SOLVER_FGMRES = 4, &
                                           LFX_SOLVER_GCR = 5

  ! lfx_solver_cfg and lfx_solve_info of include/lfx.h
  type, bind(C), public :: lfx_solver_cfg
    real(c_double)     :: r_tol
    real(c_double)     :: a_tol
    integer(c_int32_t) :: max_iter
    integer(c_int32_t) :: gcrk
    integer(c_int32_t) :: monitor_convergence
    integer(c_int32_t) :: fail_on_non_converged
  end type lfx_solver_cfg

  type, bind(C), public :: lfx_solve_info
    integer(c_int32_t) :: iterations
    integer(c_int32_t) :: converged
    real(c_double)     :: initial_norm
    real(c_double)     :: final_norm
    real(c_double)     :: final_rel
    integer(c_int32_t) :: applies
    integer(c_int32_t) :: status
    integer(c_int32_t) :: outer_iterations
    integer(c_int32_t) :: inner_iterations
  end type lfx_solve_info

  ! the device context every object of this module is made on
  type(c_ptr), save :: lfx_context = c_null_ptr

  ! ------------------------------------------------------------------ C ABI
  interface
    integer(c_int) function lfx_ctx_create(device, ctx) bind(C, name="lfx_ctx_create")
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr)           :: ctx
    end function
    integer(c_int) function lfx_ctx_destroy(ctx) bind(C, name="lfx_ctx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    type(c_ptr) function lfx_last_error(ctx) bind(C, name="lfx_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    ! ---- vectors
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
    ! ---- operators
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
    integer(c_int) function lfx_lma_create_like(src, local_stencil, precision, op) &
        bind(C, name="lfx_lma_create_like")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value        :: src
      real(c_double)            :: local_stencil(*)
      integer(c_int32_t), value :: precision
      type(c_ptr)               :: op
    end function
    integer(c_int) function lfx_lma_sum(x, a, y, op) bind(C, name="lfx_lma_sum")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value    :: x, y
      real(c_double), value :: a
      type(c_ptr)           :: op
    end function
    integer(c_int) function lfx_lma_diagonal(op, diag) bind(C, name="lfx_lma_diagonal")
      import :: c_int, c_ptr
      type(c_ptr), value :: op, diag
    end function
    integer(c_int) function lfx_op_apply(op, x, y) bind(C, name="lfx_op_apply")
      import :: c_int, c_ptr
      type(c_ptr), value :: op, x, y
    end function
    integer(c_int) function lfx_op_destroy(op) bind(C, name="lfx_op_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: op
    end function
    ! ---- column (CMA) operators
    integer(c_int) function lfx_cma_create(ctx, ncell_2d, nrow, ncol, bandwidth, alpha, beta, &
        gamma_m, gamma_p, first_dof, indirection, columnwise_matrix, cma)                     &
        bind(C, name="lfx_cma_create")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value        :: ctx
      integer(c_int32_t), value :: ncell_2d, nrow, ncol, bandwidth, alpha, beta, gamma_m, gamma_p
      integer(c_int32_t)        :: first_dof(*), indirection(*)
      real(c_double)            :: columnwise_matrix(*)
      type(c_ptr)               :: cma
    end function
    integer(c_int) function lfx_cma_assemble_from_lma(lma, nsub, dfs, column_banded_dofmap,   &
        alpha, beta, gamma_m, gamma_p, bandwidth, nrow, first_dof, indirection, cma)           &
        bind(C, name="lfx_cma_assemble_from_lma")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value        :: lma
      integer(c_int32_t), value :: nsub, alpha, beta, gamma_m, gamma_p, bandwidth, nrow
      integer(c_int32_t)        :: dfs(*), column_banded_dofmap(*), first_dof(*), indirection(*)
      type(c_ptr)               :: cma
    end function
    integer(c_int) function lfx_cma_destroy(cma) bind(C, name="lfx_cma_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: cma
    end function
    ! ---- preconditioners
    integer(c_int) function lfx_null_prec_create(ctx, p) bind(C, name="lfx_null_prec_create")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr)        :: p
    end function
    integer(c_int) function lfx_diag_prec_create(ctx, diag, p) bind(C, name="lfx_diag_prec_create")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx, diag
      type(c_ptr)        :: p
    end function
    integer(c_int) function lfx_cma_prec_create(ctx, cma, diag, precision, p) &
        bind(C, name="lfx_cma_prec_create")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value        :: ctx, cma, diag
      integer(c_int32_t), value :: precision
      type(c_ptr)               :: p
    end function
    integer(c_int) function lfx_prec_apply(p, x, y) bind(C, name="lfx_prec_apply")
      import :: c_int, c_ptr
      type(c_ptr), value :: p, x, y
    end function
    integer(c_int) function lfx_prec_destroy(p) bind(C, name="lfx_prec_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: p
    end function
    ! ---- whole solves
    integer(c_int) function lfx_solver_create(ctx, kind, op, prec, cfg, s) &
        bind(C, name="lfx_solver_create")
      import :: c_int, c_int32_t, c_ptr, lfx_solver_cfg
      type(c_ptr), value        :: ctx, op, prec
      integer(c_int32_t), value :: kind
      type(lfx_solver_cfg)      :: cfg
      type(c_ptr)               :: s
    end function
    integer(c_int) function lfx_refined_solver_create(ctx, op64, inner, inner_rtol, cfg, s) &
        bind(C, name="lfx_refined_solver_create")
      import :: c_int, c_ptr, c_double, lfx_solver_cfg
      type(c_ptr), value    :: ctx, op64, inner
      real(c_double), value :: inner_rtol
      type(lfx_solver_cfg)  :: cfg
      type(c_ptr)           :: s
    end function
    integer(c_int) function lfx_solver_apply(s, x, b, info) bind(C, name="lfx_solver_apply")
      import :: c_int, c_ptr, lfx_solve_info
      type(c_ptr), value   :: s, x, b
      type(lfx_solve_info) :: info
    end function
    integer(c_int) function lfx_solver_destroy(s) bind(C, name="lfx_solver_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: s
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
    procedure, public :: import_field => dv_import_field
    procedure, public :: export_field => dv_export_field
    final :: dv_destroy
  end type device_vector_type

  type, public, extends(abstract_linear_operator_type) :: device_lma_operator_type
    type(c_ptr) :: h = c_null_ptr
  contains
    procedure, public :: apply => dop_apply
    final :: dop_destroy
  end type device_lma_operator_type

  type, public, extends(abstract_preconditioner_type) :: device_preconditioner_type
    type(c_ptr) :: h = c_null_ptr
  contains
    procedure, public :: apply => dprec_apply
    final :: dprec_destroy
  end type device_preconditioner_type

  ! a column (CMA) operator, the input of the column preconditioner
  type, public :: device_cma_type
    type(c_ptr) :: h = c_null_ptr
  contains
    final :: dcma_destroy
  end type device_cma_type

  ! the whole solve on the device (CG, BiCGStab, GMRES, FGMRES, GCR, or FP64
  ! iterative refinement around one of them); apply(x, b) as the reference's
  ! solvers: x the initial guess in and the solution out, b unchanged
  type, public, extends(abstract_iterative_solver_type) :: device_krylov_solver_type
    type(c_ptr) :: h = c_null_ptr
    type(lfx_solve_info) :: info
  contains
    procedure, public :: apply => dsolver_apply
    final :: dsolver_destroy
  end type device_krylov_solver_type

  public :: lfx_check, lfx_device_init, lfx_device_finalise
  public :: device_vector_init, device_lma_operator_init, device_lma_operator_like, &
            device_lma_operator_sum, device_lma_diagonal, device_null_preconditioner_init, &
            device_diagonal_preconditioner_init, device_cma_init, device_cma_from_lma, &
            device_cma_preconditioner_init, device_krylov_solver_init, &
            device_refined_solver_init

contains

  subroutine lfx_check(rc, what)
    integer(c_int),   intent(in) :: rc
    character(len=*), intent(in) :: what
    if (rc /= 0) call log_event("lfx: "//what//" failed", LOG_LEVEL_ERROR)
  end subroutine lfx_check

  !> Creates the device context (one per process, on GPU `device`).
  subroutine lfx_device_init(device)
    integer(kind=i_def), intent(in) :: device
    if (c_associated(lfx_context)) return
    call lfx_check(lfx_ctx_create(int(device, c_int), lfx_context), "context creation")
  end subroutine lfx_device_init

  subroutine lfx_device_finalise()
    integer(c_int) :: rc
    if (c_associated(lfx_context)) rc = lfx_ctx_destroy(lfx_context)
    lfx_context = c_null_ptr
  end subroutine lfx_device_finalise

  ! ------------------------------------------------------------------ vectors
  !> nfields fields of undf(i) values, FP64 (LFX_R64) or FP32 (LFX_R32)
  subroutine device_vector_init(self, undf, precision)
    type(device_vector_type), intent(inout) :: self
    integer(kind=i_def),      intent(in)    :: undf(:)
    integer(c_int32_t),       intent(in)    :: precision
    integer(c_int64_t) :: n(size(undf))
    n = int(undf, c_int64_t)
    call lfx_check(lfx_vec_create(lfx_context, int(size(undf), c_int32_t), n, precision, self%h), &
                   "vector creation")
  end subroutine device_vector_init

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
    dot_prod = 0.0_r_def
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

  !> field_vector_type%import_field (sci_field_vector_mod.x90:294-312): the
  !> host data of field `position` (1-based)
  subroutine dv_import_field(self, data, position)
    class(device_vector_type), intent(inout) :: self
    real(kind=r_def),          intent(in)    :: data(:)
    integer(kind=i_def),       intent(in)    :: position
    real(c_double) :: tmp(size(data))
    tmp = real(data, c_double)
    call lfx_check(lfx_vec_import_field(self%h, int(position, c_int32_t), tmp, &
                                        int(size(data), c_int64_t)), "import_field")
  end subroutine

  !> field_vector_type%export_field (sci_field_vector_mod.x90:315-334)
  subroutine dv_export_field(self, data, position)
    class(device_vector_type), intent(in)    :: self
    real(kind=r_def),          intent(inout) :: data(:)
    integer(kind=i_def),       intent(in)    :: position
    real(c_double) :: tmp(size(data))
    call lfx_check(lfx_vec_export_field(self%h, int(position, c_int32_t), tmp, &
                                        int(size(data), c_int64_t)), "export_field")
    data = real(tmp, r_def)
  end subroutine

  subroutine dv_destroy(self)
    type(device_vector_type), intent(inout) :: self
    integer(c_int) :: rc
    if (c_associated(self%h)) rc = lfx_vec_destroy(self%h)
    self%h = c_null_ptr
  end subroutine

  ! ------------------------------------------------------------------ operators
  !> The LMA operator (operator_type, operator_mod.t90:31-122) as the
  !> reference stores it: local_stencil(ncell_2d*nlayers, ndf_to, ndf_from),
  !> dofmaps (ndf, ncell_2d) and the colouring of the cells
  !> (mesh_colouring_mod.F90:151-328); the device keeps its own copy.
  subroutine device_lma_operator_init(self, ncell_2d, nlayers, ndf_to, ndf_from, map_to, &
                                      map_from, undf_to, undf_from, local_stencil,       &
                                      ncells_per_colour, cells_in_colour, precision)
    type(device_lma_operator_type), intent(inout) :: self
    integer(kind=i_def), intent(in) :: ncell_2d, nlayers, ndf_to, ndf_from, undf_to, undf_from
    integer(kind=i_def), intent(in) :: map_to(:,:), map_from(:,:)
    real(kind=r_def),    intent(in) :: local_stencil(:,:,:)
    integer(kind=i_def), intent(in) :: ncells_per_colour(:), cells_in_colour(:,:)
    integer(c_int32_t),  intent(in) :: precision
    integer(c_int32_t) :: mt(size(map_to)), mf(size(map_from)), npc(size(ncells_per_colour)), &
                          cic(size(cells_in_colour))
    real(c_double) :: st(size(local_stencil))
    mt = int(reshape(map_to, [size(map_to)]), c_int32_t)
    mf = int(reshape(map_from, [size(map_from)]), c_int32_t)
    npc = int(ncells_per_colour, c_int32_t)
    cic = int(reshape(cells_in_colour, [size(cells_in_colour)]), c_int32_t)
    st = real(reshape(local_stencil, [size(local_stencil)]), c_double)
    call lfx_check(lfx_lma_create(lfx_context, int(ncell_2d, c_int32_t), int(nlayers, c_int32_t), &
                                  int(ndf_to, c_int32_t), int(ndf_from, c_int32_t), mt, mf,       &
                                  int(undf_to, c_int64_t), int(undf_from, c_int64_t), st,         &
                                  int(size(ncells_per_colour), c_int32_t), npc, cic,              &
                                  int(size(cells_in_colour, 2), c_int32_t), precision, self%h),   &
                   "operator creation")
  end subroutine device_lma_operator_init

  !> a second operator on the dofmaps and colouring of `src` with its own
  !> local matrices (e.g. the FP32 copy of an FP64 operator)
  subroutine device_lma_operator_like(self, src, local_stencil, precision)
    type(device_lma_operator_type), intent(inout) :: self
    type(device_lma_operator_type), intent(in)    :: src
    real(kind=r_def),               intent(in)    :: local_stencil(:,:,:)
    integer(c_int32_t),             intent(in)    :: precision
    real(c_double) :: st(size(local_stencil))
    st = real(reshape(local_stencil, [size(local_stencil)]), c_double)
    call lfx_check(lfx_lma_create_like(src%h, st, precision, self%h), "operator creation")
  end subroutine device_lma_operator_like

  !> self = x + a y (operator_x_plus_ay, sci_operator_algebra_kernel_mod.F90:92-119)
  !> for two operators on one layout, e.g. M2 + tau D^T D
  subroutine device_lma_operator_sum(self, x, a, y)
    type(device_lma_operator_type), intent(inout) :: self
    type(device_lma_operator_type), intent(in)    :: x, y
    real(kind=r_def),               intent(in)    :: a
    call lfx_check(lfx_lma_sum(x%h, real(a, c_double), y%h, self%h), "operator sum")
  end subroutine device_lma_operator_sum

  !> diag(A) (mm_diagonal_kernel_code, sci_mm_diagonal_kernel_mod.F90:99-125)
  subroutine device_lma_diagonal(op, diag)
    type(device_lma_operator_type), intent(in)    :: op
    type(device_vector_type),       intent(inout) :: diag
    call lfx_check(lfx_lma_diagonal(op%h, diag%h), "operator diagonal")
  end subroutine device_lma_diagonal

  subroutine dop_apply(self, x, y)
    class(device_lma_operator_type), intent(inout) :: self
    class(abstract_vector_type),     intent(in)    :: x
    class(abstract_vector_type),     intent(inout) :: y
    select type (x)
    type is (device_vector_type)
      select type (y)
      type is (device_vector_type)
        call lfx_check(lfx_op_apply(self%h, x%h, y%h), "operator apply")
      class default
        call log_event("lfx: operator apply: y is not a device_vector_type", LOG_LEVEL_ERROR)
      end select
    class default
      call log_event("lfx: operator apply: x is not a device_vector_type", LOG_LEVEL_ERROR)
    end select
  end subroutine

  subroutine dop_destroy(self)
    type(device_lma_operator_type), intent(inout) :: self
    integer(c_int) :: rc
    if (c_associated(self%h)) rc = lfx_op_destroy(self%h)
    self%h = c_null_ptr
  end subroutine

  ! ------------------------------------------------------------------ column operators
  !> columnwise_operator_type from its band columnwise_matrix(bandwidth, nrow,
  !> ncell_2d) (columnwise_operator_mod.f90:42-114)
  subroutine device_cma_init(self, ncell_2d, nrow, ncol, bandwidth, alpha, beta, gamma_m, &
                             gamma_p, first_dof, indirection, columnwise_matrix)
    type(device_cma_type), intent(inout) :: self
    integer(kind=i_def),   intent(in)    :: ncell_2d, nrow, ncol, bandwidth, alpha, beta, &
                                            gamma_m, gamma_p
    integer(kind=i_def),   intent(in)    :: first_dof(:), indirection(:)
    real(kind=r_def),      intent(in)    :: columnwise_matrix(:,:,:)
    integer(c_int32_t) :: f(size(first_dof)), ind(size(indirection))
    real(c_double) :: band(size(columnwise_matrix))
    f = int(first_dof, c_int32_t)
    ind = int(indirection, c_int32_t)
    band = real(reshape(columnwise_matrix, [size(columnwise_matrix)]), c_double)
    call lfx_check(lfx_cma_create(lfx_context, int(ncell_2d, c_int32_t), int(nrow, c_int32_t),   &
                                  int(ncol, c_int32_t), int(bandwidth, c_int32_t),              &
                                  int(alpha, c_int32_t), int(beta, c_int32_t),                  &
                                  int(gamma_m, c_int32_t), int(gamma_p, c_int32_t), f, ind, band, &
                                  self%h), "column operator creation")
  end subroutine device_cma_init

  !> columnwise_op_asm (sci_columnwise_op_asm_kernel_mod.F90:72-128) on the
  !> device from the sub-block `dfs` of an FP64 LMA operator
  subroutine device_cma_from_lma(self, lma, dfs, column_banded_dofmap, alpha, beta, gamma_m, &
                                 gamma_p, bandwidth, nrow, first_dof, indirection)
    type(device_cma_type),          intent(inout) :: self
    type(device_lma_operator_type), intent(in)    :: lma
    integer(kind=i_def), intent(in) :: dfs(:), column_banded_dofmap(:,:), first_dof(:), &
                                       indirection(:)
    integer(kind=i_def), intent(in) :: alpha, beta, gamma_m, gamma_p, bandwidth, nrow
    integer(c_int32_t) :: d(size(dfs)), cbd(size(column_banded_dofmap)), f(size(first_dof)), &
                          ind(size(indirection))
    d = int(dfs, c_int32_t)
    cbd = int(reshape(column_banded_dofmap, [size(column_banded_dofmap)]), c_int32_t)
    f = int(first_dof, c_int32_t)
    ind = int(indirection, c_int32_t)
    call lfx_check(lfx_cma_assemble_from_lma(lma%h, int(size(dfs), c_int32_t), d, cbd,          &
                                             int(alpha, c_int32_t), int(beta, c_int32_t),        &
                                             int(gamma_m, c_int32_t), int(gamma_p, c_int32_t),   &
                                             int(bandwidth, c_int32_t), int(nrow, c_int32_t),    &
                                             f, ind, self%h), "column operator assembly")
  end subroutine device_cma_from_lma

  subroutine dcma_destroy(self)
    type(device_cma_type), intent(inout) :: self
    integer(c_int) :: rc
    if (c_associated(self%h)) rc = lfx_cma_destroy(self%h)
    self%h = c_null_ptr
  end subroutine

  ! ------------------------------------------------------------------ preconditioners
  subroutine device_null_preconditioner_init(self)
    type(device_preconditioner_type), intent(inout) :: self
    call lfx_check(lfx_null_prec_create(lfx_context, self%h), "preconditioner creation")
  end subroutine

  !> y = x / diag (diagonal_preconditioner_type, sci_diagonal_preconditioner_alg_mod.x90:71-106)
  subroutine device_diagonal_preconditioner_init(self, diag)
    type(device_preconditioner_type), intent(inout) :: self
    type(device_vector_type),         intent(in)    :: diag
    call lfx_check(lfx_diag_prec_create(lfx_context, diag%h, self%h), "preconditioner creation")
  end subroutine

  !> Thomas on the rows the column operator covers
  !> (columnwise_op_appinv_kernel_mod.F90:77-145), y = x / diag on the others;
  !> precision: the vectors it will be applied to
  subroutine device_cma_preconditioner_init(self, cma, diag, precision)
    type(device_preconditioner_type), intent(inout) :: self
    type(device_cma_type),            intent(in)    :: cma
    type(device_vector_type),         intent(in)    :: diag
    integer(c_int32_t),               intent(in)    :: precision
    call lfx_check(lfx_cma_prec_create(lfx_context, cma%h, diag%h, precision, self%h), &
                   "preconditioner creation")
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
      class default
        call log_event("lfx: preconditioner apply: y is not a device_vector_type", LOG_LEVEL_ERROR)
      end select
    class default
      call log_event("lfx: preconditioner apply: x is not a device_vector_type", LOG_LEVEL_ERROR)
    end select
  end subroutine

  subroutine dprec_destroy(self)
    type(device_preconditioner_type), intent(inout) :: self
    integer(c_int) :: rc
    if (c_associated(self%h)) rc = lfx_prec_destroy(self%h)
    self%h = c_null_ptr
  end subroutine

  ! ------------------------------------------------------------------ solvers
  !> The constructors of conjugate_gradient_type, BiCGstab_type, gmres_type,
  !> fgmres_type and gcr_type (sci_iterative_solver_mod.f90:101-113, 137-149,
  !> 175-188): kind is LFX_SOLVER_CG ... LFX_SOLVER_GCR, gcrk is ignored by CG
  !> and BiCGStab.
  subroutine device_krylov_solver_init(self, kind, lin_op, prec, r_tol, a_tol, max_iter, &
                                       monitor_convergence, fail_on_non_converged, gcrk)
    type(device_krylov_solver_type),  intent(inout) :: self
    integer(c_int32_t),               intent(in)    :: kind
    type(device_lma_operator_type),   intent(in)    :: lin_op
    type(device_preconditioner_type), intent(in)    :: prec
    real(kind=r_def),                 intent(in)    :: r_tol, a_tol
    integer(kind=i_def),              intent(in)    :: max_iter
    logical(kind=l_def),              intent(in)    :: monitor_convergence, fail_on_non_converged
    integer(kind=i_def), optional,    intent(in)    :: gcrk
    type(lfx_solver_cfg) :: cfg
    cfg = solver_cfg(r_tol, a_tol, max_iter, monitor_convergence, fail_on_non_converged, gcrk)
    call lfx_check(lfx_solver_create(lfx_context, kind, lin_op%h, prec%h, cfg, self%h), &
                   "solver creation")
  end subroutine device_krylov_solver_init

  !> Mixed precision: FP64 iterative refinement (residual b - A x and solution
  !> update in FP64 with op64) around `inner`, an FP32 solver on an FP32 copy
  !> of the operator, each correction solved to inner_rtol.
  subroutine device_refined_solver_init(self, op64, inner, inner_rtol, r_tol, a_tol, max_iter, &
                                        monitor_convergence, fail_on_non_converged)
    type(device_krylov_solver_type), intent(inout) :: self
    type(device_lma_operator_type),  intent(in)    :: op64
    type(device_krylov_solver_type), intent(in)    :: inner
    real(kind=r_def),                intent(in)    :: inner_rtol, r_tol, a_tol
    integer(kind=i_def),             intent(in)    :: max_iter
    logical(kind=l_def),             intent(in)    :: monitor_convergence, fail_on_non_converged
    type(lfx_solver_cfg) :: cfg
    cfg = solver_cfg(r_tol, a_tol, max_iter, monitor_convergence, fail_on_non_converged)
    call lfx_check(lfx_refined_solver_create(lfx_context, op64%h, inner%h,              &
                                             real(inner_rtol, c_double), cfg, self%h), &
                   "refined solver creation")
  end subroutine device_refined_solver_init

  function solver_cfg(r_tol, a_tol, max_iter, monitor_convergence, fail_on_non_converged, &
                      gcrk) result(cfg)
    real(kind=r_def),              intent(in) :: r_tol, a_tol
    integer(kind=i_def),           intent(in) :: max_iter
    logical(kind=l_def),           intent(in) :: monitor_convergence, fail_on_non_converged
    integer(kind=i_def), optional, intent(in) :: gcrk
    type(lfx_solver_cfg) :: cfg
    cfg%r_tol = real(r_tol, c_double)
    cfg%a_tol = real(a_tol, c_double)
    cfg%max_iter = int(max_iter, c_int32_t)
    cfg%gcrk = 0_c_int32_t
    if (present(gcrk)) cfg%gcrk = int(gcrk, c_int32_t)
    cfg%monitor_convergence = merge(1_c_int32_t, 0_c_int32_t, monitor_convergence)
    cfg%fail_on_non_converged = merge(1_c_int32_t, 0_c_int32_t, fail_on_non_converged)
  end function solver_cfg

  !> apply(x, b) of abstract_iterative_solver_type: the whole solve on the
  !> device; a non-converged solve aborts only when fail_on_non_converged was
  !> set, as in the reference
  subroutine dsolver_apply(self, x, b)
    class(device_krylov_solver_type), intent(inout) :: self
    class(abstract_vector_type),      intent(inout) :: x
    class(abstract_vector_type),      intent(inout) :: b
    select type (x)
    type is (device_vector_type)
      select type (b)
      type is (device_vector_type)
        call lfx_check(lfx_solver_apply(self%h, x%h, b%h, self%info), "solve")
      class default
        call log_event("lfx: solve: b is not a device_vector_type", LOG_LEVEL_ERROR)
      end select
    class default
      call log_event("lfx: solve: x is not a device_vector_type", LOG_LEVEL_ERROR)
    end select
  end subroutine dsolver_apply

  subroutine dsolver_destroy(self)
    type(device_krylov_solver_type), intent(inout) :: self
    integer(c_int) :: rc
    if (c_associated(self%h)) rc = lfx_solver_destroy(self%h)
    self%h = c_null_ptr
  end subroutine

end module lfx_device_mod
