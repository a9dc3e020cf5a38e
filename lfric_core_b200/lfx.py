"""Python mirror of the reference's solver API over the liblfx C ABI.

The classes follow the reference's abstract types and their concrete
extensions, with the same procedure names and argument meanings:

  FieldVector            abstract_vector_type (vector_mod.F90:17-189),
                         field_vector_type / r_solver_field_vector_type
  LmaOperator            abstract_linear_operator_type + operator_type /
                         mass_matrix_operator_type (matrix_vector_kernel)
  NullPreconditioner,
  DiagonalPreconditioner,
  ColumnwisePreconditioner abstract_preconditioner_type
  ColumnwiseOperator     columnwise_operator_type (CMA)
  ConjugateGradient, BiCGStab, GMRES
                         conjugate_gradient_type, BiCGstab_type, gmres_type
                         (sci_iterative_solver_mod.f90), device resident
  RefinedSolver          FP64 iterative refinement around an FP32 inner solve

Where the reference calls log_event(..., LOG_LEVEL_ERROR) (which aborts), the
mirror raises LfxError carrying the C status code. Everything runs on the GPU
through liblfx.so; there is no CPU fallback, and importing this module on a
machine without the built library or without a GPU fails loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "liblfx.so"
_lib = None

STATUS = {0: "OK", 1: "NOT_CONVERGED", 2: "NAN_DETECTED", 3: "OUT_OF_MEMORY",
          4: "INVALID_ARGUMENT", 5: "TYPE_MISMATCH", 6: "TIMEOUT", 7: "CUDA_ERROR",
          8: "NOT_SUPPORTED"}
R64, R32 = 64, 32
CG, BICGSTAB, GMRES_KIND, FGMRES_KIND, GCR_KIND = 1, 2, 3, 4, 5

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
vp = C.c_void_p


class SolverCfg(C.Structure):
    _fields_ = [("r_tol", C.c_double), ("a_tol", C.c_double), ("max_iter", C.c_int32),
                ("gcrk", C.c_int32), ("monitor_convergence", C.c_int32),
                ("fail_on_non_converged", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32),
                ("initial_norm", C.c_double), ("final_norm", C.c_double),
                ("final_rel", C.c_double), ("applies", C.c_int32), ("status", C.c_int32),
                ("outer_iterations", C.c_int32), ("inner_iterations", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MrhsCfg(C.Structure):
    _fields_ = [("r_tol", C.c_double), ("inner_tol", C.c_double), ("max_outer", C.c_int32),
                ("max_inner", C.c_int32), ("method", C.c_int32)]


MRHS_TF32, MRHS_BF16 = 1, 2
MRHS_PER_RHS_CG, MRHS_BLOCK_CG = 0, 1


class BatchTuning(C.Structure):
    _fields_ = [("cells_per_item", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("grid", C.c_int32), ("cooperative", C.c_int32), ("group_bytes", C.c_int64),
                ("replays", C.c_int64), ("us_per_iteration", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# (name, argtypes, restype)
_SIGS = [
    ("lfx_ctx_create", [C.c_int, C.POINTER(vp)], C.c_int),
    ("lfx_ctx_destroy", [vp], C.c_int),
    ("lfx_last_error", [vp], C.c_char_p),
    ("lfx_ctx_synchronize", [vp], C.c_int),
    ("lfx_ctx_stream", [vp], vp),
    ("lfx_ctx_device_bytes", [vp], C.c_int64),
    ("lfx_ctx_enable_apply_timing", [vp, C.c_int32], C.c_int),
    ("lfx_ctx_apply_timing", [vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_double),
                              C.c_int32], C.c_int),
    ("lfx_ctx_launch_count", [vp], C.c_int64),
    ("lfx_ctx_set_apply_kernel", [vp, C.c_int32], C.c_int),
    ("lfx_ctx_check_device_error", [vp], C.c_int),
    ("lfx_vec_create", [vp, C.c_int32, i64p, C.c_int32, C.POINTER(vp)], C.c_int),
    ("lfx_vec_duplicate", [vp, C.POINTER(vp)], C.c_int),
    ("lfx_vec_destroy", [vp], C.c_int),
    ("lfx_vec_set_scalar", [vp, C.c_double], C.c_int),
    ("lfx_vec_axpy", [vp, C.c_double, vp], C.c_int),
    ("lfx_vec_aypx", [vp, C.c_double, vp], C.c_int),
    ("lfx_vec_axpby", [vp, C.c_double, vp, C.c_double, vp], C.c_int),
    ("lfx_vec_norm", [vp, C.POINTER(C.c_double)], C.c_int),
    ("lfx_vec_field_norm", [vp, C.c_int32, C.POINTER(C.c_double)], C.c_int),
    ("lfx_vec_dot", [vp, vp, C.POINTER(C.c_double)], C.c_int),
    ("lfx_vec_scale", [vp, C.c_double], C.c_int),
    ("lfx_vec_copy", [vp, vp], C.c_int),
    ("lfx_vec_size", [vp, C.POINTER(C.c_int32)], C.c_int),
    ("lfx_vec_import_field", [vp, C.c_int32, f64p, C.c_int64], C.c_int),
    ("lfx_vec_export_field", [vp, C.c_int32, f64p, C.c_int64], C.c_int),
    ("lfx_vec_import_field_async", [vp, C.c_int32, vp, C.c_int64, vp], C.c_int),
    ("lfx_vec_export_field_async", [vp, C.c_int32, vp, C.c_int64, vp], C.c_int),
    ("lfx_vec_field_device_ptr", [vp, C.c_int32, C.POINTER(vp)], C.c_int),
    ("lfx_lma_create", [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, i32p, i32p, C.c_int64,
                        C.c_int64, f64p, C.c_int32, i32p, i32p, C.c_int32, C.c_int32,
                        C.POINTER(vp)], C.c_int),
    ("lfx_lma_create_like", [vp, f64p, C.c_int32, C.POINTER(vp)], C.c_int),
    ("lfx_lma_sum", [vp, C.c_double, vp, C.POINTER(vp)], C.c_int),
    ("lfx_op_apply", [vp, vp, vp], C.c_int),
    ("lfx_op_autotune", [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                         C.POINTER(C.c_int32), C.POINTER(C.c_float)], C.c_int),
    ("lfx_op_set_apply", [vp, C.c_int32, C.c_int32, C.c_int32], C.c_int),
    ("lfx_op_storage", [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    ("lfx_op_time_apply", [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                           C.POINTER(C.c_float)], C.c_int),
    ("lfx_op_apply_transpose", [vp, vp, vp], C.c_int),
    ("lfx_op_destroy", [vp], C.c_int),
    ("lfx_lma_diagonal", [vp, vp], C.c_int),
    ("lfx_cma_create", [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                        C.c_int32, C.c_int32, i32p, i32p, vp, C.POINTER(vp)], C.c_int),
    ("lfx_cma_assemble_from_lma", [vp, C.c_int32, i32p, i32p, C.c_int32, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_int32, C.c_int32, i32p, i32p, C.POINTER(vp)],
     C.c_int),
    ("lfx_cma_create_banded", [vp] + [C.c_int32] * 8 + [vp, C.POINTER(vp)], C.c_int),
    ("lfx_cma_set_dofmap", [vp, i32p, i32p], C.c_int),
    ("lfx_cma_mul", [vp, vp, vp], C.c_int),
    ("lfx_cma_product", [vp, vp, C.POINTER(vp)], C.c_int),
    ("lfx_cma_scaledadd", [vp, vp, vp, C.c_double, C.c_double], C.c_int),
    ("lfx_cma_sum", [vp, vp, C.c_double, C.c_double, C.POINTER(vp)], C.c_int),
    ("lfx_cma_assemble_m2v_lumped_inv", [vp, i32p] + [C.c_int32] * 6 + [C.POINTER(vp)], C.c_int),
    ("lfx_cma_assemble_diag_hmht", [vp, vp, i32p] + [C.c_int32] * 6 + [C.POINTER(vp)],
     C.c_int),
    ("lfx_w2_split_create", [vp, C.c_int32, C.c_int32, i32p, i32p, i32p, i32p, C.c_int64, i32p,
                             i32p, C.POINTER(vp)], C.c_int),
    ("lfx_w2_split_field", [vp, vp, vp, vp], C.c_int),
    ("lfx_w2_combine_field", [vp, vp, vp, vp], C.c_int),
    ("lfx_w2_split_destroy", [vp], C.c_int),
    ("lfx_cma_get_band", [vp, f64p], C.c_int),
    ("lfx_cma_apply", [vp, vp, vp], C.c_int),
    ("lfx_cma_destroy", [vp], C.c_int),
    ("lfx_null_prec_create", [vp, C.POINTER(vp)], C.c_int),
    ("lfx_diag_prec_create", [vp, vp, C.POINTER(vp)], C.c_int),
    ("lfx_cma_prec_create", [vp, vp, vp, C.c_int32, C.POINTER(vp)], C.c_int),
    ("lfx_prec_apply", [vp, vp, vp], C.c_int),
    ("lfx_prec_destroy", [vp], C.c_int),
    ("lfx_solver_create", [vp, C.c_int32, vp, vp, C.POINTER(SolverCfg), C.POINTER(vp)], C.c_int),
    ("lfx_refined_solver_create", [vp, vp, vp, C.c_double, C.POINTER(SolverCfg), C.POINTER(vp)],
     C.c_int),
    ("lfx_solver_apply", [vp, vp, vp, C.POINTER(SolveInfo)], C.c_int),
    ("lfx_solver_destroy", [vp], C.c_int),
    ("lfx_solver_set_tolerance", [vp, C.c_double, C.c_double], C.c_int),
    ("lfx_fem_w0_operator", [vp, C.c_int32, C.c_int32, i32p, C.c_int64, f64p, C.c_double, i32p,
                             C.c_int64, C.c_int32, i32p, i32p, C.c_int32, C.POINTER(vp),
                             C.POINTER(vp)], C.c_int),
    ("lfx_fem_w2_operator", [vp, C.c_int32, C.c_int32, i32p, i32p, C.c_int64, f64p, C.c_double,
                             i32p, C.c_int64, C.c_int32, i32p, i32p, C.c_int32, C.POINTER(vp),
                             C.POINTER(vp)], C.c_int),
    ("lfx_batch_create", [vp, C.c_int32, C.c_int32, C.c_int64, C.c_int32, C.POINTER(vp)],
     C.c_int),
    ("lfx_batch_autotune", [vp, C.c_int32, C.POINTER(BatchTuning)], C.c_int),
    ("lfx_batch_get_tuning", [vp, C.POINTER(BatchTuning)], C.c_int),
    ("lfx_batch_set_tuning", [vp, C.c_int32, C.c_int32, C.c_int64], C.c_int),
    ("lfx_batch_set_wait_limit", [vp, C.c_double], C.c_int),
    ("lfx_batch_destroy", [vp], C.c_int),
    ("lfx_batch_admit", [vp, vp, vp, vp, vp, vp, C.c_double, C.c_int32, C.c_int64,
                         C.POINTER(C.c_int32)], C.c_int),
    ("lfx_batch_step", [vp, C.POINTER(C.c_int32)], C.c_int),
    ("lfx_batch_slot_info", [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                             C.POINTER(SolveInfo)], C.c_int),
    ("lfx_batch_retire", [vp, C.c_int32], C.c_int),
    ("lfx_precondition_only_solver_create", [vp, vp, vp, C.c_int32, C.POINTER(vp)], C.c_int),
    ("lfx_jacobi_solver_create", [vp, vp, vp, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                  C.c_int32, C.c_double, C.POINTER(vp)], C.c_int),
    ("lfx_chebyshev_solver_create", [vp, vp, vp, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                     C.c_int32, C.c_double, C.c_double, C.POINTER(vp)], C.c_int),
    ("lfx_mrhs_create", [vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(vp)], C.c_int),
    ("lfx_mrhs_destroy", [vp], C.c_int),
    ("lfx_mrhs_info", [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                       C.POINTER(C.c_int32), C.POINTER(C.c_int64)], C.c_int),
    ("lfx_mrhs_apply", [vp, vp, vp], C.c_int),
    ("lfx_mrhs_time_apply", [vp, vp, vp, C.c_int32, C.POINTER(C.c_float)], C.c_int),
    ("lfx_mrhs_autotune", [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_float)], C.c_int),
    ("lfx_mrhs_solve", [vp, vp, vp, vp, vp, C.c_int64, C.POINTER(MrhsCfg), C.POINTER(SolveInfo)],
     C.c_int),
    ("lfx_mrhs_set_gram", [vp, C.c_int32], C.c_int),
    ("lfx_mrhs_gram", [vp, vp, vp, vp, C.c_int32, C.c_int32, vp], C.c_int),
    ("lfx_dot_noalloc", [vp, vp, C.c_int64, vp, vp], C.c_int),
    ("lfx_dot_noalloc_max_n", [], C.c_int64),
    ("lfx_noalloc_last_error", [], C.c_char_p),
]
EXPORTED = [s[0] for s in _SIGS]


def load_library(path: Path | None = None):
    """Load liblfx.so (no GPU needed to load) and bind every signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else _LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is not built; run python -m lfric_core_b200.build")
    L = C.CDLL(str(p))
    for name, args, res in _SIGS:
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    if path is None:
        _lib = L
    return L


class LfxError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Context:
    """One device, one CUDA stream (lfx_ctx)."""

    def __init__(self, device: int = 0):
        self.L = load_library()
        h = vp()
        rc = self.L.lfx_ctx_create(device, C.byref(h))
        if rc:
            raise LfxError(rc, f"cannot create a context on device {device}")
        self.h = h

    def check(self, rc):
        if rc:
            raise LfxError(rc, self.L.lfx_last_error(self.h).decode())
        return rc

    def synchronize(self):
        self.check(self.L.lfx_ctx_synchronize(self.h))

    @property
    def stream(self) -> int:
        return self.L.lfx_ctx_stream(self.h) or 0

    def device_bytes(self) -> int:
        return self.L.lfx_ctx_device_bytes(self.h)

    def enable_apply_timing(self, on: bool = True):
        self.check(self.L.lfx_ctx_enable_apply_timing(self.h, 1 if on else 0))

    def apply_timing(self, precision: int = 0, reset: bool = True):
        """(launches, total ms) of the timed LMA applies of one storage
        precision (0 = all) since the last reset."""
        n = C.c_int64()
        ms = C.c_double()
        self.check(self.L.lfx_ctx_apply_timing(self.h, precision, C.byref(n), C.byref(ms),
                                               1 if reset else 0))
        return n.value, ms.value

    def launch_count(self) -> int:
        return self.L.lfx_ctx_launch_count(self.h)

    def set_apply_kernel(self, which: int):
        """-1: per-operator choice (autotuned, else register gather), 0: bulk-copy
        pipelined LMA apply, 1: register gather, 3: register gather with
        prefetched column descriptors, 4: copy-staged pipeline, 5: cell scatter
        (one launch per colour)."""
        self.check(self.L.lfx_ctx_set_apply_kernel(self.h, which))

    def check_device_error(self):
        self.check(self.L.lfx_ctx_check_device_error(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.L.lfx_ctx_destroy(self.h)
            self.h = None


class _Handle:
    _destroy = None

    def close(self):
        """Destroys the device object now (otherwise when collected)."""
        h = getattr(self, "h", None)
        if h and self._destroy and _lib is not None:
            getattr(_lib, self._destroy)(h)
        self.h = None

    def __del__(self):
        self.close()


class FieldVector(_Handle):
    """field_vector_type: nfields device fields (FP64, or FP32 for the
    r_solver variant)."""

    _destroy = "lfx_vec_destroy"

    def __init__(self, ctx: Context, undf, precision: int = R64, _h=None):
        self.ctx = ctx
        self.undf = [int(u) for u in (undf if np.ndim(undf) else [undf])]
        self.precision = precision
        if _h is not None:
            self.h = _h
            return
        h = vp()
        ctx.check(ctx.L.lfx_vec_create(ctx.h, len(self.undf), np.array(self.undf, dtype=np.int64),
                                       precision, C.byref(h)))
        self.h = h

    @classmethod
    def from_array(cls, ctx, data, precision=R64):
        v = cls(ctx, [len(data)], precision)
        v.import_field(np.asarray(data, dtype=np.float64), 1)
        return v

    # abstract_vector_type procedures
    def set_scalar(self, scalar):
        self.ctx.check(self.ctx.L.lfx_vec_set_scalar(self.h, scalar))

    def axpy(self, alpha, x):
        self.ctx.check(self.ctx.L.lfx_vec_axpy(self.h, alpha, x.h))

    def aypx(self, alpha, x):
        self.ctx.check(self.ctx.L.lfx_vec_aypx(self.h, alpha, x.h))

    def axpby(self, a, x, b, y):
        self.ctx.check(self.ctx.L.lfx_vec_axpby(self.h, a, x.h, b, y.h))

    def norm(self):
        out = C.c_double()
        self.ctx.check(self.ctx.L.lfx_vec_norm(self.h, C.byref(out)))
        return out.value

    def field_norm(self, n):
        out = C.c_double()
        self.ctx.check(self.ctx.L.lfx_vec_field_norm(self.h, n, C.byref(out)))
        return out.value

    def dot(self, x):
        out = C.c_double()
        self.ctx.check(self.ctx.L.lfx_vec_dot(self.h, x.h, C.byref(out)))
        return out.value

    def scale(self, scalar):
        self.ctx.check(self.ctx.L.lfx_vec_scale(self.h, scalar))

    def duplicate(self):
        h = vp()
        self.ctx.check(self.ctx.L.lfx_vec_duplicate(self.h, C.byref(h)))
        return FieldVector(self.ctx, self.undf, self.precision, _h=h)

    def copy(self, source):
        self.ctx.check(self.ctx.L.lfx_vec_copy(self.h, source.h))

    def vector_size(self):
        n = C.c_int32()
        self.ctx.check(self.ctx.L.lfx_vec_size(self.h, C.byref(n)))
        return n.value

    def import_field(self, data, position=1):
        a = np.ascontiguousarray(data, dtype=np.float64)
        self.ctx.check(self.ctx.L.lfx_vec_import_field(self.h, position, a, len(a)))

    def export_field(self, position=1, out=None):
        """Field `position` as FP64 host data; `out` (e.g. pinned memory) is
        filled in place when given."""
        if out is None:
            out = np.empty(self.undf[position - 1], dtype=np.float64)
        self.ctx.check(self.ctx.L.lfx_vec_export_field(self.h, position, out, len(out)))
        return out

    def import_field_async(self, host, stream: int = 0, position=1):
        """Queue the copy of FP64 host data (a pinned, contiguous float64
        array kept alive by the caller) into field `position` on `stream`
        (a cudaStream_t handle; 0 = the context's stream); returns at once."""
        assert host.dtype == np.float64 and host.flags["C_CONTIGUOUS"]
        self.ctx.check(self.ctx.L.lfx_vec_import_field_async(
            self.h, position, C.c_void_p(host.ctypes.data), len(host), C.c_void_p(stream)))

    def export_field_async(self, host, stream: int = 0, position=1):
        """Queue the copy of field `position` into FP64 host memory (pinned,
        contiguous, kept alive by the caller) on `stream`; returns at once."""
        assert host.dtype == np.float64 and host.flags["C_CONTIGUOUS"]
        self.ctx.check(self.ctx.L.lfx_vec_export_field_async(
            self.h, position, C.c_void_p(host.ctypes.data), len(host), C.c_void_p(stream)))

    def device_ptr(self, position=1) -> int:
        p = vp()
        self.ctx.check(self.ctx.L.lfx_vec_field_device_ptr(self.h, position, C.byref(p)))
        return p.value


# LMA apply kernels by number (lfx_op_autotune / lfx_op_set_apply)
APPLY_KERNEL_NAMES = {0: "pipeline", 1: "register-gather", 2: "generic",
                      3: "register-gather-prefetch", 4: "staged-pipeline", 5: "cell-scatter",
                      6: "cell-scatter-persistent"}


class LmaOperator(_Handle):
    """operator_type applied by the coloured matrix_vector_kernel: y = A x."""

    _destroy = "lfx_op_destroy"

    def __init__(self, ctx, ncell_2d, nlayers, ndf_to, ndf_from, map_to, map_from, undf_to,
                 undf_from, local_stencil, ncells_per_colour, cells_in_colour,
                 precision=R64, _h=None):
        self.ctx = ctx
        self.precision = precision
        self.undf_to, self.undf_from = int(undf_to), int(undf_from)
        self._shape = (ncell_2d, nlayers, ndf_to, ndf_from)
        if _h is not None:
            self.h = _h
            return
        cic = np.ascontiguousarray(cells_in_colour, dtype=np.int32)
        h = vp()
        ctx.check(ctx.L.lfx_lma_create(
            ctx.h, ncell_2d, nlayers, ndf_to, ndf_from,
            np.ascontiguousarray(map_to, dtype=np.int32), np.ascontiguousarray(map_from, dtype=np.int32),
            undf_to, undf_from, np.ascontiguousarray(local_stencil, dtype=np.float64),
            len(ncells_per_colour), np.ascontiguousarray(ncells_per_colour, dtype=np.int32), cic,
            cic.shape[0], precision, C.byref(h)))
        self.h = h

    def like(self, local_stencil, precision):
        """Same dofmaps and colouring, new local matrices / precision."""
        h = vp()
        self.ctx.check(self.ctx.L.lfx_lma_create_like(
            self.h, np.ascontiguousarray(local_stencil, dtype=np.float64), precision, C.byref(h)))
        op = LmaOperator(self.ctx, *self._shape, None, None, self.undf_to, self.undf_from, None,
                         None, None, precision=precision, _h=h)
        op._parent = self
        return op

    def x_plus_ay(self, a, y: "LmaOperator") -> "LmaOperator":
        """operator_x_plus_ay: a new operator self + a y on the same layout
        (y made from self, or self from y, by like())."""
        h = vp()
        self.ctx.check(self.ctx.L.lfx_lma_sum(self.h, float(a), y.h, C.byref(h)))
        op = LmaOperator(self.ctx, *self._shape, None, None, self.undf_to, self.undf_from, None,
                         None, None, precision=self.precision, _h=h)
        op._parent = self
        return op

    def apply(self, x, y):
        self.ctx.check(self.ctx.L.lfx_op_apply(self.h, x.h, y.h))

    def autotune(self, reps: int = 10) -> dict:
        """Time the apply launch configurations on this operator and keep the
        fastest; returns the choice."""
        k, s, w, us = C.c_int32(), C.c_int32(), C.c_int32(), C.c_float()
        self.ctx.check(self.ctx.L.lfx_op_autotune(self.h, reps, C.byref(k), C.byref(s),
                                                   C.byref(w), C.byref(us)))
        return {"kernel": APPLY_KERNEL_NAMES[k.value], "stages": s.value, "warps": w.value,
                "us": round(us.value, 2)}

    def storage(self) -> dict:
        """Bytes of the full local-matrix copy and of the packed upper
        triangle (0 unless the operator is symmetric on one dofmap)."""
        f, p = C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.L.lfx_op_storage(self.h, C.byref(f), C.byref(p)))
        return {"full_bytes": f.value, "packed_bytes": p.value}

    def set_apply(self, kernel: int, stages: int = 0, warps: int = 0):
        """Keep one apply launch configuration for this operator (as the
        autotuner would); raises if it does not fit."""
        self.ctx.check(self.ctx.L.lfx_op_set_apply(self.h, kernel, stages, warps))

    def time_apply(self, kernel: int, stages: int = 0, warps: int = 0, reps: int = 10):
        us = C.c_float()
        rc = self.ctx.L.lfx_op_time_apply(self.h, kernel, stages, warps, reps, C.byref(us))
        if rc == 8:  # configuration does not fit
            return None
        self.ctx.check(rc)
        return us.value

    def apply_transpose(self, x, y):
        self.ctx.check(self.ctx.L.lfx_op_apply_transpose(self.h, x.h, y.h))

    def diagonal(self, diag):
        self.ctx.check(self.ctx.L.lfx_lma_diagonal(self.h, diag.h))


def fem_operators(ctx, mesh, space, coef, precisions=(R64, R32)):
    """Assemble the W0 (A = M + coef K) or W2 (A = M2 + coef D^T D) local
    matrices of an extruded mesh on the device; returns {precision: LmaOperator}
    sharing one layout, plus the dofmap and undf."""
    from . import meshgen as mg
    m, undf = mesh.dofmap(space)
    npc, cic = mesh.colour_lookup()
    h64, h32 = vp(), vp()
    p64 = C.byref(h64) if R64 in precisions else None
    p32 = C.byref(h32) if R32 in precisions else None
    nv = len(mesh.vert_xyz)
    args = (ctx.h, mesh.ncell_2d, mesh.nlayers)
    tail = (m, undf, len(npc), npc, np.ascontiguousarray(cic), cic.shape[0], p64, p32)
    if space == mg.W0:
        ctx.check(ctx.L.lfx_fem_w0_operator(*args, mesh.verts_on_cell, nv, mesh.xyz3d, coef, *tail))
        ndf = 8
    else:
        ctx.check(ctx.L.lfx_fem_w2_operator(*args, mesh.cell_next, mesh.verts_on_cell, nv,
                                            mesh.xyz3d, coef, *tail))
        ndf = 6
    ops = {}
    for prec, h in ((R64, h64), (R32, h32)):
        if prec in precisions:
            ops[prec] = LmaOperator(ctx, mesh.ncell_2d, mesh.nlayers, ndf, ndf, None, None, undf,
                                    undf, None, None, None, precision=prec, _h=h)
    first = ops.get(R64)
    for op in ops.values():
        if op is not first and first is not None:
            op._parent = first
    return ops, m, undf


class MultiRhsOperator(_Handle):
    """One LMA operator applied to nrhs right-hand sides at once, the per-cell
    products on the tensor cores (lfx_mrhs). Vectors are device arrays of
    undf x nrhs FP32 values, dof-major, passed as device pointers (ints)."""

    _destroy = "lfx_mrhs_destroy"

    def __init__(self, op: "LmaOperator", kind: int = MRHS_TF32, nrhs: int = 64,
                 cells_per_patch: int = 0):
        self.ctx = op.ctx
        self.op = op
        self.kind = kind
        self.nrhs = nrhs
        h = vp()
        self.ctx.check(self.ctx.L.lfx_mrhs_create(op.h, kind, nrhs, cells_per_patch, C.byref(h)))
        self.h = h

    def info(self) -> dict:
        npatch, mo, mc = C.c_int32(), C.c_int32(), C.c_int32()
        cl, mb = C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.L.lfx_mrhs_info(self.h, C.byref(npatch), C.byref(cl), C.byref(mo),
                                                C.byref(mc), C.byref(mb)))
        return {"patches": npatch.value, "cell_levels": cl.value, "max_owned": mo.value,
                "max_colours": mc.value, "matrix_bytes": mb.value}

    def apply(self, x_ptr: int, y_ptr: int):
        self.ctx.check(self.ctx.L.lfx_mrhs_apply(self.h, x_ptr, y_ptr))

    def time_apply(self, x_ptr: int, y_ptr: int, reps: int = 20) -> float:
        us = C.c_float()
        self.ctx.check(self.ctx.L.lfx_mrhs_time_apply(self.h, x_ptr, y_ptr, reps, C.byref(us)))
        return us.value

    def autotune(self, reps: int = 10) -> dict:
        lb, us = C.c_int32(), C.c_float()
        self.ctx.check(self.ctx.L.lfx_mrhs_autotune(self.h, reps, C.byref(lb), C.byref(us)))
        return {"levels_per_block": lb.value, "us": us.value}

    def set_gram(self, tensor: bool):
        """Block CG Gram products on the tcgen05 tensor cores (True) or the
        FP32 cores."""
        self.ctx.check(self.ctx.L.lfx_mrhs_set_gram(self.h, 1 if tensor else 0))

    def gram(self, u_ptr: int, v0_ptr: int, v1_ptr: int, nv: int, tensor: bool, out_ptr: int):
        """out (device nv x 64 x 64 FP64) = U^T V_v for device FP32 blocks."""
        self.ctx.check(self.ctx.L.lfx_mrhs_gram(self.h, u_ptr, v0_ptr, v1_ptr or None, nv,
                                                1 if tensor else 0, out_ptr))

    def solve(self, op64: "LmaOperator", diag: "FieldVector", b_ptr: int, x_ptr: int, ld: int,
              r_tol=1e-8, inner_tol=1e-2, max_outer=20, max_inner=5000, method=MRHS_PER_RHS_CG):
        """FP64 refinement around the FP32 tensor-core CG for all right-hand
        sides (method: MRHS_PER_RHS_CG, or MRHS_BLOCK_CG for 64 right-hand
        sides); b, x: device FP64 arrays, right-hand side r at offset r * ld.
        Returns one SolveInfo per right-hand side."""
        cfg = MrhsCfg(r_tol, inner_tol, max_outer, max_inner, method)
        info = (SolveInfo * self.nrhs)()
        self.ctx.check(self.ctx.L.lfx_mrhs_solve(self.h, op64.h, diag.h, b_ptr, x_ptr, ld,
                                                 C.byref(cfg), info))
        return list(info)


class Batch(_Handle):
    """Continuous batching of independent SPD solves (lfx_batch): one
    persistent kernel launch per step runs `iters` CG iterations of every
    admitted slot. Admission takes the slot's Krylov state from free device
    memory and is refused (admit returns None) while it would leave less than
    reserve_bytes free or when every slot is taken."""

    _destroy = "lfx_batch_destroy"

    def __init__(self, ctx, ndf, max_slots, reserve_bytes=2 << 30, iters=8):
        self.ctx = ctx
        h = vp()
        ctx.check(ctx.L.lfx_batch_create(ctx.h, ndf, max_slots, int(reserve_bytes), iters,
                                         C.byref(h)))
        self.h = h
        self.max_slots = max_slots
        self._keep = {}

    def admit(self, op64, op32, prec32, b, x, tol, max_iter=10000, tag=0):
        s = C.c_int32()
        rc = self.ctx.L.lfx_batch_admit(self.h, op64.h, op32.h, prec32.h, b.h, x.h, tol, max_iter,
                                        tag, C.byref(s))
        if rc == 3:  # memory or slots full
            return None
        self.ctx.check(rc)
        self._keep[s.value] = (op64, op32, prec32, b, x)
        return s.value

    def autotune(self, iters=4):
        t = BatchTuning()
        self.ctx.check(self.ctx.L.lfx_batch_autotune(self.h, iters, C.byref(t)))
        return t.as_dict()

    def tuning(self):
        t = BatchTuning()
        self.ctx.check(self.ctx.L.lfx_batch_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, cells_per_item, blocks_per_sm, group_bytes):
        self.ctx.check(self.ctx.L.lfx_batch_set_tuning(self.h, cells_per_item, blocks_per_sm,
                                                       int(group_bytes)))

    def set_wait_limit(self, seconds):
        self.ctx.check(self.ctx.L.lfx_batch_set_wait_limit(self.h, float(seconds)))

    def step(self):
        nd = C.c_int32()
        self.ctx.check(self.ctx.L.lfx_batch_step(self.h, C.byref(nd)))
        return nd.value

    def slot(self, s):
        ph, tag, info = C.c_int32(), C.c_int64(), SolveInfo()
        self.ctx.check(self.ctx.L.lfx_batch_slot_info(self.h, s, C.byref(ph), C.byref(tag),
                                                      C.byref(info)))
        return ph.value, tag.value, info

    def done_slots(self):
        return [s for s in range(self.max_slots) if self.slot(s)[0] == 3]

    def retire(self, s):
        self.ctx.check(self.ctx.L.lfx_batch_retire(self.h, s))
        self._keep.pop(s, None)


class ColumnwiseOperator(_Handle):
    """columnwise_operator_type: banded matrix per column."""

    _destroy = "lfx_cma_destroy"

    def __init__(self, ctx, h, ncell_2d, nrow, bandwidth, ncol=None, params=None):
        self.ctx, self.h = ctx, h
        self.ncell_2d, self.nrow, self.bandwidth = ncell_2d, nrow, bandwidth
        self.ncol = nrow if ncol is None else ncol
        self.params = params  # (alpha, beta, gamma_m, gamma_p) when known

    @staticmethod
    def _gcd(a, b):
        while b:
            a, b = b, a % b
        return a

    @classmethod
    def banded(cls, ctx, ncell_2d, nrow, ncol, bandwidth, alpha, beta, gamma_m, gamma_p,
               band=None):
        """A map-free (possibly rectangular) operator from a host band, for
        the set-up algebra."""
        h = vp()
        b = None if band is None else np.ascontiguousarray(band, dtype=np.float64)
        ctx.check(ctx.L.lfx_cma_create_banded(ctx.h, ncell_2d, nrow, ncol, bandwidth, alpha, beta,
                                              gamma_m, gamma_p,
                                              None if b is None else b.ctypes.data, C.byref(h)))
        return cls(ctx, h, ncell_2d, nrow, bandwidth, ncol, (alpha, beta, gamma_m, gamma_p))

    @staticmethod
    def _derived(alpha, beta, gm, gp):
        g = ColumnwiseOperator._gcd(alpha, beta)
        if g > 1:
            alpha, beta, gm, gp = alpha // g, beta // g, gm // g, gp // g
        return (alpha, beta, gm, gp), 1 + -((-(gm + gp)) // beta)

    def product(self, other: "ColumnwiseOperator") -> "ColumnwiseOperator":
        """columnwise_operator_product + mul: self . other"""
        h = vp()
        self.ctx.check(self.ctx.L.lfx_cma_product(self.h, other.h, C.byref(h)))
        (a1, b1, m1, p1), (a2, b2, m2, p2) = self.params, other.params
        prm, bw = self._derived(a1 * a2, b1 * b2, a2 * m1 + b1 * m2, a2 * p1 + b1 * p2)
        return ColumnwiseOperator(self.ctx, h, self.ncell_2d, self.nrow, bw, other.ncol, prm)

    def sum(self, other: "ColumnwiseOperator", alpha, beta) -> "ColumnwiseOperator":
        """columnwise_operator_sum + scaledadd: alpha self + beta other"""
        h = vp()
        self.ctx.check(self.ctx.L.lfx_cma_sum(self.h, other.h, alpha, beta, C.byref(h)))
        (a1, b1, m1, p1), (_, _, m2, p2) = self.params, other.params
        prm, bw = self._derived(a1, b1, max(m1, m2), max(p1, p2))
        return ColumnwiseOperator(self.ctx, h, self.ncell_2d, self.nrow, bw, self.ncol, prm)

    def set_dofmap(self, first_dof, indirection):
        self.ctx.check(self.ctx.L.lfx_cma_set_dofmap(
            self.h, np.ascontiguousarray(first_dof, dtype=np.int32),
            np.ascontiguousarray(indirection, dtype=np.int32)))

    @classmethod
    def m2v_lumped_inv(cls, lma: "LmaOperator", column_banded_dofmap, params, bandwidth, nrow):
        """columnwise_op_asm_m2v_lumped_inv from a square FP64 LMA."""
        ctx = lma.ctx
        h = vp()
        cbd = np.ascontiguousarray(column_banded_dofmap, dtype=np.int32)
        ctx.check(ctx.L.lfx_cma_assemble_m2v_lumped_inv(lma.h, cbd, *params, bandwidth, nrow,
                                                        C.byref(h)))
        return cls(ctx, h, lma._shape[0], nrow, bandwidth, nrow, tuple(params))

    @classmethod
    def diag_hmht(cls, dh: "LmaOperator", m2h: "LmaOperator", column_banded_dofmap, params,
                  bandwidth, nrow):
        """columnwise_op_asm_diag_hmht from the W2h -> W3 LMA and the W2h mass."""
        ctx = dh.ctx
        h = vp()
        cbd = np.ascontiguousarray(column_banded_dofmap, dtype=np.int32)
        ctx.check(ctx.L.lfx_cma_assemble_diag_hmht(dh.h, m2h.h, cbd, *params, bandwidth, nrow,
                                                   C.byref(h)))
        return cls(ctx, h, dh._shape[0], nrow, bandwidth, nrow, tuple(params))

    @classmethod
    def from_band(cls, ctx, ncell_2d, nrow, bandwidth, alpha, beta, gamma_m, gamma_p, first_dof,
                  indirection, band):
        h = vp()
        b = np.ascontiguousarray(band, dtype=np.float64)
        ctx.check(ctx.L.lfx_cma_create(ctx.h, ncell_2d, nrow, nrow, bandwidth, alpha, beta,
                                       gamma_m, gamma_p,
                                       np.ascontiguousarray(first_dof, dtype=np.int32),
                                       np.ascontiguousarray(indirection, dtype=np.int32),
                                       b.ctypes.data, C.byref(h)))
        return cls(ctx, h, ncell_2d, nrow, bandwidth)

    @classmethod
    def assemble(cls, lma: LmaOperator, dfs, column_banded_dofmap, params, first_dof):
        """columnwise_op_asm from the local dofs `dfs` (1-based) of an FP64 LMA."""
        ctx = lma.ctx
        h = vp()
        cbd = np.ascontiguousarray(column_banded_dofmap, dtype=np.int32)
        ctx.check(ctx.L.lfx_cma_assemble_from_lma(
            lma.h, len(dfs), np.ascontiguousarray(dfs, dtype=np.int32), cbd, params["alpha"],
            params["beta"], params["gamma_m"], params["gamma_p"], params["bandwidth"],
            params["nrow"], np.ascontiguousarray(first_dof, dtype=np.int32),
            np.ascontiguousarray(params["indirection"], dtype=np.int32), C.byref(h)))
        return cls(ctx, h, lma._shape[0], params["nrow"], params["bandwidth"])

    def mul_into(self, other: "ColumnwiseOperator", out: "ColumnwiseOperator"):
        """out += self . other (columnwise_op_mul_kernel)"""
        self.ctx.check(self.ctx.L.lfx_cma_mul(self.h, other.h, out.h))

    def band(self):
        out = np.empty(self.ncell_2d * self.nrow * self.bandwidth)
        self.ctx.check(self.ctx.L.lfx_cma_get_band(self.h, out))
        return out

    def apply(self, x, y):
        self.ctx.check(self.ctx.L.lfx_cma_apply(self.h, x.h, y.h))


class W2Split(_Handle):
    """split_w2_field / combine_w2_field (lowest order): W2 <-> W2h + W2v.
    Maps are (ncell_2d, ndf) 1-based arrays."""

    _destroy = "lfx_w2_split_destroy"

    def __init__(self, ctx, nlayers, map_w2, map_w2h, map_w2v, map_w3_2d, undf_w3_2d,
                 face_selector_ew, face_selector_ns):
        self.ctx = ctx
        h = vp()
        as_i = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        ctx.check(ctx.L.lfx_w2_split_create(ctx.h, len(map_w2), nlayers, as_i(map_w2),
                                            as_i(map_w2h), as_i(map_w2v), as_i(map_w3_2d),
                                            undf_w3_2d, as_i(face_selector_ew),
                                            as_i(face_selector_ns), C.byref(h)))
        self.h = h

    def split(self, uvw, uv, w):
        self.ctx.check(self.ctx.L.lfx_w2_split_field(self.h, uvw.h, uv.h, w.h))

    def combine(self, uv, w, uvw):
        self.ctx.check(self.ctx.L.lfx_w2_combine_field(self.h, uv.h, w.h, uvw.h))


class _Prec(_Handle):
    _destroy = "lfx_prec_destroy"

    def apply(self, x, y):
        self.ctx.check(self.ctx.L.lfx_prec_apply(self.h, x.h, y.h))


class NullPreconditioner(_Prec):
    def __init__(self, ctx):
        self.ctx = ctx
        h = vp()
        ctx.check(ctx.L.lfx_null_prec_create(ctx.h, C.byref(h)))
        self.h = h


class DiagonalPreconditioner(_Prec):
    def __init__(self, ctx, diag: FieldVector):
        self.ctx = ctx
        h = vp()
        ctx.check(ctx.L.lfx_diag_prec_create(ctx.h, diag.h, C.byref(h)))
        self.h = h


class ColumnwisePreconditioner(_Prec):
    """Column tridiagonal inverse on the CMA's rows, Jacobi elsewhere."""

    def __init__(self, ctx, cma: ColumnwiseOperator, diag: FieldVector | None, precision=R64):
        self.ctx = ctx
        h = vp()
        ctx.check(ctx.L.lfx_cma_prec_create(ctx.h, cma.h, diag.h if diag is not None else None,
                                            precision, C.byref(h)))
        self.h = h
        self._keep = (cma, diag)


class _Solver(_Handle):
    _destroy = "lfx_solver_destroy"

    def set_tolerance(self, r_tol, a_tol=0.0):
        self.ctx.check(self.ctx.L.lfx_solver_set_tolerance(self.h, r_tol, a_tol))

    def apply(self, x: FieldVector, b: FieldVector) -> SolveInfo:
        info = SolveInfo()
        rc = self.ctx.L.lfx_solver_apply(self.h, x.h, b.h, C.byref(info))
        self.last_info = info
        if rc:
            self.ctx.check(rc)
        return info


def _cfg(r_tol, a_tol, max_iter, gcrk, monitor, fail):
    return SolverCfg(r_tol, a_tol, max_iter, gcrk, 1 if monitor else 0, 1 if fail else 0)


class _KrylovSolver(_Solver):
    KIND = 0

    def __init__(self, lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence=True,
                 fail_on_non_converged=False, gcrk=1):
        self.ctx = lin_op.ctx
        self.precision = lin_op.precision
        cfg = _cfg(r_tol, a_tol, max_iter, gcrk, monitor_convergence, fail_on_non_converged)
        h = vp()
        self.ctx.check(self.ctx.L.lfx_solver_create(self.ctx.h, self.KIND, lin_op.h, prec.h,
                                                     C.byref(cfg), C.byref(h)))
        self.h = h
        self._keep = (lin_op, prec)


class ConjugateGradient(_KrylovSolver):
    """conjugate_gradient_type(lin_op, prec, r_tol, a_tol, max_iter, ...)"""
    KIND = CG


class BiCGStab(_KrylovSolver):
    """BiCGstab_type(lin_op, prec, r_tol, a_tol, max_iter, ...)"""
    KIND = BICGSTAB


class GMRES(_KrylovSolver):
    """gmres_type(lin_op, prec, gcrk, r_tol, a_tol, max_iter, ...)"""
    KIND = GMRES_KIND

    def __init__(self, lin_op, prec, gcrk, r_tol, a_tol, max_iter, monitor_convergence=True,
                 fail_on_non_converged=False):
        super().__init__(lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence,
                         fail_on_non_converged, gcrk=gcrk)


class FGMRES(_KrylovSolver):
    """fgmres_type(lin_op, prec, gcrk, r_tol, a_tol, max_iter, ...): flexible
    GMRES; like the reference it starts from b (zero initial guess assumed)
    and adds the correction to x."""
    KIND = FGMRES_KIND

    def __init__(self, lin_op, prec, gcrk, r_tol, a_tol, max_iter, monitor_convergence=True,
                 fail_on_non_converged=False):
        super().__init__(lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence,
                         fail_on_non_converged, gcrk=gcrk)


class GCR(_KrylovSolver):
    """gcr_type(lin_op, prec, gcrk, r_tol, a_tol, max_iter, ...): right
    preconditioned GCR(gcrk); non-convergence (monitored) always raises, as
    the reference logs it as an error in both branches."""
    KIND = GCR_KIND

    def __init__(self, lin_op, prec, gcrk, r_tol, a_tol, max_iter, monitor_convergence=True,
                 fail_on_non_converged=False):
        super().__init__(lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence,
                         fail_on_non_converged, gcrk=gcrk)


class PreconditionOnly(_Solver):
    """precondition_only_type(lin_op, prec, monitor_convergence): x = P b."""

    def __init__(self, lin_op, prec, monitor_convergence=True):
        self.ctx = lin_op.ctx
        self.precision = lin_op.precision
        h = vp()
        self.ctx.check(self.ctx.L.lfx_precondition_only_solver_create(
            self.ctx.h, lin_op.h, prec.h, 1 if monitor_convergence else 0, C.byref(h)))
        self.h = h
        self._keep = (lin_op, prec)


class Jacobi(_Solver):
    """jacobi_type(lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence,
    fail_on_non_converged, rho_relax): x += -rho_relax P (A x - b)."""

    def __init__(self, lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence=True,
                 fail_on_non_converged=False, rho_relax=1.0):
        self.ctx = lin_op.ctx
        self.precision = lin_op.precision
        h = vp()
        self.ctx.check(self.ctx.L.lfx_jacobi_solver_create(
            self.ctx.h, lin_op.h, prec.h, r_tol, a_tol, max_iter, 1 if monitor_convergence else 0,
            1 if fail_on_non_converged else 0, rho_relax, C.byref(h)))
        self.h = h
        self._keep = (lin_op, prec)


class Chebyshev(_Solver):
    """chebyshev_type(lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence,
    fail_on_non_converged, lmin, lmax): max_iter Chebyshev steps from x = 0."""

    def __init__(self, lin_op, prec, r_tol, a_tol, max_iter, monitor_convergence=True,
                 fail_on_non_converged=False, lmin=0.0, lmax=2.0):
        self.ctx = lin_op.ctx
        self.precision = lin_op.precision
        h = vp()
        self.ctx.check(self.ctx.L.lfx_chebyshev_solver_create(
            self.ctx.h, lin_op.h, prec.h, r_tol, a_tol, max_iter, 1 if monitor_convergence else 0,
            1 if fail_on_non_converged else 0, lmin, lmax, C.byref(h)))
        self.h = h
        self._keep = (lin_op, prec)


class RefinedSolver(_Solver):
    """FP64 iterative refinement: r = b - A64 x in FP64, correction from an FP32
    inner solver run to inner_rtol, x += ||r|| d. Converged when
    ||b - A x|| / ||b - A x0|| <= r_tol."""

    def __init__(self, op64: LmaOperator, inner: _Solver, inner_rtol, r_tol, a_tol=0.0,
                 max_outer=20, fail_on_non_converged=False):
        self.ctx = op64.ctx
        self.precision = R64
        cfg = _cfg(r_tol, a_tol, max_outer, 0, True, fail_on_non_converged)
        h = vp()
        self.ctx.check(self.ctx.L.lfx_refined_solver_create(self.ctx.h, op64.h, inner.h,
                                                             inner_rtol, C.byref(cfg), C.byref(h)))
        self.h = h
        self._keep = (op64, inner)
