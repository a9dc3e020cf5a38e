"""ctypes wrapper of the oracle library (CPU FP64 restatement of the path).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, never by the lfric_core_b200 package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class Info(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32),
                ("initial_norm", C.c_double), ("final_norm", C.c_double),
                ("final_rel", C.c_double), ("applies", C.c_int32)]


def lib():
    global _lib
    if _lib is None:
        path = HERE / "build" / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing; run python oracle/build.py")
        L = C.CDLL(str(path))
        L.or_set_reduction_order.argtypes = [C.c_int]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_dot.argtypes = [f64p, f64p, C.c_int64]
        L.or_dot.restype = C.c_double
        L.or_sumsq.argtypes = [f64p, C.c_int64]
        L.or_sumsq.restype = C.c_double
        L.or_setval_c.argtypes = [f64p, C.c_double, C.c_int64]
        L.or_setval_x.argtypes = [f64p, f64p, C.c_int64]
        L.or_inc_x_plus_by.argtypes = [f64p, C.c_double, f64p, C.c_int64]
        L.or_inc_ax_plus_y.argtypes = [C.c_double, f64p, f64p, C.c_int64]
        L.or_ax_plus_by.argtypes = [f64p, C.c_double, f64p, C.c_double, f64p, C.c_int64]
        L.or_inc_a_times_x.argtypes = [C.c_double, f64p, C.c_int64]
        L.or_x_divideby_y.argtypes = [f64p, f64p, f64p, C.c_int64]
        L.or_matrix_vector_code.argtypes = [C.c_int32, C.c_int32, f64p, f64p, C.c_int64, f64p,
                                            C.c_int32, i32p, C.c_int32, i32p]
        L.or_transpose_matrix_vector_code.argtypes = L.or_matrix_vector_code.argtypes
        L.or_dg_matrix_vector_code.argtypes = L.or_matrix_vector_code.argtypes
        L.or_operator_x_plus_ay_code.argtypes = [C.c_int32, C.c_int32, C.c_int64, f64p, f64p,
                                                 C.c_double, f64p, C.c_int32, C.c_int32]
        L.or_tri_solve_code.argtypes = [C.c_int32, f64p, f64p, f64p, f64p, f64p, i32p]
        L.or_columnwise_op_asm_code.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64, f64p,
                                                f64p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                                C.c_int32, C.c_int32, C.c_int32, C.c_int32, i32p,
                                                C.c_int32, i32p]
        I = C.c_int32
        band_args = [f64p, I, I, I, I, I, I, I]  # band, nrow, ncol, bw, alpha, beta, g_m, g_p
        L.or_columnwise_op_mul_code.argtypes = [I, I] + band_args * 3
        L.or_columnwise_op_scaledadd_code.argtypes = [I, I] + band_args * 3 + [C.c_double,
                                                                               C.c_double]
        L.or_columnwise_op_asm_m2v_lumped_inv_code.argtypes = [I, I, I, I, f64p, f64p, I, I, I,
                                                               i32p]
        L.or_columnwise_op_asm_diag_hmht_code.argtypes = [I, I, I, I, f64p, f64p, f64p, I, I, I,
                                                          I, I, I, I, i32p, I]
        L.or_face_selector_code.argtypes = [i32p, i32p, i32p, i32p, i32p]
        L.or_split_w2_field_code.argtypes = [C.c_int32, f64p, f64p, f64p, i32p, i32p, i32p, i32p,
                                             i32p, i32p]
        L.or_combine_w2_field_code.argtypes = [C.c_int32, f64p, f64p, f64p, i32p, i32p, i32p,
                                               i32p, i32p, i32p]
        L.or_columnwise_op_app_code.argtypes = [C.c_int32, f64p, f64p, f64p, C.c_int32, C.c_int32,
                                                C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                                C.c_int32, i32p, i32p, i32p, i32p]
        L.or_columnwise_op_appinv_code.argtypes = [C.c_int32, f64p, f64p, f64p, C.c_int32,
                                                   C.c_int32, i32p, i32p]
        L.or_lma_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, i32p, i32p,
                                    C.c_int64, C.c_int64, f64p, C.c_int32, i32p, i32p,
                                    C.c_int32, C.c_int32]
        L.or_lma_create.restype = C.c_void_p
        L.or_op_apply.argtypes = [C.c_void_p, f64p, f64p]
        L.or_op_destroy.argtypes = [C.c_void_p]
        L.or_lma_diagonal.argtypes = [C.c_void_p, f64p]
        L.or_null_prec_create.argtypes = [C.c_int64]
        L.or_null_prec_create.restype = C.c_void_p
        L.or_diag_prec_create.argtypes = [f64p, C.c_int64]
        L.or_diag_prec_create.restype = C.c_void_p
        L.or_cma_prec_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, i32p, i32p, f64p,
                                         C.c_void_p, C.c_int64]
        L.or_cma_prec_create.restype = C.c_void_p
        L.or_prec_apply.argtypes = [C.c_void_p, f64p, f64p]
        L.or_prec_destroy.argtypes = [C.c_void_p]
        for name in ("or_cg", "or_bicgstab"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_void_p, f64p, f64p, C.c_int64, C.c_double,
                                         C.c_double, C.c_int32, C.POINTER(Info)]
        L.or_gmres.argtypes = [C.c_void_p, C.c_void_p, f64p, f64p, C.c_int64, C.c_int32,
                               C.c_double, C.c_double, C.c_int32, C.POINTER(Info)]
        L.or_fgmres.argtypes = L.or_gmres.argtypes
        L.or_gcr.argtypes = L.or_gmres.argtypes + [C.POINTER(C.c_int32)]
        L.or_precondition_only.argtypes = [C.c_void_p, C.c_void_p, f64p, f64p, C.c_int64,
                                           C.POINTER(Info)]
        L.or_jacobi.argtypes = [C.c_void_p, C.c_void_p, f64p, f64p, C.c_int64, C.c_double,
                                C.c_double, C.c_int32, C.c_double, C.POINTER(Info)]
        L.or_chebyshev.argtypes = [C.c_void_p, C.c_void_p, f64p, f64p, C.c_int64, C.c_int32,
                                   C.c_double, C.c_double, C.POINTER(Info)]
        _lib = L
    return _lib


class LmaOperator:
    """Coloured LMA apply, y = A x (matrix_vector_kernel over colours)."""

    def __init__(self, ncell_2d, nlayers, ndf_to, ndf_from, map_to, map_from, undf_to,
                 undf_from, stencil, ncells_per_colour, cells_in_colour, transpose=False):
        self._keep = [np.ascontiguousarray(a) for a in
                      (map_to, map_from, stencil, ncells_per_colour, cells_in_colour)]
        mt, mf, st, npc, cic = self._keep
        self.undf_to, self.undf_from = int(undf_to), int(undf_from)
        self.transpose = transpose
        self.h = lib().or_lma_create(ncell_2d, nlayers, ndf_to, ndf_from, mt, mf, undf_to,
                                     undf_from, st, len(npc), npc, cic, cic.shape[0],
                                     1 if transpose else 0)

    def apply(self, x):
        y = np.empty(self.undf_from if self.transpose else self.undf_to)
        lib().or_op_apply(self.h, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def diagonal(self):
        d = np.empty(self.undf_to)
        lib().or_lma_diagonal(self.h, d)
        return d

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_op_destroy(self.h)


class Preconditioner:
    def __init__(self, h, n, keep):
        self.h, self.n, self._keep = h, n, keep

    @classmethod
    def null(cls, n):
        return cls(lib().or_null_prec_create(n), n, [])

    @classmethod
    def diagonal(cls, diag):
        d = np.ascontiguousarray(diag, dtype=np.float64)
        return cls(lib().or_diag_prec_create(d, len(d)), len(d), [d])

    @classmethod
    def cma(cls, ncell_2d, nrow, bandwidth, first_dof, indirection, band, diag, n):
        keep = [np.ascontiguousarray(first_dof, dtype=np.int32),
                np.ascontiguousarray(indirection, dtype=np.int32),
                np.ascontiguousarray(band, dtype=np.float64)]
        dptr = None
        if diag is not None:
            keep.append(np.ascontiguousarray(diag, dtype=np.float64))
            dptr = keep[-1].ctypes.data
        h = lib().or_cma_prec_create(ncell_2d, nrow, bandwidth, keep[0], keep[1], keep[2], dptr, n)
        return cls(h, n, keep)

    def apply(self, x):
        y = np.zeros(self.n)
        lib().or_prec_apply(self.h, np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.or_prec_destroy(self.h)


def solve(kind, op, prec, b, x0=None, r_tol=1e-8, a_tol=1e-16, max_iter=1000, gcrk=10,
          rho_relax=1.0, lmin=0.0, lmax=2.0):
    """Run the oracle's cg / bicgstab / gmres / fgmres / gcr / precondition_only
    / jacobi / chebyshev; returns (x, Info) (for gcr, Info gains iv_final: the
    inner step of the last check)."""
    n = len(b)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    info = Info()
    L = lib()
    if kind == "cg":
        L.or_cg(op.h, prec.h, x, b, n, r_tol, a_tol, max_iter, C.byref(info))
    elif kind == "bicgstab":
        L.or_bicgstab(op.h, prec.h, x, b, n, r_tol, a_tol, max_iter, C.byref(info))
    elif kind == "gmres":
        L.or_gmres(op.h, prec.h, x, b, n, gcrk, r_tol, a_tol, max_iter, C.byref(info))
    elif kind == "fgmres":
        L.or_fgmres(op.h, prec.h, x, b, n, gcrk, r_tol, a_tol, max_iter, C.byref(info))
    elif kind == "gcr":
        ivf = C.c_int32()
        L.or_gcr(op.h, prec.h, x, b, n, gcrk, r_tol, a_tol, max_iter, C.byref(info), C.byref(ivf))
        info.iv_final = ivf.value
    elif kind == "precondition_only":
        L.or_precondition_only(op.h, prec.h, x, b, n, C.byref(info))
    elif kind == "jacobi":
        L.or_jacobi(op.h, prec.h, x, b, n, r_tol, a_tol, max_iter, rho_relax, C.byref(info))
    elif kind == "chebyshev":
        L.or_chebyshev(op.h, prec.h, x, b, n, max_iter, lmin, lmax, C.byref(info))
    else:
        raise ValueError(kind)
    return x, info


def assemble_cma(lma_sub, ncell_2d, nlayers, params):
    """columnwise_op_asm over every column of a (ncell_3d, ndf, ndf) sub-LMA."""
    L = lib()
    bw, nrow, ncol = params["bandwidth"], params["nrow"], params["ncol"]
    band = np.zeros(ncell_2d * bw * nrow)
    cbd = np.ascontiguousarray(params["column_banded_dofmap"], dtype=np.int32)
    ndf = cbd.shape[1]
    lma = np.ascontiguousarray(lma_sub, dtype=np.float64)
    for cell in range(1, ncell_2d + 1):
        L.or_columnwise_op_asm_code(cell, nlayers, ncell_2d, ncell_2d * nlayers, lma, band, nrow,
                                    ncol, bw, params["alpha"], params["beta"], params["gamma_m"],
                                    params["gamma_p"], ndf, cbd, ndf, cbd)
    return band


# ------------------------------------------------------------------ CMA set-up
class Band:
    """A columnwise operator's band, Fortran (bw, nrow, ncell_2d) flattened,
    with its parameters (columnwise_operator_mod.f90:42-114)."""

    def __init__(self, ncell_2d, nrow, ncol, bw, alpha, beta, gamma_m, gamma_p, band=None):
        self.ncell_2d, self.nrow, self.ncol, self.bw = ncell_2d, nrow, ncol, bw
        self.alpha, self.beta, self.gamma_m, self.gamma_p = alpha, beta, gamma_m, gamma_p
        self.band = (np.zeros(bw * nrow * ncell_2d) if band is None
                     else np.ascontiguousarray(band, dtype=np.float64).reshape(-1))

    def args(self):
        return [self.band, self.nrow, self.ncol, self.bw, self.alpha, self.beta, self.gamma_m,
                self.gamma_p]


def _gcd(a, b):
    while b:
        a, b = b, a % b
    return a


def _ceil_div(a, b):
    return -((-a) // b)


def operator_x_plus_ay(x, a, y, ncell_2d, nlayers, ndf1, ndf2):
    """x + a y of two (ncell_2d*nlayers, ndf1, ndf2) Fortran-order operators,
    cell by cell as the reference's kernel loop."""
    nc3 = ncell_2d * nlayers
    out = np.zeros(nc3 * ndf1 * ndf2)
    xa = np.ascontiguousarray(x, dtype=np.float64)
    ya = np.ascontiguousarray(y, dtype=np.float64)
    L = lib()
    for cell in range(1, ncell_2d + 1):
        L.or_operator_x_plus_ay_code(cell, nlayers, nc3, out, xa, float(a), ya, ndf1, ndf2)
    return out


def cma_params(alpha, beta, gamma_m, gamma_p):
    """divide_by_gcd and the bandwidth 1 + ceiling((g_m + g_p)/beta)
    (columnwise_operator_mod.f90:216-247, 316-332)."""
    g = _gcd(alpha, beta)
    if g > 1:
        alpha, beta, gamma_m, gamma_p = alpha // g, beta // g, gamma_m // g, gamma_p // g
    return alpha, beta, gamma_m, gamma_p, 1 + _ceil_div(gamma_m + gamma_p, beta)


def cma_product(A: Band, B: Band) -> Band:
    """columnwise_operator_product (columnwise_operator_mod.f90) + the mul kernel
    over every column: C = A B."""
    al, be, gm, gp, bw = cma_params(A.alpha * B.alpha, A.beta * B.beta,
                                    B.alpha * A.gamma_m + A.beta * B.gamma_m,
                                    B.alpha * A.gamma_p + A.beta * B.gamma_p)
    Cb = Band(A.ncell_2d, A.nrow, B.ncol, bw, al, be, gm, gp)
    for c in range(1, A.ncell_2d + 1):
        lib().or_columnwise_op_mul_code(c, A.ncell_2d, *A.args(), *B.args(), *Cb.args())
    return Cb


def cma_scaledadd(A: Band, B: Band, alpha, beta) -> Band:
    """columnwise_operator_sum + the scaledadd kernel: C = alpha A + beta B."""
    al, be, gm, gp, bw = cma_params(A.alpha, A.beta, max(A.gamma_m, B.gamma_m),
                                    max(A.gamma_p, B.gamma_p))
    Cb = Band(A.ncell_2d, A.nrow, A.ncol, bw, al, be, gm, gp)
    for c in range(1, A.ncell_2d + 1):
        lib().or_columnwise_op_scaledadd_code(c, A.ncell_2d, *A.args(), *B.args(), *Cb.args(),
                                              alpha, beta)
    return Cb


def cma_m2v_lumped_inv(local_stencil, ncell_2d, nlayers, ndf, cbd, nrow, bw, params):
    """asm_m2v_lumped_inv over every column; cbd Fortran (ndf, nlayers) as a
    (nlayers, ndf) C array."""
    Cb = Band(ncell_2d, nrow, nrow, bw, *params)
    cbd = np.ascontiguousarray(cbd, dtype=np.int32)
    st = np.ascontiguousarray(local_stencil, dtype=np.float64).reshape(-1)
    for c in range(1, ncell_2d + 1):
        lib().or_columnwise_op_asm_m2v_lumped_inv_code(c, nlayers, ncell_2d, ncell_2d * nlayers,
                                                       st, Cb.band, nrow, bw, ndf, cbd)
    return Cb


def cma_diag_hmht(Dh, M2h, ncell_2d, nlayers, ndf_w3, ndf_w2h, cbd, nrow, bw, params):
    """asm_diag_hmht over every column (params = alpha, beta, gamma_m, gamma_p)."""
    Cb = Band(ncell_2d, nrow, nrow, bw, *params)
    cbd = np.ascontiguousarray(cbd, dtype=np.int32)
    Dh = np.ascontiguousarray(Dh, dtype=np.float64).reshape(-1)
    M2h = np.ascontiguousarray(M2h, dtype=np.float64).reshape(-1)
    al, be, gm, gp = params
    for c in range(1, ncell_2d + 1):
        lib().or_columnwise_op_asm_diag_hmht_code(c, nlayers, ncell_2d, ncell_2d * nlayers, Dh, M2h,
                                                  Cb.band, nrow, bw, al, be, gm, gp, ndf_w3, cbd,
                                                  ndf_w2h)
    return Cb


# ------------------------------------------------------------------ W2 split / combine
def face_selectors(map_w3_2d, map_w2h, undf_w3_2d, undf_w2h):
    """compute_face_selectors (sci_geometric_constants_mod.x90:203-253): both
    selectors set to 1, then face_selector_code over the cells in order."""
    ew = np.ones(undf_w3_2d, dtype=np.int32)
    ns = np.ones(undf_w3_2d, dtype=np.int32)
    cnt = np.zeros(undf_w2h, dtype=np.int32)
    m3 = np.ascontiguousarray(map_w3_2d, dtype=np.int32)
    mh = np.ascontiguousarray(map_w2h, dtype=np.int32)
    for c in range(m3.shape[0]):
        lib().or_face_selector_code(ew, ns, cnt, m3[c].copy(), mh[c].copy())
    return ew, ns


def split_w2(nlayers, uvw, maps, ew, ns, undf_w2h, undf_w2v):
    """split_w2_field over every cell: returns (uv, w); maps = dict of
    (ncell, ndf) 1-based maps w2, w2h, w2v, w3_2d."""
    uv, w = np.zeros(undf_w2h), np.zeros(undf_w2v)
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    m = {k: np.ascontiguousarray(v, dtype=np.int32) for k, v in maps.items()}
    for c in range(m["w2"].shape[0]):
        lib().or_split_w2_field_code(nlayers, uv, w, uvw, ew, ns, m["w2h"][c].copy(),
                                     m["w2v"][c].copy(), m["w2"][c].copy(), m["w3_2d"][c].copy())
    return uv, w


def combine_w2(nlayers, uv, w, maps, ew, ns, undf_w2):
    uvw = np.zeros(undf_w2)
    uv = np.ascontiguousarray(uv, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    m = {k: np.ascontiguousarray(v, dtype=np.int32) for k, v in maps.items()}
    for c in range(m["w2"].shape[0]):
        lib().or_combine_w2_field_code(nlayers, uvw, uv, w, ew, ns, m["w2"][c].copy(),
                                       m["w2h"][c].copy(), m["w2v"][c].copy(), m["w3_2d"][c].copy())
    return uvw
