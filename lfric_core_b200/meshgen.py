"""Synthetic inputs for the Krylov-solve path (host side, numpy + liblfx_meshgen).

Builds what an LFRic algorithm layer hands to the solver: an extruded
cubed-sphere mesh with column-contiguous dofmaps and its 4-colouring, the
per-cell local matrices (LMA, Fortran layout ``local_stencil(ncell_3d, ndf_to,
ndf_from)``, operator_mod.t90:113-119) and seeded right-hand sides.

Workloads:
  * ``w0_problem``  Q1 nodal W0, A = M + nu*K (mass + diffusion), Jacobi
  * ``w2_problem``  RT0 W2 with W3 divergence, A = M2 + tau*D^T D, with the
    vertical W2V block as a column tridiagonal (CMA) and the W2H rows Jacobi.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "liblfx_meshgen.so"
_lib = None

W0, W2, W3 = 0, 2, 3
NDF = {W0: 8, W2: 6, W3: 1}

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(f"{_LIB_PATH} is not built; run python -m lfric_core_b200.build")
        L = C.CDLL(str(_LIB_PATH))
        L.lfx_mg_cubed_sphere.argtypes = [C.c_int32, i32p, i32p, f64p]
        L.lfx_mg_colour_cubed_sphere.argtypes = [C.c_int32, i32p, i32p]
        L.lfx_mg_test_colours.argtypes = [C.c_int32, i32p, i32p]
        L.lfx_mg_dofmap.argtypes = [C.c_int32, C.c_int32, C.c_int32, i32p, i32p, i32p]
        L.lfx_mg_dofmap.restype = C.c_int64
        L.lfx_mg_geometry.argtypes = [C.c_int32, C.c_int32, f64p, C.c_uint64, C.c_double, f64p]
        L.lfx_mg_lma_w0.argtypes = [C.c_int32, C.c_int32, i32p, f64p, C.c_double, f64p]
        L.lfx_mg_lma_w2.argtypes = [C.c_int32, C.c_int32, i32p, i32p, f64p, C.c_double,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
        L.lfx_mg_uniform.argtypes = [C.c_uint64, C.c_int64, C.c_double, C.c_double, f64p]
        L.lfx_mg_normal.argtypes = [C.c_uint64, C.c_int64, f64p]
        _lib = L
    return _lib


@dataclass
class ColumnMesh:
    """Extruded cubed-sphere mesh: 2D topology, colouring, 3D geometry."""

    n: int
    nlayers: int
    cell_next: np.ndarray      # (ncell, 4) W,S,E,N, 1-based
    verts_on_cell: np.ndarray  # (ncell, 4) SWB,SEB,NEB,NWB, 1-based
    vert_xyz: np.ndarray       # (nvert, 3) unit sphere
    colour_map: np.ndarray     # (ncell,) 1-based colours
    ncolours: int
    xyz3d: np.ndarray = field(repr=False, default=None)

    @property
    def ncell_2d(self) -> int:
        return 6 * self.n * self.n

    @property
    def ncell_3d(self) -> int:
        return self.ncell_2d * self.nlayers

    def colour_lookup(self):
        """(ncells_per_colour, cells_in_colour) as create_colour_map_lookup
        builds them (mesh_colouring_mod.F90): cells_in_colour is the Fortran
        (ncolours, maxc) array, returned as a C-contiguous (maxc, ncolours)
        numpy array so its memory order is the Fortran one."""
        counts = np.bincount(self.colour_map, minlength=self.ncolours + 1)[1:].astype(np.int32)
        maxc = int(counts.max())
        cic = np.zeros((maxc, self.ncolours), dtype=np.int32)
        for col in range(self.ncolours):
            cells = np.nonzero(self.colour_map == col + 1)[0].astype(np.int32) + 1
            cic[: len(cells), col] = cells
        return counts, cic

    def dofmap(self, space: int):
        ndf = NDF[space]
        m = np.zeros((self.ncell_2d, ndf), dtype=np.int32)
        undf = lib().lfx_mg_dofmap(space, self.ncell_2d, self.nlayers, self.cell_next,
                                   self.verts_on_cell, m)
        if undf < 0:
            raise RuntimeError("dofmap generation failed")
        return m, int(undf)


def cubed_sphere(n: int, nlayers: int, seed: int = 0, perturb: float = 0.05) -> ColumnMesh:
    L = lib()
    ncell = 6 * n * n
    nvert = ncell + 2
    cn = np.zeros((ncell, 4), dtype=np.int32)
    vc = np.zeros((ncell, 4), dtype=np.int32)
    xyz = np.zeros((nvert, 3), dtype=np.float64)
    if L.lfx_mg_cubed_sphere(n, cn, vc, xyz) != 0:
        raise RuntimeError("cubed sphere generation failed")
    cm = np.zeros(ncell, dtype=np.int32)
    ncol = L.lfx_mg_colour_cubed_sphere(n, cn, cm)
    if ncol <= 0:
        raise RuntimeError("colouring failed")
    xyz3d = np.zeros((nvert * (nlayers + 1), 3), dtype=np.float64)
    L.lfx_mg_geometry(n, nlayers, xyz, np.uint64(seed), perturb, xyz3d)
    return ColumnMesh(n, nlayers, cn, vc, xyz, cm, int(ncol), xyz3d)


def uniform(seed: int, n: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    lib().lfx_mg_uniform(np.uint64(seed), n, lo, hi, out)
    return out


def normal(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    lib().lfx_mg_normal(np.uint64(seed), n, out)
    return out


@dataclass
class Problem:
    """One linear system A x = b in the reference's native array formats."""

    mesh: ColumnMesh
    space: int
    map: np.ndarray          # (ncell_2d, ndf) 1-based
    undf: int
    lma: np.ndarray          # Fortran local_stencil flattened (ik fastest)
    rhs: np.ndarray
    ndf: int
    extra: dict = field(default_factory=dict)

    @property
    def nlayers(self):
        return self.mesh.nlayers

    @property
    def ncell_2d(self):
        return self.mesh.ncell_2d


def w0_problem(n: int, nlayers: int, seed: int = 1, nu: float = 1.0,
               perturb: float = 0.05, rhs: str = "uniform") -> Problem:
    """Q1 W0 mass + diffusion on C<n> x <nlayers>; b ~ U[-1,1] (or N(0,1))."""
    mesh = cubed_sphere(n, nlayers, seed=seed, perturb=perturb)
    m, undf = mesh.dofmap(W0)
    lma = np.zeros(mesh.ncell_3d * 64, dtype=np.float64)
    lib().lfx_mg_lma_w0(mesh.ncell_2d, nlayers, mesh.verts_on_cell, mesh.xyz3d, nu, lma)
    b = uniform(seed + 101, undf) if rhs == "uniform" else normal(seed + 101, undf)
    return Problem(mesh, W0, m, undf, lma, b, 8)


W2V_DFS = (4, 5)   # bottom, top faces (0-based local W2 dofs)
W2H_DFS = (0, 1, 2, 3)


def w2_problem(n: int, nlayers: int, seed: int = 2, tau: float = 0.1,
               perturb: float = 0.05, keep_parts: bool = False) -> Problem:
    """RT0 W2 Helmholtz-type operator A = M2 + tau D^T D on C<n> x <nlayers>;
    b ~ N(0,1). extra: W2V column data for the CMA preconditioner."""
    mesh = cubed_sphere(n, nlayers, seed=seed, perturb=perturb)
    m, undf = mesh.dofmap(W2)
    nc3 = mesh.ncell_3d
    a = np.zeros(nc3 * 36, dtype=np.float64)
    m2 = np.zeros(nc3 * 36, dtype=np.float64) if keep_parts else None
    dv = np.zeros(nc3 * 6, dtype=np.float64) if keep_parts else None
    ptr = (lambda x: None if x is None else x.ctypes.data)
    lib().lfx_mg_lma_w2(mesh.ncell_2d, nlayers, mesh.cell_next, mesh.verts_on_cell,
                        mesh.xyz3d, tau, ptr(m2), ptr(dv), a.ctypes.data)
    b = normal(seed + 202, undf)
    extra = {"tau": tau}
    if keep_parts:
        extra["m2"] = m2
        extra["div"] = dv
        m3, undf3 = mesh.dofmap(W3)
        extra["map_w3"] = m3
        extra["undf_w3"] = undf3
    return Problem(mesh, W2, m, undf, a, b, 6, extra)


def lma_block(lma: np.ndarray, ncell_3d: int, ndf: int, dfs) -> np.ndarray:
    """Sub-block local_stencil(:, dfs, dfs) of a Fortran (ncell_3d, ndf, ndf) LMA."""
    full = lma.reshape(ndf, ndf, ncell_3d)  # [df2][df1][ik]
    sub = full[np.ix_(list(dfs), list(dfs))]
    return np.ascontiguousarray(sub).reshape(-1)


def w2v_cma_params(nlayers: int):
    """Banded-matrix parameters of the W2V -> W2V columnwise operator
    (columnwise_operator_mod.f90:170-198, 350-396): ndof_face_v = 1, no
    interior dofs, so alpha = beta = 1, gamma_m = gamma_p = 1, bandwidth 3,
    nrow = ncol = nlayers + 1, identity indirection."""
    nrow = nlayers + 1
    cbd = np.zeros((nlayers, 2), dtype=np.int32)  # Fortran (ndf=2, nlayers)
    for k in range(1, nlayers + 1):
        cbd[k - 1, 0] = k
        cbd[k - 1, 1] = k + 1
    ind = np.arange(1, nrow + 1, dtype=np.int32)
    return dict(alpha=1, beta=1, gamma_m=1, gamma_p=1, bandwidth=3, nrow=nrow, ncol=nrow,
                column_banded_dofmap=cbd, indirection=ind)


def w2_subspace_maps(map_w2: np.ndarray, nlayers: int):
    """Dofmaps of the W2h and W2v parts and of W3-2D for a lowest-order W2
    dofmap (faces W S E N B T), column-contiguous as dofmap_setup numbers
    them: each horizontal face column keeps its nlayers dofs, each vertical
    face column its nlayers + 1, in the order of their W2 numbering. Returns
    (map_w2h, undf_w2h, map_w2v, undf_w2v, map_w3_2d, undf_w3_2d)."""
    m = np.asarray(map_w2)
    hb = np.unique(m[:, :4])
    hidx = {int(b): i for i, b in enumerate(hb)}
    map_h = np.vectorize(lambda b: hidx[int(b)] * nlayers + 1)(m[:, :4]).astype(np.int32)
    vb = np.unique(m[:, 4])
    vidx = {int(b): i for i, b in enumerate(vb)}
    bot = np.array([vidx[int(b)] * (nlayers + 1) + 1 for b in m[:, 4]], dtype=np.int32)
    map_v = np.stack([bot, bot + 1], axis=1)
    map_3 = np.arange(1, len(m) + 1, dtype=np.int32).reshape(-1, 1)
    return map_h, len(hb) * nlayers, map_v, len(vb) * (nlayers + 1), map_3, len(m)
