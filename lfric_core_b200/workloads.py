"""Device set-up of the two operator families of the solve path.

``device_w0``  Q1 W0 mass + diffusion with the Jacobi preconditioner
               (the mass_matrix_solver_alg path: sci_mass_matrix_solver_alg_mod.x90:151-311)
``device_w2``  RT0 W2 Helmholtz-type operator M2 + tau D^T D with the
               column-tridiagonal preconditioner on the vertical (W2V) faces,
               assembled on the device by columnwise_op_asm from the operator's
               W2V-W2V block, and Jacobi on the horizontal (W2H) faces.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import lfx
from . import meshgen as mg


@dataclass
class DeviceSystem:
    ctx: lfx.Context
    problem: mg.Problem
    op: lfx.LmaOperator
    prec: object
    diag: lfx.FieldVector
    precision: int
    cma: object = None
    op64: lfx.LmaOperator = None

    def vector(self, data=None):
        v = lfx.FieldVector(self.ctx, [self.problem.undf], self.precision)
        if data is not None:
            v.import_field(data)
        else:
            v.set_scalar(0.0)
        return v


def _lma(ctx, p: mg.Problem, precision):
    npc, cic = p.mesh.colour_lookup()
    return lfx.LmaOperator(ctx, p.ncell_2d, p.nlayers, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf,
                           p.lma, npc, cic, precision=precision)


def device_w0(ctx, p: mg.Problem, precision=lfx.R64) -> DeviceSystem:
    op = _lma(ctx, p, precision)
    diag = lfx.FieldVector(ctx, [p.undf], precision)
    op.diagonal(diag)
    prec = lfx.DiagonalPreconditioner(ctx, diag)
    return DeviceSystem(ctx, p, op, prec, diag, precision)


def w2_cma(op64: lfx.LmaOperator, p: mg.Problem):
    prm = mg.w2v_cma_params(p.nlayers)
    dfs = [d + 1 for d in mg.W2V_DFS]
    return lfx.ColumnwiseOperator.assemble(op64, dfs, prm["column_banded_dofmap"], prm,
                                           np.ascontiguousarray(p.map[:, mg.W2V_DFS[0]]))


def device_w2(ctx, p: mg.Problem, precision=lfx.R64, op64=None, cma=None, diag64=None) -> DeviceSystem:
    """FP64 operator (always built: it owns the CMA assembly) plus, for
    precision 32, an FP32 copy of the operator and an FP32 preconditioner
    whose column factorisation was done in FP64."""
    op64 = op64 or _lma(ctx, p, lfx.R64)
    cma = cma or w2_cma(op64, p)
    if diag64 is None:
        diag64 = lfx.FieldVector(ctx, [p.undf], lfx.R64)
        op64.diagonal(diag64)
    if precision == lfx.R64:
        prec = lfx.ColumnwisePreconditioner(ctx, cma, diag64, lfx.R64)
        return DeviceSystem(ctx, p, op64, prec, diag64, lfx.R64, cma, op64)
    op32 = op64.like(p.lma, lfx.R32)
    prec32 = lfx.ColumnwisePreconditioner(ctx, cma, diag64, lfx.R32)
    return DeviceSystem(ctx, p, op32, prec32, diag64, lfx.R32, cma, op64)


@dataclass
class BatchSystem:
    """One independent SPD system for lfx.Batch, assembled on the device:
    FP64 and FP32 copies of the operator, the FP32 preconditioner the batch
    iterates with and the FP64 one for plain FP64 solves, and a right-hand side."""

    space: int
    n: int
    nlayers: int
    undf: int
    entities: int
    columns: int
    ops: dict
    prec32: object
    prec64: object
    b: lfx.FieldVector
    keep: tuple = ()

    def cg64(self, r_tol, max_iter=20000):
        return lfx.ConjugateGradient(self.ops[lfx.R64], self.prec64, r_tol, 0.0, max_iter)


def batch_system(ctx, n, nlayers, seed, space, rhs_seed=None) -> BatchSystem:
    mesh = mg.cubed_sphere(n, nlayers, seed=seed)
    ncell = 6 * n * n
    rhs_seed = seed + 1000 if rhs_seed is None else rhs_seed
    if space == mg.W0:
        ops, m, undf = lfx.fem_operators(ctx, mesh, mg.W0, 1.0)
        d32 = lfx.FieldVector(ctx, [undf], lfx.R32)
        ops[lfx.R32].diagonal(d32)
        d64 = lfx.FieldVector(ctx, [undf], lfx.R64)
        ops[lfx.R64].diagonal(d64)
        p32 = lfx.DiagonalPreconditioner(ctx, d32)
        p64 = lfx.DiagonalPreconditioner(ctx, d64)
        b = lfx.FieldVector.from_array(ctx, mg.uniform(rhs_seed, undf))
        return BatchSystem(space, n, nlayers, undf, ncell + 2, 0, ops, p32, p64, b, (d32, d64))
    ops, m, undf = lfx.fem_operators(ctx, mesh, mg.W2, 0.1)
    prm = mg.w2v_cma_params(nlayers)
    cma = lfx.ColumnwiseOperator.assemble(ops[lfx.R64], [d + 1 for d in mg.W2V_DFS],
                                          prm["column_banded_dofmap"], prm,
                                          np.ascontiguousarray(m[:, mg.W2V_DFS[0]]))
    d64 = lfx.FieldVector(ctx, [undf], lfx.R64)
    ops[lfx.R64].diagonal(d64)
    p64 = lfx.ColumnwisePreconditioner(ctx, cma, d64, lfx.R64)
    p32 = lfx.ColumnwisePreconditioner(ctx, cma, d64, lfx.R32)
    b = lfx.FieldVector.from_array(ctx, mg.normal(rhs_seed, undf))
    return BatchSystem(space, n, nlayers, undf, 3 * ncell, ncell, ops, p32, p64, b, (cma, d64))


def config3_specs(count=256, seed=3):
    """Uneven batch: N ~ U{12..48}, nlayers ~ U{10..70}, tol ~ logU[1e-10, 1e-6]."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(12, 49, count)
    ls = rng.integers(10, 71, count)
    tols = 10.0 ** rng.uniform(-10, -6, count)
    return [(int(n), int(l), float(t), 100 + i) for i, (n, l, t) in enumerate(zip(ns, ls, tols))]


def config4_stream(nreq=200, rate=2000.0, pool=12, seed=4):
    """Poisson arrivals (rate per second) of W2 Helmholtz solves drawn from a
    pool of operators with N ~ U{12..96}, nlayers ~ U{20..70}; tol ~ logU[1e-10, 1e-6]."""
    rng = np.random.default_rng(seed)
    shapes = [(int(n), int(l)) for n, l in zip(rng.integers(12, 97, pool), rng.integers(20, 71, pool))]
    t = np.cumsum(rng.exponential(1.0 / rate, nreq))
    which = rng.integers(0, pool, nreq)
    tols = 10.0 ** rng.uniform(-10, -6, nreq)
    return shapes, [(float(a), int(w), float(tl)) for a, w, tl in zip(t, which, tols)]


def refined_gmres(sys32: DeviceSystem, gcrk=10, inner_rtol=1e-4, inner_cycles=50, r_tol=1e-8,
                  max_outer=20):
    """FP32 GMRES(gcrk) inner solve wrapped in FP64 iterative refinement."""
    inner = lfx.GMRES(sys32.op, sys32.prec, gcrk, inner_rtol, 0.0, inner_cycles)
    outer = lfx.RefinedSolver(sys32.op64, inner, inner_rtol, r_tol, 0.0, max_outer)
    outer._inner = inner
    return outer
