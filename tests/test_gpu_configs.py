"""The reduced-precision configurations at their own sizes, checked against
the oracle (the CPU FP64 restatement of the reference), not against the
device itself.

  * many right-hand sides (C48 x 30 W0, 64 N(0,1) right-hand sides, TF32 and
    BF16 tensor-core applies inside FP64 refinement)
  * a batch shaped like the 256 uneven solves (C12-C48, 10-70 levels,
    tolerances 1e-10..1e-6, W0, one persistent kernel per replay)
  * W2 Helmholtz requests of mixed size through the same batch engine with
    the column preconditioner

Every result must reach its tolerance on the true residual computed with the
oracle's FP64 apply. Its solution is then compared with the oracle's own FP64
CG solution at the same tolerance: two solutions whose residuals are both
within tol of ||b|| differ by at most 2 cond(A) tol relatively, and cond(A)
stays under 5e3 for these meshes (the diffusion term scales as h, the mass
term as h^3, h >= 1/48 on the unit shell), so the stated bound is
ERR_FACTOR * tol with ERR_FACTOR = 1e4.
"""
import numpy as np
import pytest
import torch

from lfric_core_b200 import lfx
from lfric_core_b200 import meshgen as mg
from lfric_core_b200 import workloads as wl
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

ERR_FACTOR = 1e4


def o_lma(p):
    npc, cic = p.mesh.colour_lookup()
    return orc.LmaOperator(p.ncell_2d, p.nlayers, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf,
                           p.lma, npc, cic)


def o_w2_prec(p, op):
    prm = mg.w2v_cma_params(p.nlayers)
    band = orc.assemble_cma(mg.lma_block(p.lma, p.mesh.ncell_3d, 6, mg.W2V_DFS), p.ncell_2d,
                            p.nlayers, prm)
    return orc.Preconditioner.cma(p.ncell_2d, prm["nrow"], 3, p.map[:, 4], prm["indirection"],
                                  band, op.diagonal(), p.undf)


def rel_err(x, xo):
    return float(np.linalg.norm(x - xo) / np.linalg.norm(xo))


@pytest.mark.parametrize("method", [lfx.MRHS_PER_RHS_CG, lfx.MRHS_BLOCK_CG])
@pytest.mark.parametrize("kind", [lfx.MRHS_TF32, lfx.MRHS_BF16])
def test_multi_rhs_c48x30_64rhs_against_oracle(ctx, kind, method):
    p = mg.w0_problem(48, 30, seed=1, rhs="normal")
    s = wl.device_w0(ctx, p)
    nrhs, rtol = 64, 1e-8
    B = np.stack([mg.normal(1000 + r, p.undf) for r in range(nrhs)])
    b = torch.from_numpy(B).cuda()
    x = torch.zeros_like(b)
    M = lfx.MultiRhsOperator(s.op, kind, nrhs)
    torch.cuda.synchronize()
    info = M.solve(s.op, s.diag, b.data_ptr(), x.data_ptr(), p.undf, r_tol=rtol, method=method)
    ctx.synchronize()
    X = x.cpu().numpy()
    o = o_lma(p)
    for r in range(nrhs):
        assert info[r].converged and info[r].status == 0, r
        rel = np.linalg.norm(B[r] - o.apply(X[r])) / np.linalg.norm(B[r])
        assert rel <= rtol * 1.0001, (r, rel)
    od = orc.Preconditioner.diagonal(o.diagonal())
    for r in (0, 21, 42, 63):
        xo, oi = orc.solve("cg", o, od, B[r], r_tol=rtol, a_tol=0.0, max_iter=20000)
        assert oi.converged
        assert rel_err(X[r], xo) <= ERR_FACTOR * rtol, (r, rel_err(X[r], xo))


# (N, levels, tolerance, seed): the corners of the uneven batch's ranges,
# points between them, and the level counts at a segment boundary (30, 31,
# 32 levels: one or two 31-row segments per cell column)
CONFIG3_SUBSET = [(12, 10, 1e-6, 101), (48, 70, 1e-10, 102), (20, 33, 1e-8, 103),
                  (36, 12, 1e-9, 104), (16, 64, 1e-7, 105), (30, 47, 1e-10, 106),
                  (44, 25, 1e-6, 107), (25, 58, 1e-9, 108), (47, 31, 1e-8, 109),
                  (17, 30, 1e-9, 110), (13, 32, 1e-7, 111), (40, 62, 1e-8, 112)]


def test_batch_uneven_w0_subset_against_oracle(ctx):
    systems = [wl.batch_system(ctx, n, nl, sd, mg.W0) for n, nl, _, sd in CONFIG3_SUBSET]
    B = lfx.Batch(ctx, 8, len(systems), reserve_bytes=1 << 30, iters=8)
    xs = []
    for s, (_, _, tol, _) in zip(systems, CONFIG3_SUBSET):
        x = lfx.FieldVector(ctx, [s.undf])
        x.set_scalar(0.0)
        xs.append((B.admit(s.ops[lfx.R64], s.ops[lfx.R32], s.prec32, s.b, x, tol, 20000), x))
    B.autotune(iters=2)
    for _ in range(5000):
        if B.step() == len(systems):
            break
    for (slot, x), s, (n, nl, tol, sd) in zip(xs, systems, CONFIG3_SUBSET):
        ph, _, info = B.slot(slot)
        assert ph == 3 and info.status == 0, (n, nl, info.as_dict())
        p = mg.w0_problem(n, nl, seed=sd)
        o = o_lma(p)
        b = s.b.export_field()
        xv = x.export_field()
        rel = np.linalg.norm(b - o.apply(xv)) / np.linalg.norm(b)
        assert rel <= tol * 1.0001, (n, nl, rel, tol)
        xo, oi = orc.solve("cg", o, orc.Preconditioner.diagonal(o.diagonal()), b, r_tol=tol,
                           a_tol=0.0, max_iter=20000)
        assert oi.converged
        assert rel_err(xv, xo) <= ERR_FACTOR * tol, (n, nl, rel_err(xv, xo))


CONFIG4_SUBSET = [(12, 20, 1e-6, 501), (24, 45, 1e-10, 502), (32, 70, 1e-8, 503),
                  (21, 31, 1e-9, 504)]


def test_batch_w2_requests_against_oracle(ctx):
    systems = [wl.batch_system(ctx, n, nl, sd, mg.W2) for n, nl, _, sd in CONFIG4_SUBSET]
    B = lfx.Batch(ctx, 6, len(systems), reserve_bytes=1 << 30, iters=8)
    xs = []
    for s, (_, _, tol, _) in zip(systems, CONFIG4_SUBSET):
        x = lfx.FieldVector(ctx, [s.undf])
        x.set_scalar(0.0)
        xs.append((B.admit(s.ops[lfx.R64], s.ops[lfx.R32], s.prec32, s.b, x, tol, 20000), x))
    for _ in range(5000):
        if B.step() == len(systems):
            break
    for (slot, x), s, (n, nl, tol, sd) in zip(xs, systems, CONFIG4_SUBSET):
        ph, _, info = B.slot(slot)
        assert ph == 3 and info.status == 0, (n, nl, info.as_dict())
        p = mg.w2_problem(n, nl, seed=sd)
        o = o_lma(p)
        b = s.b.export_field()
        xv = x.export_field()
        rel = np.linalg.norm(b - o.apply(xv)) / np.linalg.norm(b)
        assert rel <= tol * 1.0001, (n, nl, rel, tol)
        xo, oi = orc.solve("cg", o, o_w2_prec(p, o), b, r_tol=tol, a_tol=0.0, max_iter=20000)
        assert oi.converged
        assert rel_err(xv, xo) <= ERR_FACTOR * tol, (n, nl, rel_err(xv, xo))
