"""Many right-hand sides at once (lfx_mrhs): the tensor-core apply against the
oracle's FP64 apply, and the refined multi-RHS solve against the oracle's CG.

Bounds: a TF32 (BF16) product rounds both factors to 11 (8) significant bits,
u = 2^-11 (2^-8), and accumulates in FP32, so every entry of y = A x lies
within 4 u (|A| |x|) of the exact FP64 product. The refined solve must reach
the FP64 tolerance on the true residual, checked here with the oracle."""
import numpy as np
import pytest
import torch

from lfric_core_b200 import lfx
from lfric_core_b200 import meshgen as mg
from lfric_core_b200 import workloads as wl
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

U = {lfx.MRHS_TF32: 2.0 ** -11, lfx.MRHS_BF16: 2.0 ** -8}
TF32, BF16 = lfx.MRHS_TF32, lfx.MRHS_BF16


def o_lma(p, lma=None):
    npc, cic = p.mesh.colour_lookup()
    return orc.LmaOperator(p.ncell_2d, p.nlayers, 8, 8, p.map, p.map, p.undf, p.undf,
                           p.lma if lma is None else lma, npc, cic)


def mrhs_apply(ctx, M, X):
    x = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    y = torch.full_like(x, float("nan"))
    torch.cuda.synchronize()
    M.apply(x.data_ptr(), y.data_ptr())
    ctx.synchronize()
    return y.cpu().numpy()


@pytest.mark.parametrize("n,nl,kind,nrhs,patch", [
    (6, 7, TF32, 64, 0), (6, 7, BF16, 64, 0), (5, 10, TF32, 32, 4), (5, 10, BF16, 16, 64),
    (8, 4, TF32, 64, 1), (4, 13, BF16, 32, 7)])
def test_mrhs_apply_within_rounding_bound(ctx, n, nl, kind, nrhs, patch):
    p = mg.w0_problem(n, nl, seed=7 + n)
    s = wl.device_w0(ctx, p)
    M = lfx.MultiRhsOperator(s.op, kind, nrhs, patch)
    info = M.info()
    assert info["cell_levels"] >= p.mesh.ncell_3d
    rng = np.random.default_rng(100 * n + nl)
    X = rng.standard_normal((p.undf, nrhs)).astype(np.float32)
    Y = mrhs_apply(ctx, M, X)
    assert np.all(np.isfinite(Y))
    # deterministic: the same bits on a second apply
    assert np.array_equal(Y, mrhs_apply(ctx, M, X))
    o, oa = o_lma(p), o_lma(p, np.abs(p.lma))
    for r in range(nrhs):
        x = X[:, r].astype(np.float64)
        err = np.abs(Y[:, r] - o.apply(x))
        bound = 4 * U[kind] * oa.apply(np.abs(x))
        assert np.all(err <= bound), (r, float(np.max(err / np.maximum(bound, 1e-300))))


def test_mrhs_patch_sizes_agree_within_bound(ctx):
    p = mg.w0_problem(7, 9, seed=11)
    s = wl.device_w0(ctx, p)
    X = np.random.default_rng(5).standard_normal((p.undf, 32)).astype(np.float32)
    Ys = [mrhs_apply(ctx, lfx.MultiRhsOperator(s.op, TF32, 32, pp), X) for pp in (1, 9, 40)]
    oa = o_lma(p, np.abs(p.lma))
    for r in range(32):
        ya = oa.apply(np.abs(X[:, r]).astype(np.float64))
        for Y in Ys[1:]:
            assert np.all(np.abs(Y[:, r] - Ys[0][:, r]) <= 8 * U[TF32] * ya)


@pytest.mark.parametrize("kind", [TF32, BF16])
def test_mrhs_autotune_keeps_results_within_bound(ctx, kind):
    p = mg.w0_problem(6, 11, seed=21)
    s = wl.device_w0(ctx, p)
    M = lfx.MultiRhsOperator(s.op, kind, 64)
    X = np.random.default_rng(8).standard_normal((p.undf, 64)).astype(np.float32)
    before = mrhs_apply(ctx, M, X)
    t = M.autotune(reps=3)
    assert t["levels_per_block"] in (2, 4, 8) and t["us"] > 0
    after = mrhs_apply(ctx, M, X)
    oa = o_lma(p, np.abs(p.lma))
    for r in range(0, 64, 7):
        ya = oa.apply(np.abs(X[:, r]).astype(np.float64))
        assert np.all(np.abs(after[:, r] - before[:, r]) <= 8 * U[kind] * ya)


def test_mrhs_rejects_non_nodal_operator(ctx):
    p = mg.w2_problem(4, 3)
    s = wl.device_w2(ctx, p)
    with pytest.raises(lfx.LfxError) as e:
        lfx.MultiRhsOperator(s.op, TF32, 64)
    assert e.value.status == 8
    s0 = wl.device_w0(ctx, mg.w0_problem(4, 3))
    with pytest.raises(lfx.LfxError):
        lfx.MultiRhsOperator(s0.op, TF32, 48)


@pytest.mark.parametrize("kind", [TF32, BF16])
def test_mrhs_refined_solve_reaches_fp64_tolerance(ctx, kind):
    p = mg.w0_problem(8, 6, seed=3)
    s = wl.device_w0(ctx, p)
    nrhs = 16
    M = lfx.MultiRhsOperator(s.op, kind, nrhs)
    B = np.stack([mg.normal(900 + r, p.undf) for r in range(nrhs)])
    b = torch.from_numpy(B).cuda()
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    info = M.solve(s.op, s.diag, b.data_ptr(), x.data_ptr(), p.undf, r_tol=1e-8, inner_tol=1e-2)
    ctx.synchronize()
    X = x.cpu().numpy()
    o = o_lma(p)
    L = orc.lib()
    od = orc.Preconditioner.diagonal(o.diagonal())
    for r in range(nrhs):
        assert info[r].converged and info[r].status == 0
        assert info[r].outer_iterations >= 2
        res = B[r] - o.apply(X[r])
        # the device residual is the oracle's apply and reduction order: same norm
        assert np.sqrt(L.or_sumsq(res, len(res))) == pytest.approx(info[r].final_norm, rel=1e-12)
        rel = np.linalg.norm(res) / np.linalg.norm(B[r])
        assert rel <= 1e-8
    for r in (0, 7):
        xo, oi = orc.solve("cg", o, od, B[r], r_tol=1e-10, max_iter=5000)
        assert np.linalg.norm(X[r] - xo) <= 1e-5 * np.linalg.norm(xo)


def test_mrhs_solve_nonzero_initial_guess_and_converged_rhs(ctx):
    p = mg.w0_problem(6, 5, seed=4)
    s = wl.device_w0(ctx, p)
    nrhs = 16
    M = lfx.MultiRhsOperator(s.op, TF32, nrhs)
    B = np.stack([mg.normal(50 + r, p.undf) for r in range(nrhs)])
    B[3] = 0.0  # zero right-hand side with zero guess: converged at once
    X0 = np.zeros_like(B)
    X0[5] = mg.normal(7, p.undf)
    b, x = torch.from_numpy(B).cuda(), torch.from_numpy(X0).cuda()
    torch.cuda.synchronize()
    info = M.solve(s.op, s.diag, b.data_ptr(), x.data_ptr(), p.undf, r_tol=1e-9)
    ctx.synchronize()
    X = x.cpu().numpy()
    assert info[3].converged and info[3].outer_iterations == 0 and np.all(X[3] == 0.0)
    o = o_lma(p)
    for r in range(nrhs):
        assert info[r].converged
        if r == 3:
            continue
        r0 = np.linalg.norm(B[r] - o.apply(X0[r]))
        assert np.linalg.norm(B[r] - o.apply(X[r])) <= 1e-9 * r0 * (1 + 1e-9)


@pytest.mark.parametrize("kind", [TF32, BF16])
def test_mrhs_block_cg_reaches_fp64_tolerance(ctx, kind):
    """Block CG over the 64 right-hand sides: every right-hand side reaches
    the FP64 tolerance on the oracle's residual, in fewer inner iterations
    than CG run on each right-hand side alone, and its solutions agree with
    the oracle's FP64 CG."""
    p = mg.w0_problem(8, 6, seed=3)
    s = wl.device_w0(ctx, p)
    nrhs = 64
    M = lfx.MultiRhsOperator(s.op, kind, nrhs)
    B = np.stack([mg.normal(900 + r, p.undf) for r in range(nrhs)])
    B[5] = 0.0  # a zero right-hand side: converged at once, left out of the block
    b = torch.from_numpy(B).cuda()
    out = {}
    for method in (lfx.MRHS_PER_RHS_CG, lfx.MRHS_BLOCK_CG):
        x = torch.zeros_like(b)
        torch.cuda.synchronize()
        info = M.solve(s.op, s.diag, b.data_ptr(), x.data_ptr(), p.undf, r_tol=1e-8,
                       inner_tol=1e-3, method=method)
        ctx.synchronize()
        out[method] = (x.cpu().numpy(), info)
    X, info = out[lfx.MRHS_BLOCK_CG]
    o = o_lma(p)
    od = orc.Preconditioner.diagonal(o.diagonal())
    assert info[5].converged and np.all(X[5] == 0.0)
    for r in range(nrhs):
        assert info[r].converged and info[r].status == 0, r
        if r == 5:
            continue
        rel = np.linalg.norm(B[r] - o.apply(X[r])) / np.linalg.norm(B[r])
        assert rel <= 1e-8, (r, rel)
    for r in (0, 33):
        xo, _ = orc.solve("cg", o, od, B[r], r_tol=1e-10, max_iter=5000)
        assert np.linalg.norm(X[r] - xo) <= 1e-5 * np.linalg.norm(xo)
    per = max(i.inner_iterations for i in out[lfx.MRHS_PER_RHS_CG][1])
    blk = max(i.inner_iterations for i in info)
    assert blk < per, (blk, per)


@pytest.mark.parametrize("nv", [1, 2])
def test_block_cg_gram_products_match_fp64(ctx, nv):
    """The block CG's Gram products U^T [V0 V1] of n x 64 blocks: on the
    tcgen05 tensor cores (FP32 split into TF32 hi + lo, three MMAs per step,
    FP32 accumulation in tensor memory) and on the FP32 cores, each within
    5e-5 of |U|^T |V| of the FP64 product entry by entry (n = 72 618 rows,
    not a multiple of the 32-row chunk), and run to run the same bits."""
    p = mg.w0_problem(24, 20, seed=1)
    s = wl.device_w0(ctx, p)
    M = lfx.MultiRhsOperator(s.op, TF32, 64)
    n = p.undf
    g = torch.Generator(device="cpu").manual_seed(77)
    U = torch.randn(n, 64, generator=g).cuda()
    V = [torch.randn(n, 64, generator=g).cuda() for _ in range(nv)]
    Vc = torch.cat(V, dim=1).double()
    want = (U.double().T @ Vc).cpu().numpy()
    bound = 5e-5 * (U.double().abs().T @ Vc.abs()).cpu().numpy()
    out = torch.empty(nv, 64, 64, dtype=torch.float64, device="cuda")
    for tensor in (True, False):
        got = []
        for _ in range(2):
            out.fill_(float("nan"))
            torch.cuda.synchronize()
            M.gram(U.data_ptr(), V[0].data_ptr(), V[-1].data_ptr() if nv == 2 else 0, nv, tensor,
                   out.data_ptr())
            got.append(out.cpu().numpy().copy())
        assert np.array_equal(got[0], got[1]), tensor
        G = np.concatenate(list(got[0]), axis=1)  # 64 x 64 nv
        assert np.all(np.abs(G - want) <= bound), (tensor, float(np.max(np.abs(G - want) / bound)))
