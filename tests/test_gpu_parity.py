"""GPU parity of the CUDA path (through the C ABI) against the oracle.

FP64 results are compared bit for bit: the device reproduces the reference's
coloured summation order in the LMA apply and shares the oracle's fixed
reduction order, and both compute every a + b*c as one fma. FP32 results are
compared with stated tolerances."""
import numpy as np
import pytest

from lfric_core_b200 import lfx
from lfric_core_b200 import meshgen as mg
from lfric_core_b200 import workloads as wl
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def o_lma(p):
    npc, cic = p.mesh.colour_lookup()
    return orc.LmaOperator(p.ncell_2d, p.nlayers, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf, p.lma,
                           npc, cic)


def o_w2_prec(p, op):
    prm = mg.w2v_cma_params(p.nlayers)
    band = orc.assemble_cma(mg.lma_block(p.lma, p.mesh.ncell_3d, 6, mg.W2V_DFS), p.ncell_2d,
                            p.nlayers, prm)
    diag = op.diagonal()
    return orc.Preconditioner.cma(p.ncell_2d, prm["nrow"], 3, p.map[:, 4], prm["indirection"],
                                  band, diag, p.undf), band


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


# ------------------------------------------------------------------ vectors
@pytest.mark.parametrize("n", [1, 2047, 2048, 100003])
def test_vector_ops_bitwise(ctx, n):
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    L = orc.lib()
    X, Y = lfx.FieldVector.from_array(ctx, x), lfx.FieldVector.from_array(ctx, y)
    assert X.dot(Y) == L.or_dot(x, y, n)
    assert X.norm() == np.sqrt(L.or_sumsq(x, n))
    Z = X.duplicate()
    Z.copy(X)
    Z.axpy(0.37, Y)
    z = x.copy()
    L.or_inc_x_plus_by(z, 0.37, y, n)
    assert same(Z.export_field(), z)
    Z.aypx(-1.25, Y)
    L.or_inc_ax_plus_y(-1.25, z, y, n)
    assert same(Z.export_field(), z)
    Z.axpby(2.5, X, -0.5, Y)
    L.or_ax_plus_by(z, 2.5, x, -0.5, y, n)
    assert same(Z.export_field(), z)
    Z.scale(1.0 / 3.0)
    L.or_inc_a_times_x(1.0 / 3.0, z, n)
    assert same(Z.export_field(), z)
    Z.set_scalar(4.0)
    assert np.all(Z.export_field() == 4.0)
    assert Z.vector_size() == 1


def test_fp32_vector_semantics(ctx):
    n = 50000
    rng = np.random.default_rng(2)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    X, Y = lfx.FieldVector.from_array(ctx, x, lfx.R32), lfx.FieldVector.from_array(ctx, y, lfx.R32)
    x32, y32 = x.astype(np.float32), y.astype(np.float32)
    np.testing.assert_allclose(X.dot(Y), float(x32.astype(np.float64) @ y32.astype(np.float64)),
                               rtol=1e-13)
    X.axpy(0.5, Y)
    np.testing.assert_allclose(X.export_field(), (x32 + np.float32(0.5) * y32).astype(np.float64),
                               rtol=1e-6)


def test_async_field_transfers(ctx):
    """Asynchronous FP64 imports/exports on a caller stream (torch side
    stream, ordered with events) give back exactly the data; FP32 fields are
    refused."""
    import torch
    n = 100003
    src = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    dst = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    src[:] = mg.normal(5, n)
    v = lfx.FieldVector(ctx, [n])
    cs = torch.cuda.Stream()
    v.import_field_async(src, cs.cuda_stream)
    done = torch.cuda.Event()
    done.record(cs)
    main = torch.cuda.ExternalStream(ctx.stream)
    main.wait_event(done)
    v.scale(2.0)                                   # on the context's stream
    back = torch.cuda.Event()
    back.record(main)
    cs.wait_event(back)
    v.export_field_async(dst, cs.cuda_stream)
    cs.synchronize()
    assert same(dst, 2.0 * src)
    v.import_field_async(src)                      # the context's stream
    v.export_field_async(dst)
    ctx.synchronize()
    assert same(dst, src)
    w = lfx.FieldVector(ctx, [n], lfx.R32)
    with pytest.raises(lfx.LfxError):
        w.import_field_async(src)


def test_multifield_vector(ctx):
    undf = [1000, 3001]
    rng = np.random.default_rng(4)
    v = lfx.FieldVector(ctx, undf)
    w = v.duplicate()
    a, b = [rng.standard_normal(u) for u in undf], [rng.standard_normal(u) for u in undf]
    for i in range(2):
        v.import_field(a[i], i + 1)
        w.import_field(b[i], i + 1)
    L = orc.lib()
    want = 0.0 + L.or_dot(a[0], b[0], undf[0])
    want = want + L.or_dot(a[1], b[1], undf[1])
    assert v.dot(w) == want
    assert v.vector_size() == 2
    assert v.field_norm(2) == np.sqrt(L.or_sumsq(a[1], undf[1]))
    with pytest.raises(lfx.LfxError):
        v.import_field(a[0], 3)


# ------------------------------------------------------------------ operators
@pytest.mark.parametrize("n,nl", [(4, 3), (12, 7), (24, 20)])
def test_lma_apply_w0_bitwise(ctx, n, nl):
    p = mg.w0_problem(n, nl, seed=n)
    sysd = wl.device_w0(ctx, p)
    op = o_lma(p)
    x = mg.uniform(99, p.undf)
    X, Y = sysd.vector(x), sysd.vector()
    sysd.op.apply(X, Y)
    assert same(Y.export_field(), op.apply(x))
    assert same(sysd.diag.export_field(), op.diagonal())


@pytest.mark.parametrize("n,nl", [(3, 2), (12, 10), (24, 30)])
def test_lma_apply_w2_bitwise(ctx, n, nl):
    p = mg.w2_problem(n, nl, seed=n + 1)
    sysd = wl.device_w2(ctx, p)
    op = o_lma(p)
    x = mg.normal(7, p.undf)
    X, Y = sysd.vector(x), sysd.vector()
    sysd.op.apply(X, Y)
    assert same(Y.export_field(), op.apply(x))
    assert same(sysd.diag.export_field(), op.diagonal())


@pytest.mark.parametrize("kernel", [0, 1, 3, 4, 5, 6])
@pytest.mark.parametrize("space,n,nl,prec", [("w0", 6, 5, 64), ("w2", 8, 7, 64), ("w2", 8, 7, 32),
                                             ("w2", 12, 30, 64), ("w0", 5, 21, 32),
                                             ("w2", 6, 40, 64), ("w2", 7, 33, 32)])
def test_apply_kernels_agree(ctx, kernel, space, n, nl, prec):
    """Both LMA apply kernels (bulk-copy pipelined and register gather) give
    the oracle's FP64 result bit for bit, and the same FP32 result."""
    p = mg.w0_problem(n, nl, seed=3) if space == "w0" else mg.w2_problem(n, nl, seed=3)
    npc, cic = p.mesh.colour_lookup()
    ctx.set_apply_kernel(kernel)
    try:
        op = lfx.LmaOperator(ctx, p.ncell_2d, nl, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf,
                             p.lma, npc, cic, precision=prec)
        x = mg.normal(17, p.undf)
        X = lfx.FieldVector.from_array(ctx, x, prec)
        Y = lfx.FieldVector(ctx, [p.undf], prec)
        op.apply(X, Y)
        got = Y.export_field()
        ctx.check_device_error()
    finally:
        ctx.set_apply_kernel(-1)
    if prec == 64:
        assert same(got, o_lma(p).apply(x))
    else:
        ctx.set_apply_kernel(1 if kernel != 1 else 0)
        try:
            op.apply(X, Y)
            other = Y.export_field()
        finally:
            ctx.set_apply_kernel(-1)
        assert same(got, other)


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("space", ["w2", "w0"])
def test_cell_scatter_nonsymmetric(ctx, prec, space):
    """The cell scatter on local matrices that are not symmetric (full
    storage) gives the oracle's FP64 bits and the register gather's FP32 bits;
    forced inside a GMRES solve (whose residuals take a gather) the FP64 solve
    still matches the oracle bit for bit."""
    p = mg.w2_problem(7, 9, seed=21) if space == "w2" else mg.w0_problem(7, 9, seed=21)
    rng = np.random.default_rng(4)
    lma = p.lma * (1.0 + 0.01 * rng.standard_normal(p.lma.shape))
    npc, cic = p.mesh.colour_lookup()
    op = lfx.LmaOperator(ctx, p.ncell_2d, 9, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf, lma,
                         npc, cic, precision=prec)
    assert op.time_apply(5, 0, 0, reps=1) is not None
    x = mg.normal(8, p.undf)
    X = lfx.FieldVector.from_array(ctx, x, prec)
    Y = lfx.FieldVector(ctx, [p.undf], prec)
    got = {}
    for k, st, w in ((5, 0, 0), (5, 2, 0), (5, 3, 0), (1, 0, 0), (6, 4, 4)):
        op.set_apply(k, st, w)
        op.apply(X, Y)
        got[(k, st)] = Y.export_field()
    for k, st in ((5, 0), (5, 2), (5, 3), (6, 4)):
        assert same(got[(k, st)], got[(1, 0)])
    if prec == 64:
        oop = orc.LmaOperator(p.ncell_2d, 9, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf, lma,
                              npc, cic)
        assert same(got[(5, 0)], oop.apply(x))


@pytest.mark.parametrize("space,n,nl", [("w2", 9, 30), ("w0", 6, 20), ("w2", 5, 31)])
@pytest.mark.parametrize("prec", [64, 32])
def test_cell_scatter_stages_symmetric(ctx, space, n, nl, prec):
    """Symmetric operators (packed upper triangle) in every cell-scatter
    configuration: FP64 equals the oracle, FP32 the register gather, bit for
    bit; 31 levels fill the warp (the top dof of a column on lane 31)."""
    p = mg.w2_problem(n, nl, seed=5) if space == "w2" else mg.w0_problem(n, nl, seed=5)
    npc, cic = p.mesh.colour_lookup()
    op = lfx.LmaOperator(ctx, p.ncell_2d, nl, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf, p.lma,
                         npc, cic, precision=prec)
    x = mg.normal(9, p.undf)
    X = lfx.FieldVector.from_array(ctx, x, prec)
    Y = lfx.FieldVector(ctx, [p.undf], prec)
    op.set_apply(1)
    op.apply(X, Y)
    ref = o_lma(p).apply(x) if prec == 64 else Y.export_field()
    for st in (0, 2, 3):
        op.set_apply(5, st)
        Y.set_scalar(7.0)
        op.apply(X, Y)
        assert same(Y.export_field(), ref)
    # the persistent form in every ring shape that fits (at least one does)
    ran = 0
    for st, w in ((4, 4), (4, 8), (6, 4), (6, 8)):
        if op.time_apply(6, st, w, reps=1) is None:
            continue
        op.set_apply(6, st, w)
        Y.set_scalar(7.0)
        op.apply(X, Y)
        ctx.check_device_error()
        assert same(Y.export_field(), ref), (st, w)
        ran += 1
    assert ran >= 1


@pytest.mark.parametrize("space,n,nl", [("w2", 5, 32), ("w2", 4, 40), ("w0", 4, 63),
                                         ("w2", 3, 70), ("w0", 3, 70)])
@pytest.mark.parametrize("prec", [64, 32])
def test_cell_scatter_long_columns(ctx, space, n, nl, prec):
    """Columns of more than 31 levels take several warps per cell column
    (segments whose lane 0 supplies the face shared with the segment below):
    FP64 equals the oracle and FP32 the register gather, bit for bit, for the
    packed symmetric and the full (non-symmetric) storage."""
    p = mg.w2_problem(n, nl, seed=6) if space == "w2" else mg.w0_problem(n, nl, seed=6)
    npc, cic = p.mesh.colour_lookup()
    rng = np.random.default_rng(8)
    x = mg.normal(10, p.undf)
    for lma in (p.lma, p.lma * (1.0 + 0.01 * rng.standard_normal(p.lma.shape))):
        op = lfx.LmaOperator(ctx, p.ncell_2d, nl, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf,
                             lma, npc, cic, precision=prec)
        X = lfx.FieldVector.from_array(ctx, x, prec)
        Y = lfx.FieldVector(ctx, [p.undf], prec)
        op.set_apply(1)
        op.apply(X, Y)
        gather = Y.export_field()
        op.set_apply(5, 0)
        Y.set_scalar(3.0)
        op.apply(X, Y)
        got = Y.export_field()
        ctx.check_device_error()
        if prec == 64:
            oop = orc.LmaOperator(p.ncell_2d, nl, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf,
                                  lma, npc, cic)
            assert same(got, oop.apply(x))
        assert same(got, gather)


def test_cell_scatter_long_columns_in_gmres(ctx):
    """A 40-level W2 GMRES solve through the segmented cell scatter (plain and
    residual-form applies) equals the oracle's solve bit for bit."""
    p = mg.w2_problem(6, 40, seed=2)
    sysd = wl.device_w2(ctx, p)
    op = o_lma(p)
    oprec, _ = o_w2_prec(p, op)
    x_o, info_o = orc.solve("gmres", op, oprec, p.rhs, r_tol=1e-8, a_tol=1e-16, max_iter=200,
                            gcrk=10)
    sysd.op.set_apply(5, 0)
    g = lfx.GMRES(sysd.op, sysd.prec, 10, 1e-8, 1e-16, 200)
    X, B = sysd.vector(), sysd.vector(p.rhs)
    info = g.apply(X, B)
    assert info.converged and info.iterations == info_o.iterations
    assert same(X.export_field(), x_o)


@pytest.mark.parametrize("kernel", [5, 6])
def test_cell_scatter_in_gmres(ctx, kernel):
    """A W2 GMRES solve with every apply (plain and residual form) through the
    cell scatter, per colour or as one persistent launch, equals the oracle's
    solve bit for bit."""
    p = mg.w2_problem(16, 12, seed=2)
    sysd = wl.device_w2(ctx, p)
    op = o_lma(p)
    oprec, _ = o_w2_prec(p, op)
    x_o, info_o = orc.solve("gmres", op, oprec, p.rhs, r_tol=1e-8, a_tol=1e-16, max_iter=200,
                            gcrk=10)
    ctx.set_apply_kernel(kernel)
    try:
        g = lfx.GMRES(sysd.op, sysd.prec, 10, 1e-8, 1e-16, 200)
        X, B = sysd.vector(), sysd.vector(p.rhs)
        info = g.apply(X, B)
        ctx.check_device_error()
    finally:
        ctx.set_apply_kernel(-1)
    assert info.converged and info.iterations == info_o.iterations
    assert same(X.export_field(), x_o)


@pytest.mark.parametrize("prec", [64, 32])
def test_prefetch_gather_variants(ctx, prec):
    """Both register caps of the prefetching gather time and give the register
    gather's bits on W2; W0 (columns of four cells) is refused."""
    p = mg.w2_problem(9, 12, seed=12)
    npc, cic = p.mesh.colour_lookup()
    op = lfx.LmaOperator(ctx, p.ncell_2d, 12, 6, 6, p.map, p.map, p.undf, p.undf, p.lma, npc, cic,
                         precision=prec)
    for stages in (0, 1):
        assert op.time_apply(3, stages, 0, reps=2) > 0
    assert op.time_apply(3, 2, 0, reps=1) is None     # no such variant
    q = mg.w0_problem(5, 4, seed=1)
    nq, cq = q.mesh.colour_lookup()
    op0 = lfx.LmaOperator(ctx, q.ncell_2d, 4, 8, 8, q.map, q.map, q.undf, q.undf, q.lma, nq, cq)
    assert op0.time_apply(3, 0, 0, reps=1) is None


def test_autotune_keeps_results(ctx):
    p = mg.w2_problem(12, 10, seed=6)
    npc, cic = p.mesh.colour_lookup()
    op = lfx.LmaOperator(ctx, p.ncell_2d, 10, 6, 6, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
    x = mg.normal(2, p.undf)
    X, Y = lfx.FieldVector.from_array(ctx, x), lfx.FieldVector(ctx, [p.undf])
    choice = op.autotune(reps=3)
    assert choice["us"] > 0 and choice["kernel"] in ("pipeline", "register-gather",
                                                     "register-gather-prefetch",
                                                     "staged-pipeline", "cell-scatter",
                                                     "cell-scatter-persistent")
    op.apply(X, Y)
    assert same(Y.export_field(), o_lma(p).apply(x))


@pytest.mark.parametrize("kernel", [1, 3])
def test_divergence_and_transpose_bitwise(ctx, kernel):
    q = mg.w2_problem(6, 4, seed=3, keep_parts=True)
    npc, cic = q.mesh.colour_lookup()
    m3, u3 = q.extra["map_w3"], q.extra["undf_w3"]
    D = lfx.LmaOperator(ctx, q.ncell_2d, 4, 1, 6, m3, q.map, u3, q.undf, q.extra["div"], npc, cic)
    oD = orc.LmaOperator(q.ncell_2d, 4, 1, 6, m3, q.map, u3, q.undf, q.extra["div"], npc, cic)
    oDt = orc.LmaOperator(q.ncell_2d, 4, 1, 6, m3, q.map, u3, q.undf, q.extra["div"], npc, cic,
                          transpose=True)
    u = mg.normal(5, q.undf)
    w = mg.normal(6, u3)
    U = lfx.FieldVector.from_array(ctx, u)
    W = lfx.FieldVector(ctx, [u3])
    ctx.set_apply_kernel(kernel)
    try:
        D.apply(U, W)  # dg_matrix_vector: W2 -> W3
    finally:
        ctx.set_apply_kernel(-1)
    assert same(W.export_field(), oD.apply(u))
    W.import_field(w)
    U2 = lfx.FieldVector(ctx, [q.undf])
    D.apply_transpose(W, U2)  # transpose_matrix_vector: W3 -> W2
    assert same(U2.export_field(), oDt.apply(w))


def test_lma_fp32_apply(ctx):
    p = mg.w2_problem(12, 10, seed=8)
    s32 = wl.device_w2(ctx, p, lfx.R32)
    x = mg.normal(3, p.undf)
    X, Y = s32.vector(x), s32.vector()
    s32.op.apply(X, Y)
    ref = o_lma(p).apply(x)
    err = np.linalg.norm(Y.export_field() - ref) / np.linalg.norm(ref)
    assert err < 1e-6


# ------------------------------------------------------------------ CMA
@pytest.mark.parametrize("n,nl", [(12, 10), (5, 70)])
def test_cma_assembly_and_preconditioner_bitwise(ctx, n, nl):
    """Column assembly and Thomas sweeps equal the oracle bit for bit (5 x 70:
    columns of 71 rows, a partial block of columns); the FP32 preconditioner
    agrees to FP32 rounding."""
    p = mg.w2_problem(n, nl, seed=5)
    sysd = wl.device_w2(ctx, p)
    op = o_lma(p)
    oprec, band = o_w2_prec(p, op)
    assert same(sysd.cma.band(), band)
    x = mg.normal(11, p.undf)
    X, Y = sysd.vector(x), sysd.vector()
    sysd.prec.apply(X, Y)
    want = oprec.apply(x)
    assert same(Y.export_field(), want)
    s32 = wl.device_w2(ctx, p, lfx.R32, op64=sysd.op64, cma=sysd.cma, diag64=sysd.diag)
    X32, Y32 = s32.vector(x), s32.vector()
    s32.prec.apply(X32, Y32)
    got32 = Y32.export_field()
    assert np.linalg.norm(got32 - want) <= 1e-6 * np.linalg.norm(want)
    if nl != 10:
        return
    # y += A x on the column space (columnwise_op_app)
    prm = mg.w2v_cma_params(p.nlayers)
    y0 = mg.normal(12, p.undf)
    Y.import_field(y0)
    sysd.cma.apply(X, Y)
    want = y0.copy()
    first = np.ascontiguousarray(p.map[:, 4])
    for c in range(p.ncell_2d):
        orc.lib().or_columnwise_op_app_code(c + 1, want, x, band, prm["nrow"], prm["nrow"], 3, 1, 1,
                                            1, 1, first[c:c + 1], prm["indirection"], first[c:c + 1],
                                            prm["indirection"])
    assert same(Y.export_field(), want)


def test_cma_zero_pivot_is_reported(ctx):
    nrow, ncell = 5, 3
    band = np.zeros(3 * nrow * ncell)
    ind = np.arange(1, nrow + 1, dtype=np.int32)
    first = np.array([1, 6, 11], dtype=np.int32)
    cma = lfx.ColumnwiseOperator.from_band(ctx, ncell, nrow, 3, 1, 1, 1, 1, first, ind, band)
    with pytest.raises(lfx.LfxError) as e:
        lfx.ColumnwisePreconditioner(ctx, cma, None)
    assert e.value.status == 2


# ------------------------------------------------------------------ solvers
def test_cg_config0_parity(ctx):
    """C24 x 20 W0 mass+diffusion, Jacobi CG to 1e-8: the device solve equals
    the oracle's: same iteration count, bit-identical residual and solution."""
    p = mg.w0_problem(24, 20, seed=1)
    sysd = wl.device_w0(ctx, p)
    op = o_lma(p)
    x_o, info_o = orc.solve("cg", op, orc.Preconditioner.diagonal(op.diagonal()), p.rhs,
                            r_tol=1e-8, a_tol=1e-16, max_iter=2000)
    cg = lfx.ConjugateGradient(sysd.op, sysd.prec, 1e-8, 1e-16, 2000)
    X, B = sysd.vector(), sysd.vector(p.rhs)
    info = cg.apply(X, B)
    assert info.converged and info_o.converged
    assert info.iterations == info_o.iterations
    assert abs(info.final_rel - info_o.final_rel) <= 1e-12 * info_o.final_rel
    assert same(X.export_field(), x_o)


@pytest.mark.parametrize("kind", ["bicgstab", "gmres"])
def test_w0_solvers_parity(ctx, kind):
    p = mg.w0_problem(12, 10, seed=2)
    sysd = wl.device_w0(ctx, p)
    op = o_lma(p)
    P = orc.Preconditioner.diagonal(op.diagonal())
    x_o, info_o = orc.solve(kind, op, P, p.rhs, r_tol=1e-8, a_tol=1e-16, max_iter=2000, gcrk=10)
    if kind == "bicgstab":
        s = lfx.BiCGStab(sysd.op, sysd.prec, 1e-8, 1e-16, 2000)
    else:
        s = lfx.GMRES(sysd.op, sysd.prec, 10, 1e-8, 1e-16, 2000)
    X, B = sysd.vector(), sysd.vector(p.rhs)
    info = s.apply(X, B)
    assert info.converged and info.iterations == info_o.iterations
    assert abs(info.final_rel - info_o.final_rel) <= 1e-12 * info_o.final_rel
    assert same(X.export_field(), x_o)


@pytest.mark.parametrize("n,nl", [(24, 30), (96, 30)])
def test_gmres_w2_cma_parity(ctx, n, nl):
    """W2-W3 Helmholtz GMRES(10) with the column-tridiagonal preconditioner
    (the C96 x 30 case is the full-size configuration)."""
    p = mg.w2_problem(n, nl, seed=2)
    sysd = wl.device_w2(ctx, p)
    op = o_lma(p)
    oprec, _ = o_w2_prec(p, op)
    x_o, info_o = orc.solve("gmres", op, oprec, p.rhs, r_tol=1e-8, a_tol=1e-16, max_iter=200,
                            gcrk=10)
    g = lfx.GMRES(sysd.op, sysd.prec, 10, 1e-8, 1e-16, 200)
    X, B = sysd.vector(), sysd.vector(p.rhs)
    info = g.apply(X, B)
    assert info.converged and info.iterations == info_o.iterations
    assert abs(info.final_rel - info_o.final_rel) <= 1e-12 * info_o.final_rel
    assert same(X.export_field(), x_o)


def test_gmres_nonzero_initial_guess(ctx):
    """A nonzero initial guess takes the full residual apply (a zero one skips
    it, since b - A 0 = b): both equal the oracle bit for bit."""
    p = mg.w2_problem(12, 10, seed=7)
    sysd = wl.device_w2(ctx, p)
    op = o_lma(p)
    oprec, _ = o_w2_prec(p, op)
    x0 = 1e-3 * mg.normal(21, p.undf)
    x_o, info_o = orc.solve("gmres", op, oprec, p.rhs, x0=x0, r_tol=1e-8, a_tol=1e-16,
                            max_iter=200, gcrk=10)
    g = lfx.GMRES(sysd.op, sysd.prec, 10, 1e-8, 1e-16, 200)
    X, B = sysd.vector(x0), sysd.vector(p.rhs)
    info = g.apply(X, B)
    assert info.converged and info.iterations == info_o.iterations
    assert same(X.export_field(), x_o)


@pytest.mark.parametrize("kind", ["fgmres", "gcr"])
@pytest.mark.parametrize("space", ["w0", "w2"])
def test_flexible_solvers_parity(ctx, kind, space):
    """FGMRES and GCR (device vector calls, host recurrences) equal the
    oracle's restatements: same cycles, bit-identical solution."""
    if space == "w0":
        p = mg.w0_problem(10, 8, seed=5)
        sysd = wl.device_w0(ctx, p)
        op = o_lma(p)
        P = orc.Preconditioner.diagonal(op.diagonal())
    else:
        p = mg.w2_problem(12, 15, seed=5)
        sysd = wl.device_w2(ctx, p)
        op = o_lma(p)
        P, _ = o_w2_prec(p, op)
    x0 = mg.normal(9, p.undf)
    x_o, info_o = orc.solve(kind, op, P, p.rhs, x0=x0, r_tol=1e-9, a_tol=1e-16, max_iter=300,
                            gcrk=8)
    cls = lfx.FGMRES if kind == "fgmres" else lfx.GCR
    s = cls(sysd.op, sysd.prec, 8, 1e-9, 1e-16, 300)
    X, B = sysd.vector(x0), sysd.vector(p.rhs)
    info = s.apply(X, B)
    assert info.converged and info_o.converged
    assert info.iterations == info_o.iterations
    if kind == "gcr":
        assert info.inner_iterations == info_o.iv_final
    assert info.final_rel == info_o.final_rel
    assert same(X.export_field(), x_o)


@pytest.mark.parametrize("kind", ["precondition_only", "jacobi", "chebyshev"])
def test_stationary_solvers_parity(ctx, kind):
    """Precondition-only, Jacobi and Chebyshev (device vector calls) equal the
    oracle's restatements bit for bit."""
    p = mg.w2_problem(10, 12, seed=6)
    sysd = wl.device_w2(ctx, p)
    op = o_lma(p)
    P, _ = o_w2_prec(p, op)
    x0 = mg.normal(4, p.undf)
    it = 30 if kind == "chebyshev" else 400
    args = dict(r_tol=1e-7, a_tol=0.0, max_iter=it, rho_relax=0.8, lmin=0.05, lmax=1.6)
    x_o, info_o = orc.solve(kind, op, P, p.rhs, x0=x0, **args)
    if kind == "precondition_only":
        s = lfx.PreconditionOnly(sysd.op, sysd.prec)
    elif kind == "jacobi":
        s = lfx.Jacobi(sysd.op, sysd.prec, 1e-7, 0.0, 400, rho_relax=0.8)
    else:
        s = lfx.Chebyshev(sysd.op, sysd.prec, 1e-7, 0.0, 30, lmin=0.05, lmax=1.6)
    X, B = sysd.vector(x0), sysd.vector(p.rhs)
    info = s.apply(X, B)
    assert info.iterations == info_o.iterations
    assert info.final_rel == info_o.final_rel
    assert same(X.export_field(), x_o)
    if kind == "chebyshev":
        with pytest.raises(lfx.LfxError):
            lfx.Chebyshev(sysd.op, sysd.prec, 1e-7, 0.0, 5, fail_on_non_converged=True,
                          lmin=0.05, lmax=1.6).apply(X, B)


def test_gcr_nonconvergence_always_fails(ctx):
    """gcr_solve logs non-convergence as an error in both branches, so the
    device GCR returns LFX_NOT_CONVERGED even without fail_on_non_converged;
    FGMRES follows fail_on_non_converged."""
    p = mg.w2_problem(8, 6, seed=3)
    sysd = wl.device_w2(ctx, p)
    X, B = sysd.vector(), sysd.vector(p.rhs)
    with pytest.raises(lfx.LfxError) as e:
        lfx.GCR(sysd.op, sysd.prec, 2, 1e-12, 0.0, 1).apply(X, B)
    assert e.value.status == 1
    X.set_scalar(0.0)
    info = lfx.FGMRES(sysd.op, sysd.prec, 2, 1e-12, 0.0, 1).apply(X, B)
    assert not info.converged
    with pytest.raises(lfx.LfxError):
        lfx.FGMRES(sysd.op, sysd.prec, 2, 1e-12, 0.0, 1, fail_on_non_converged=True).apply(X, B)


def test_mixed_precision_refinement(ctx):
    """FP32 GMRES inside FP64 refinement reaches the 1e-8 true FP64 residual;
    the solution agrees with the FP64 oracle within the solve tolerance."""
    p = mg.w2_problem(24, 30, seed=4)
    s32 = wl.device_w2(ctx, p, lfx.R32)
    ir = wl.refined_gmres(s32, gcrk=10, inner_rtol=1e-4)
    X = lfx.FieldVector(ctx, [p.undf])
    X.set_scalar(0.0)
    B = lfx.FieldVector.from_array(ctx, p.rhs)
    info = ir.apply(X, B)
    assert info.converged and info.final_rel <= 1e-8
    op = o_lma(p)
    x = X.export_field()
    true_rel = np.linalg.norm(p.rhs - op.apply(x)) / np.linalg.norm(p.rhs)
    assert true_rel <= 1.01e-8
    oprec, _ = o_w2_prec(p, op)
    x_o, _ = orc.solve("gmres", op, oprec, p.rhs, r_tol=1e-10, max_iter=200, gcrk=10)
    assert np.linalg.norm(x - x_o) / np.linalg.norm(x_o) < 1e-6


# ------------------------------------------------------------------ edge cases
def test_zero_rhs_and_nan_and_nonconvergence(ctx):
    p = mg.w0_problem(6, 4, seed=3)
    sysd = wl.device_w0(ctx, p)
    for cls in (lfx.ConjugateGradient, lfx.BiCGStab):
        X, B = sysd.vector(), sysd.vector()
        info = cls(sysd.op, sysd.prec, 1e-8, 1e-16, 50).apply(X, B)
        assert info.converged and info.iterations == 0
    info = lfx.GMRES(sysd.op, sysd.prec, 5, 1e-8, 1e-16, 50).apply(sysd.vector(), sysd.vector())
    assert info.converged and info.iterations == 0
    bad = p.rhs.copy()
    bad[17] = np.nan
    with pytest.raises(lfx.LfxError) as e:
        lfx.ConjugateGradient(sysd.op, sysd.prec, 1e-8, 1e-16, 50).apply(sysd.vector(), sysd.vector(bad))
    assert e.value.status == 2
    # one iteration only: reported, and an error when fail_on_non_converged
    info = lfx.ConjugateGradient(sysd.op, sysd.prec, 1e-8, 1e-16, 1).apply(sysd.vector(),
                                                                           sysd.vector(p.rhs))
    assert not info.converged and info.iterations == 1
    with pytest.raises(lfx.LfxError) as e:
        lfx.ConjugateGradient(sysd.op, sysd.prec, 1e-8, 1e-16, 1, True, True).apply(
            sysd.vector(), sysd.vector(p.rhs))
    assert e.value.status == 1


def test_argument_errors(ctx):
    p = mg.w0_problem(4, 2, seed=1)
    sysd = wl.device_w0(ctx, p)
    X = sysd.vector()
    Y32 = lfx.FieldVector(ctx, [p.undf], lfx.R32)
    with pytest.raises(lfx.LfxError) as e:
        sysd.op.apply(X, Y32)
    assert e.value.status == 5
    with pytest.raises(lfx.LfxError) as e:
        X.axpy(1.0, lfx.FieldVector(ctx, [p.undf + 1]))
    assert e.value.status == 5
    npc, cic = p.mesh.colour_lookup()
    cic_bad = cic.copy()
    cic_bad[0, 0] = cic_bad[0, 1]  # a cell listed twice
    with pytest.raises(lfx.LfxError) as e:
        lfx.LmaOperator(ctx, p.ncell_2d, 2, 8, 8, p.map, p.map, p.undf, p.undf, p.lma, npc, cic_bad)
    assert e.value.status == 4


def test_lma_sum_operator_x_plus_ay_bitwise(ctx):
    """A = M2 + tau D^T D formed on the device from two operators on one
    layout (operator_x_plus_ay) applies bit for bit like the oracle's operator
    built from the oracle's own sum, with every apply kernel; the FP32 pair
    agrees to FP32 rounding."""
    q = mg.w2_problem(6, 5, seed=9, keep_parts=True)
    nc3, tau = q.mesh.ncell_3d, q.extra["tau"]
    D = q.extra["div"].reshape(6, nc3)          # Fortran (nc3, 1, 6): [j][ik]
    dtd = (D[None, :, :] * D[:, None, :]).ravel()  # Fortran (nc3, 6, 6): [j][i][ik] = D_i D_j
    m2 = q.extra["m2"]
    npc, cic = q.mesh.colour_lookup()
    opM = lfx.LmaOperator(ctx, q.ncell_2d, 5, 6, 6, q.map, q.map, q.undf, q.undf, m2, npc, cic)
    opA = opM.x_plus_ay(tau, opM.like(dtd, lfx.R64))
    host = orc.operator_x_plus_ay(m2, tau, dtd, q.ncell_2d, 5, 6, 6)
    assert np.allclose(host, q.lma, rtol=1e-12, atol=1e-15)
    oA = orc.LmaOperator(q.ncell_2d, 5, 6, 6, q.map, q.map, q.undf, q.undf, host, npc, cic)
    x = mg.normal(17, q.undf)
    want = oA.apply(x)
    X, Y = lfx.FieldVector.from_array(ctx, x), lfx.FieldVector(ctx, [q.undf])
    for kernel in (1, 3, 5):
        ctx.set_apply_kernel(kernel)
        try:
            opA.apply(X, Y)
        finally:
            ctx.set_apply_kernel(-1)
        assert same(Y.export_field(), want), kernel
    op32 = opM.like(m2, lfx.R32).x_plus_ay(tau, opM.like(dtd, lfx.R32))
    X32, Y32 = lfx.FieldVector.from_array(ctx, x, lfx.R32), lfx.FieldVector(ctx, [q.undf], lfx.R32)
    op32.apply(X32, Y32)
    err = np.linalg.norm(Y32.export_field() - want) / np.linalg.norm(want)
    assert err < 1e-6
    with pytest.raises(lfx.LfxError) as e:
        opM.x_plus_ay(1.0, op32)  # precisions differ
    assert e.value.status == 5
