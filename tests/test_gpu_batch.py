"""GPU tests of the device FEM assembly and of batched (continuously admitted)
mixed-precision solves."""
import numpy as np
import pytest

from lfric_core_b200 import lfx
from lfric_core_b200 import meshgen as mg
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


@pytest.mark.parametrize("space", [mg.W0, mg.W2])
def test_device_fem_assembly_matches_host(ctx, space):
    """The device assembly produces the host generator's local matrices: the
    two operators apply bit-identically."""
    p = mg.w0_problem(6, 5, seed=4) if space == mg.W0 else mg.w2_problem(6, 5, seed=4)
    ops, m, undf = lfx.fem_operators(ctx, p.mesh, space, 1.0 if space == mg.W0 else 0.1)
    assert np.array_equal(m, p.map) and undf == p.undf
    npc, cic = p.mesh.colour_lookup()
    host = lfx.LmaOperator(ctx, p.ncell_2d, p.nlayers, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf,
                           p.lma, npc, cic)
    x = mg.normal(3, p.undf)
    X = lfx.FieldVector.from_array(ctx, x)
    Y1, Y2 = lfx.FieldVector(ctx, [p.undf]), lfx.FieldVector(ctx, [p.undf])
    host.apply(X, Y1)
    ops[lfx.R64].apply(X, Y2)
    assert same(Y1.export_field(), Y2.export_field())


def w0_system(ctx, n, nl, seed):
    mesh = mg.cubed_sphere(n, nl, seed=seed)
    ops, m, undf = lfx.fem_operators(ctx, mesh, mg.W0, 1.0)
    d32 = lfx.FieldVector(ctx, [undf], lfx.R32)
    ops[lfx.R32].diagonal(d32)
    prec = lfx.DiagonalPreconditioner(ctx, d32)
    b = lfx.FieldVector.from_array(ctx, mg.uniform(seed + 7, undf))
    return dict(mesh=mesh, ops=ops, prec=prec, b=b, undf=undf, map=m)


def run_batch(ctx, systems, tols, ndf=8, iters=4, shape=None):
    B = lfx.Batch(ctx, ndf, len(systems), reserve_bytes=1 << 30, iters=iters)
    if shape:
        B.set_tuning(*shape)
    xs = []
    for i, (s, tol) in enumerate(zip(systems, tols)):
        x = lfx.FieldVector(ctx, [s["undf"]])
        x.set_scalar(0.0)
        slot = B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x, tol, 5000, tag=i)
        assert slot is not None
        xs.append((slot, x))
    for _ in range(2000):
        if B.step() == len(systems):
            break
    out = []
    for slot, x in xs:
        ph, tag, info = B.slot(slot)
        assert ph == 3 and info.status == 0, (ph, info.as_dict())
        out.append((x.export_field(), info.as_dict()))
        B.retire(slot)
    return out


def test_batch_results_same_alone_and_in_the_mix(ctx):
    specs = [(4, 3, 1, 1e-6), (6, 5, 2, 1e-8), (5, 7, 3, 1e-10), (8, 4, 4, 1e-9)]
    systems = [w0_system(ctx, n, nl, sd) for n, nl, sd, _ in specs]
    tols = [t for *_, t in specs]
    mixed = run_batch(ctx, systems, tols)
    for i, s in enumerate(systems):
        alone = run_batch(ctx, [s], [tols[i]])[0]
        assert same(alone[0], mixed[i][0])
        assert alone[1]["iterations"] == mixed[i][1]["iterations"]
    # every solution meets its tolerance on the FP64 operator (oracle apply)
    for (n, nl, sd, tol), s, (x, info) in zip(specs, systems, mixed):
        p = mg.w0_problem(n, nl, seed=sd)
        npc, cic = p.mesh.colour_lookup()
        op = orc.LmaOperator(p.ncell_2d, nl, 8, 8, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
        b = s["b"].export_field()
        rel = np.linalg.norm(b - op.apply(x)) / np.linalg.norm(b)
        assert rel <= tol * 1.0001, (rel, tol, info)


def test_batch_results_do_not_depend_on_the_launch_shape(ctx):
    """Columns per work item, blocks per SM and L2 group size change how the
    persistent kernel splits the work, not the sums: the same bits."""
    specs = [(5, 33, 1, 1e-9), (7, 12, 2, 1e-8), (4, 40, 3, 1e-10), (6, 31, 4, 1e-9),
             (5, 30, 5, 1e-8)]
    systems = [w0_system(ctx, n, nl, sd) for n, nl, sd, _ in specs]
    tols = [t for *_, t in specs]
    ref = run_batch(ctx, systems, tols, shape=(4, 2, 1 << 40))
    for shape in ((1, 1, 1 << 40), (8, 2, 1), (2, 2, 40_000)):
        got = run_batch(ctx, systems, tols, iters=3, shape=shape)
        for (xa, ia), (xb, ib) in zip(ref, got):
            assert same(xa, xb) and ia["iterations"] == ib["iterations"], shape


def test_batch_autotune_keeps_results(ctx):
    """The autotuner's timed replays advance the solves; the results are the
    bits of an untuned run."""
    specs = [(6, 20, 4, 1e-9), (5, 45, 5, 1e-8)]
    systems = [w0_system(ctx, n, nl, sd) for n, nl, sd, _ in specs]
    tols = [t for *_, t in specs]
    ref = run_batch(ctx, systems, tols)
    B = lfx.Batch(ctx, 8, 2, reserve_bytes=1 << 30, iters=4)
    xs = []
    for s, tol in zip(systems, tols):
        x = lfx.FieldVector(ctx, [s["undf"]])
        x.set_scalar(0.0)
        xs.append((B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x, tol, 5000), x))
    t = B.autotune(iters=2)
    assert t["cells_per_item"] in (1, 2, 4, 8) and t["us_per_iteration"] > 0
    for _ in range(2000):
        if B.step() == 2:
            break
    for (slot, x), (xr, ir) in zip(xs, ref):
        ph, _, info = B.slot(slot)
        assert ph == 3 and info.iterations == ir["iterations"]
        assert same(x.export_field(), xr)


def test_batch_admission_while_running(ctx):
    """Slots admitted while others are iterating: results are unchanged."""
    systems = [w0_system(ctx, 6, 5, 10 + i) for i in range(3)]
    ref = [run_batch(ctx, [s], [1e-8])[0][0] for s in systems]
    B = lfx.Batch(ctx, 8, 2, reserve_bytes=1 << 30, iters=2)
    xs = {}
    pending = list(range(3))
    finished = {}
    for _ in range(5000):
        while pending:
            i = pending[0]
            x = lfx.FieldVector(ctx, [systems[i]["undf"]])
            x.set_scalar(0.0)
            s = systems[i]
            slot = B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x, 1e-8, 5000, i)
            if slot is None:
                break
            xs[slot] = (i, x)
            pending.pop(0)
        B.step()
        for slot in B.done_slots():
            i, x = xs.pop(slot)
            finished[i] = x.export_field()
            B.retire(slot)
        if len(finished) == 3:
            break
    assert len(finished) == 3
    for i in range(3):
        assert same(finished[i], ref[i])


def test_batch_w2_line_preconditioner(ctx):
    """W2 Helmholtz systems with the column preconditioner: batch results are
    the same alone and in the mix, and reach the tolerance on FP64."""
    from lfric_core_b200 import workloads as wl
    systems = [wl.batch_system(ctx, n, nl, sd, mg.W2) for n, nl, sd in ((4, 6, 1), (6, 5, 2), (5, 9, 3))]
    tols = [1e-7, 1e-9, 1e-10]
    tot = sum(s.undf for s in systems)
    ent = sum(s.entities for s in systems)
    col = sum(s.columns for s in systems)

    def run(idx):
        B = lfx.Batch(ctx, 6, len(idx), reserve_bytes=1 << 30, iters=3)
        xs = []
        for i in idx:
            s = systems[i]
            x = lfx.FieldVector(ctx, [s.undf])
            x.set_scalar(0.0)
            xs.append((B.admit(s.ops[lfx.R64], s.ops[lfx.R32], s.prec32, s.b, x, tols[i], 5000), x))
        for _ in range(3000):
            if B.step() == len(idx):
                break
        out = []
        for slot, x in xs:
            ph, _, info = B.slot(slot)
            assert ph == 3 and info.status == 0
            out.append(x.export_field())
        return out

    assert tot and ent and col
    mixed = run([0, 1, 2])
    for (n, nl, sd), i in zip(((4, 6, 1), (6, 5, 2), (5, 9, 3)), range(3)):
        assert same(run([i])[0], mixed[i])
        # the true residual with the oracle's FP64 apply of the same system
        # (the device assembly equals the host generator's matrices)
        p = mg.w2_problem(n, nl, seed=sd)
        npc, cic = p.mesh.colour_lookup()
        op = orc.LmaOperator(p.ncell_2d, nl, 6, 6, p.map, p.map, p.undf, p.undf, p.lma, npc, cic)
        b = systems[i].b.export_field()
        rel = np.linalg.norm(b - op.apply(mixed[i])) / np.linalg.norm(b)
        assert rel <= tols[i] * 1.0001, (i, rel)


def test_batch_refuses_when_full(ctx):
    s = w0_system(ctx, 4, 3, 5)
    B = lfx.Batch(ctx, 8, 1, reserve_bytes=1 << 30, iters=2)
    x1, x2 = lfx.FieldVector(ctx, [s["undf"]]), lfx.FieldVector(ctx, [s["undf"]])
    assert B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x1, 1e-8) is not None
    assert B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x2, 1e-8) is None


def test_batch_admission_by_free_device_memory(ctx):
    """A reserve larger than the device's memory refuses every admission; a
    small one admits."""
    import torch
    s = w0_system(ctx, 4, 3, 6)
    total = torch.cuda.get_device_properties(0).total_memory
    x = lfx.FieldVector(ctx, [s["undf"]])
    full = lfx.Batch(ctx, 8, 4, reserve_bytes=total, iters=2)
    assert full.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x, 1e-8) is None
    ok = lfx.Batch(ctx, 8, 4, reserve_bytes=1 << 20, iters=2)
    x.set_scalar(0.0)
    slot = ok.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x, 1e-8)
    assert slot is not None
    for _ in range(1000):
        if ok.step() == 1:
            break
    assert ok.slot(slot)[0] == 3


def test_batch_barrier_wait_limit_runs_out_and_context_survives(ctx):
    """With a wait limit of one nanosecond every grid-barrier wait of the
    persistent kernel gives up at its first poll: the kernel sets LFX_TIMEOUT
    and every block leaves at its next barrier (no copy is in flight in that
    kernel). The step reports the timeout, and the context then runs a fresh
    batch to the same bits as before."""
    s = w0_system(ctx, 5, 6, 31)
    ref = run_batch(ctx, [s], [1e-8])[0][0]
    B = lfx.Batch(ctx, 8, 1, reserve_bytes=1 << 30, iters=2)
    B.set_wait_limit(1e-9)
    x = lfx.FieldVector(ctx, [s["undf"]])
    x.set_scalar(0.0)
    assert B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x, 1e-8) is not None
    with pytest.raises(lfx.LfxError) as e:
        B.step()
    assert e.value.status == 6  # LFX_TIMEOUT
    B.close()
    assert same(run_batch(ctx, [s], [1e-8])[0][0], ref)


def test_batch_general_pair_structure_matches_oracle(ctx):
    """The batch apply specialises the vertical-pair structure of the
    reference elements (W0: bottom vertices 0-3 under top vertices 4-7); an
    operator with another uniform structure takes the general path. The W0
    operator with its local dofs interleaved (bottom, top, bottom, top, ...,
    pairs (0, 1), (2, 3), ...) is the same global operator: the batch solve
    reaches its tolerance on the oracle's FP64 residual and agrees with the
    oracle's CG solution, and its bits differ from the reference-numbered
    solve's (the per-cell sums run in another order), so the other path ran."""
    p = mg.w0_problem(12, 31, seed=5)
    perm = [0, 4, 1, 5, 2, 6, 3, 7]
    full = p.lma.reshape(p.ndf, p.ndf, -1)
    lma_p = np.ascontiguousarray(full[np.ix_(perm, perm)]).reshape(-1)
    map_p = np.ascontiguousarray(p.map[:, perm])
    npc, cic = p.mesh.colour_lookup()
    b = lfx.FieldVector.from_array(ctx, mg.uniform(11, p.undf))
    tol = 1e-9
    xs = []
    for m, lma in ((map_p, lma_p), (p.map, p.lma)):
        op64 = lfx.LmaOperator(ctx, p.ncell_2d, p.nlayers, p.ndf, p.ndf, m, m, p.undf, p.undf,
                               lma, npc, cic, precision=lfx.R64)
        ops = {lfx.R64: op64, lfx.R32: op64.like(lma, lfx.R32)}
        d32 = lfx.FieldVector(ctx, [p.undf], lfx.R32)
        ops[lfx.R32].diagonal(d32)
        prec = lfx.DiagonalPreconditioner(ctx, d32)
        B = lfx.Batch(ctx, 8, 1, reserve_bytes=1 << 30, iters=8)
        x = lfx.FieldVector(ctx, [p.undf])
        x.set_scalar(0.0)
        slot = B.admit(ops[lfx.R64], ops[lfx.R32], prec, b, x, tol, 20000)
        for _ in range(2000):
            if B.step() == 1:
                break
        ph, _, info = B.slot(slot)
        assert ph == 3 and info.status == 0, info.as_dict()
        xs.append(x.export_field())
    o = orc.LmaOperator(p.ncell_2d, p.nlayers, p.ndf, p.ndf, p.map, p.map, p.undf, p.undf, p.lma,
                        npc, cic)
    bh = b.export_field()
    xo, oi = orc.solve("cg", o, orc.Preconditioner.diagonal(o.diagonal()), bh, r_tol=tol,
                       a_tol=0.0, max_iter=20000)
    assert oi.converged
    for xv in xs:
        rel = np.linalg.norm(bh - o.apply(xv)) / np.linalg.norm(bh)
        assert rel <= tol * 1.0001, rel
        assert np.linalg.norm(xv - xo) <= 1e4 * tol * np.linalg.norm(xo)
    assert not same(xs[0], xs[1])
