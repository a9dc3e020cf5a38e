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


def run_batch(ctx, systems, tols, ndf=8, iters=4):
    tot = sum(s["undf"] for s in systems)
    ent = sum(len(np.unique(s["map"][:, :4])) if ndf == 8 else s["undf"] for s in systems) * 2
    B = lfx.Batch(ctx, ndf, len(systems), tot, ent, 0, iters)
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


def test_batch_admission_while_running(ctx):
    """Slots admitted while others are iterating: results are unchanged."""
    systems = [w0_system(ctx, 6, 5, 10 + i) for i in range(3)]
    ref = [run_batch(ctx, [s], [1e-8])[0][0] for s in systems]
    tot = sum(s["undf"] for s in systems)
    B = lfx.Batch(ctx, 8, 2, tot, tot, 0, 2)
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
        B = lfx.Batch(ctx, 6, len(idx), sum(systems[i].undf for i in idx),
                      sum(systems[i].entities for i in idx), sum(systems[i].columns for i in idx), 3)
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
    for i in range(3):
        assert same(run([i])[0], mixed[i])
        s = systems[i]
        X = lfx.FieldVector.from_array(ctx, mixed[i])
        R = lfx.FieldVector(ctx, [s.undf])
        s.ops[lfx.R64].apply(X, R)
        R.aypx(-1.0, s.b)
        assert R.norm() / s.b.norm() <= tols[i] * 1.0001


def test_batch_refuses_when_full(ctx):
    s = w0_system(ctx, 4, 3, 5)
    B = lfx.Batch(ctx, 8, 1, s["undf"], s["undf"], 0, 2)
    x1, x2 = lfx.FieldVector(ctx, [s["undf"]]), lfx.FieldVector(ctx, [s["undf"]])
    assert B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x1, 1e-8) is not None
    assert B.admit(s["ops"][lfx.R64], s["ops"][lfx.R32], s["prec"], s["b"], x2, 1e-8) is None
