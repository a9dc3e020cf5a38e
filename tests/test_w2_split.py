"""W2 split / combine (split_w2_field_kernel_mod.F90, combine_w2_field_kernel_mod.F90):
the oracle's round trip on the CPU, the device against the oracle on a GPU."""
import numpy as np
import pytest

from lfric_core_b200 import meshgen as mg
from oracle import oracle as orc


def setup(n, nl, seed=3):
    p = mg.w2_problem(n, nl, seed=seed)
    mh, uh, mv, uv, m3, u3 = mg.w2_subspace_maps(p.map, nl)
    ew, ns = orc.face_selectors(m3, mh, u3, uh)
    maps = dict(w2=p.map, w2h=mh, w2v=mv, w3_2d=m3)
    return p, maps, (uh, uv, u3), ew, ns


@pytest.mark.parametrize("n,nl", [(3, 2), (6, 7), (5, 11)])
def test_oracle_split_combine_round_trip(n, nl):
    p, maps, (uh, uv, u3), ew, ns = setup(n, nl)
    # every cell copies W and S plus its selected E / N faces: 2..4 faces
    assert set(np.unique(ew)) <= {1, 2} and set(np.unique(ns)) <= {1, 2}
    x = np.random.default_rng(n).standard_normal(p.undf)
    a, b = orc.split_w2(nl, x, maps, ew, ns, uh, uv)
    assert np.array_equal(orc.combine_w2(nl, a, b, maps, ew, ns, p.undf), x)
    # the split pieces hold exactly the horizontal / vertical dofs of x
    assert np.isclose(np.sum(a * a) + np.sum(b * b), np.sum(x * x), rtol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [64, 32])
def test_device_split_combine_matches_oracle(ctx, prec):
    from lfric_core_b200 import lfx
    n, nl = 9, 13
    p, maps, (uh, uv, u3), ew, ns = setup(n, nl, seed=8)
    S = lfx.W2Split(ctx, nl, p.map, maps["w2h"], maps["w2v"], maps["w3_2d"], u3, ew, ns)
    x = np.random.default_rng(2).standard_normal(p.undf)
    if prec == 32:
        x = x.astype(np.float32).astype(np.float64)
    X = lfx.FieldVector.from_array(ctx, x, prec)
    A, B = lfx.FieldVector(ctx, [uh], prec), lfx.FieldVector(ctx, [uv], prec)
    A.set_scalar(0.0)
    B.set_scalar(0.0)
    S.split(X, A, B)
    a_o, b_o = orc.split_w2(nl, x, maps, ew, ns, uh, uv)
    assert np.array_equal(A.export_field(), a_o) and np.array_equal(B.export_field(), b_o)
    Y = lfx.FieldVector(ctx, [p.undf], prec)
    Y.set_scalar(0.0)
    S.combine(A, B, Y)
    assert np.array_equal(Y.export_field(), x)
    with pytest.raises(lfx.LfxError):
        S.split(X, lfx.FieldVector(ctx, [uh - 1], prec), B)
