"""CPU tests: generated mesh topology, dofmaps and colouring; the C ABI
libraries load and export every symbol their headers declare."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from lfric_core_b200 import meshgen as mg

ROOT = Path(__file__).resolve().parent.parent
SIDE_VERTS = {0: (0, 3), 1: (0, 1), 2: (1, 2), 3: (2, 3)}  # W,S,E,N -> (SW,SE,NE,NW) pairs


@pytest.mark.parametrize("n", [2, 3, 4, 5, 12])
def test_cubed_sphere_topology(n):
    m = mg.cubed_sphere(n, 3)
    ncell = 6 * n * n
    cn, vc = m.cell_next, m.verts_on_cell
    assert len(np.unique(vc)) == ncell + 2  # Euler: V = F + 2 on the sphere
    for c in range(ncell):
        for s in range(4):
            t = cn[c, s] - 1
            assert c + 1 in cn[t]
            a, b = SIDE_VERTS[s]
            assert {vc[c, a], vc[c, b]} <= set(vc[t])
    X = m.vert_xyz
    o = np.einsum("ij,ij->i", np.cross(X[vc[:, 1] - 1] - X[vc[:, 0] - 1],
                                       X[vc[:, 3] - 1] - X[vc[:, 0] - 1]), X[vc[:, 0] - 1])
    assert np.all(o > 0)  # every cell positively oriented
    np.testing.assert_allclose(np.linalg.norm(X, axis=1), 1.0, atol=1e-14)


@pytest.mark.parametrize("n,expect", [(2, 4), (4, 4), (24, 4), (3, None), (5, None)])
def test_colouring(n, expect):
    m = mg.cubed_sphere(n, 2)
    assert mg.lib().lfx_mg_test_colours(6 * n * n, m.cell_next, m.colour_map) == 1
    if expect:
        assert m.ncolours == expect  # panel pattern for even n
    npc, cic = m.colour_lookup()
    assert npc.sum() == 6 * n * n
    assert sorted(cic[cic > 0].tolist()) == list(range(1, 6 * n * n + 1))
    # no dof of W0 (vertices) is shared by two cells of one colour
    for col in range(1, m.ncolours + 1):
        cells = np.nonzero(m.colour_map == col)[0]
        verts = m.verts_on_cell[cells].ravel()
        assert len(verts) == len(np.unique(verts))


@pytest.mark.parametrize("nl", [1, 5, 20])
def test_dofmaps(nl):
    n = 6
    m = mg.cubed_sphere(n, nl)
    ncell = 6 * n * n
    nv, ne = ncell + 2, 2 * ncell
    m0, u0 = m.dofmap(mg.W0)
    m2, u2 = m.dofmap(mg.W2)
    m3, u3 = m.dofmap(mg.W3)
    assert u0 == nv * (nl + 1)
    assert u2 == ne * nl + ncell * (nl + 1)
    assert u3 == ncell * nl
    # top dof = bottom dof + 1 (column-contiguous numbering)
    assert np.all(m0[:, 4:] == m0[:, :4] + 1)
    assert np.all(m2[:, 5] == m2[:, 4] + 1)
    # every dof covered exactly once by the entity columns
    for mp, h_of in ((m0, lambda df: nl + 1 if df < 4 else None), (m3, lambda df: nl)):
        seen = np.zeros(u0 if mp is m0 else u3, dtype=np.int32)
        starts = set()
        for c in range(ncell):
            for df in range(mp.shape[1]):
                h = h_of(df)
                if h is None or mp[c, df] in starts:
                    continue
                starts.add(mp[c, df])
                seen[mp[c, df] - 1: mp[c, df] - 1 + h] += 1
        assert np.all(seen == 1)


def test_lma_symmetry_and_positivity():
    p = mg.w0_problem(4, 3, seed=5)
    A = p.lma.reshape(8, 8, -1)
    assert np.abs(A - A.transpose(1, 0, 2)).max() < 1e-15
    ev = np.linalg.eigvalsh(np.moveaxis(0.5 * (A + A.transpose(1, 0, 2)), 2, 0))
    assert ev.min() > 0
    q = mg.w2_problem(4, 3, seed=6, keep_parts=True)
    B = q.lma.reshape(6, 6, -1)
    assert np.abs(B - B.transpose(1, 0, 2)).max() < 1e-13
    assert np.linalg.eigvalsh(np.moveaxis(B, 2, 0)).min() > 0
    # A = M2 + tau D^T D
    M2 = q.extra["m2"].reshape(6, 6, -1)
    D = q.extra["div"].reshape(6, 1, -1)
    DtD = np.einsum("ik,jk->jik", D[:, 0, :], D[:, 0, :])
    np.testing.assert_allclose(B, M2 + 0.1 * DtD, atol=1e-13)


def _declared(header: Path):
    txt = header.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(lfx_\w+)\s*\(", txt)))


def test_lfx_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(ROOT / "lfric_core_b200" / "lib" / "liblfx.so"))
    names = _declared(ROOT / "include" / "lfx.h")
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from lfric_core_b200 import lfx
    assert set(lfx.EXPORTED) == set(names), set(names) ^ set(lfx.EXPORTED)
    lfx.load_library()  # binds every signature


def test_meshgen_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(ROOT / "lfric_core_b200" / "lib" / "liblfx_meshgen.so"))
    names = _declared(ROOT / "include" / "lfx_meshgen.h")
    assert names and all(hasattr(lib, n) for n in names)


def test_no_cpu_fallback_in_product():
    """The product package never imports or loads the oracle."""
    for f in (ROOT / "lfric_core_b200").rglob("*.py"):
        src = f.read_text()
        assert "oracle" not in src.replace("oracle", "ORACLE_WORD") or "import oracle" not in src
        assert "liboracle" not in src and "from oracle" not in src and "import oracle" not in src
