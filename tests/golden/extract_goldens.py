"""Extract the known-answer data of the reference's pFUnit kernel tests into
tests/golden/kernel_goldens.json.

Run in a checkout that has the reference tree (default location given by
--ref). The tests read only the JSON; the reference is not needed at test
time. Each entry records the .pf file it came from.

Sources (paths inside the reference project):
  components/science/unit-test/kernel/algebra/matrix_vector_mod_test.pf
  components/science/unit-test/kernel/solver/sci_tri_solve_kernel_mod_test.pf
  components/science/unit-test/kernel/columnwise_operators/columnwise_op_appinv_kernel_mod_test.pf
  components/science/unit-test/kernel/columnwise_operators/columnwise_op_asm_kernel_mod_test.pf
  components/science/unit-test/kernel/columnwise_operators/columnwise_op_app_kernel_mod_test.pf
"""
from __future__ import annotations

import argparse
import json
import re
from pathlib import Path

NUM = r"[-+]?\d+\.?\d*(?:[eEdD][-+]?\d+)?"


def fnum(tok: str) -> float:
    tok = tok.split("_")[0].replace("d", "e").replace("D", "e")
    return float(tok)


def matrix_vector(text: str) -> dict:
    # first (real64) test: d(1,i,:) = (/ a, b /) rows and x(:) = (/ .. /)
    body = text.split("subroutine test_real64")[1].split("end subroutine test_real64")[0]
    rows = re.findall(r"d\(1,(\d),:\)\s*=\s*\(/\s*(" + NUM + r")_r_double,\s*(" + NUM + r")_r_double", body)
    d = [[fnum(a), fnum(b)] for _, a, b in sorted(rows)]
    xs = re.search(r"x\(:\)\s*=\s*\(/\s*(" + NUM + r")_r_double,\s*(" + NUM + r")_r_double", body)
    tol = re.search(r"tol\s*=\s*(" + NUM + r")_r_double", body)
    return {"d": d, "x": [fnum(xs.group(1)), fnum(xs.group(2))], "tol": fnum(tol.group(1))}


def tri_solve(text: str) -> dict:
    x = re.search(r"x\s*=\s*real\(\(/([^/]*)/\)", text).group(1)
    ans = re.search(r"answer\s*=\s*\(/(.*?)/\)", text, re.S).group(1)
    a0 = re.search(r"A0\s*=\s*(" + NUM + ")", text).group(1)
    ap = re.search(r"AP\s*=\s*(" + NUM + ")", text).group(1)
    am = re.search(r"AM\s*=\s*(" + NUM + ")", text).group(1)
    nz = re.search(r"nz\s*=\s*(\d+)", text).group(1)
    return {
        "nz": int(nz),
        "x": [float(v) for v in x.split(",")],
        "answer": [fnum(v) for v in re.findall(NUM + r"_r_def", ans)],
        "A0": fnum(a0), "AP": fnum(ap), "AM": fnum(am),
        "reference_tol": fnum(re.search(r"tol\s*=\s*(" + NUM + ")", text).group(1)),
    }


def cma_band(text: str) -> dict:
    # the 1/3, 1/6, 2/3 tridiagonal pattern on a Wtheta column of nlayers layers
    nl = int(re.search(r"nlayers\s*=\s*(\d+)", text).group(1))
    tol = fnum(re.search(r"tol\s*=\s*(" + NUM + ")", text).group(1))
    return {"nlayers": nl, "nrow": nl + 1, "first_row": [None, 1 / 3, 1 / 6],
            "interior_row": [1 / 6, 2 / 3, 1 / 6], "last_row": [1 / 6, 1 / 3, None],
            "reference_tol": tol}


def cma_asm(text: str) -> dict:
    nl = int(re.search(r"nlayers\s*=\s*(\d+)", text).group(1))
    m = re.search(r"reshape\(\s*\(/\s*1\.0_r_solver/3\.0_r_solver,\s*1\.0_r_solver/6\.0_r_solver,"
                  r"\s*&?\s*1\.0_r_solver/6\.0_r_solver,\s*1\.0_r_solver/3\.0_r_solver\s*/\)", text)
    assert m, "asm stencil not found"
    return {"nlayers": nl, "local_stencil": [[1 / 3, 1 / 6], [1 / 6, 1 / 3]],
            "band_first": [None, 1 / 3, 1 / 6], "band_interior": [1 / 6, 2 / 3, 1 / 6],
            "band_last": [1 / 6, 1 / 3, None],
            "reference_tol": fnum(re.search(r"tol\s*=\s*(" + NUM + ")", text).group(1))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=str(Path(__file__).with_name("kernel_goldens.json")))
    a = ap.parse_args()
    ut = Path(a.ref) / "components/science/unit-test/kernel"
    src = {
        "matrix_vector": ut / "algebra/matrix_vector_mod_test.pf",
        "tri_solve": ut / "solver/sci_tri_solve_kernel_mod_test.pf",
        "cma_appinv": ut / "columnwise_operators/columnwise_op_appinv_kernel_mod_test.pf",
        "cma_app": ut / "columnwise_operators/columnwise_op_app_kernel_mod_test.pf",
        "cma_asm": ut / "columnwise_operators/columnwise_op_asm_kernel_mod_test.pf",
    }
    out = {
        "matrix_vector": matrix_vector(src["matrix_vector"].read_text()),
        "tri_solve": tri_solve(src["tri_solve"].read_text()),
        "cma_appinv": cma_band(src["cma_appinv"].read_text()),
        "cma_app": cma_band(src["cma_app"].read_text()),
        "cma_asm": cma_asm(src["cma_asm"].read_text()),
    }
    for k, p in src.items():
        out[k]["source"] = str(p.relative_to(Path(a.ref)))
    Path(a.out).write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", a.out)


if __name__ == "__main__":
    main()
