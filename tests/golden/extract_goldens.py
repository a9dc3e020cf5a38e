"""Extract the known-answer data of the reference's pFUnit kernel tests into
tests/golden/kernel_goldens.json.

Run with --ref pointing at a checkout of the reference tree. The tests read
only the JSON; the reference is not needed at test time. Each entry records the .pf file it came from.

Sources (paths inside the reference project):
  components/science/unit-test/kernel/algebra/matrix_vector_mod_test.pf
  components/science/unit-test/kernel/solver/sci_tri_solve_kernel_mod_test.pf
  components/science/unit-test/kernel/columnwise_operators/columnwise_op_appinv_kernel_mod_test.pf
  components/science/unit-test/kernel/columnwise_operators/columnwise_op_asm_kernel_mod_test.pf
  components/science/unit-test/kernel/columnwise_operators/columnwise_op_app_kernel_mod_test.pf
  components/science/unit-test/kernel/columnwise_operators/columnwise_op_{mul,scaledadd,
      asm_m2v_lumped_inv,asm_diag_hmht}_kernel_mod_test.pf
  components/science/unit-test/kernel/algebra/operator_algebra_kernel_mod_test.pf
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


def cma_mul(text: str) -> dict:
    # D (W3 <- Wtheta) band entries 1, 2 and its transpose's, nlayers
    nl = int(re.search(r"nlayers\s*=\s*(\d+)_i_def", text).group(1))
    d1 = fnum(re.search(r"clm_mat_D\(1_i_def,i,cell\)\s*=\s*(" + NUM + ")", text).group(1))
    d2 = fnum(re.search(r"clm_mat_D\(2_i_def,i,cell\)\s*=\s*(" + NUM + ")", text).group(1))
    t1 = fnum(re.search(r"clm_mat_DT\(1_i_def,i,cell\)\s*=\s*(" + NUM + ")", text).group(1))
    t2 = fnum(re.search(r"clm_mat_DT\(2_i_def,i,cell\)\s*=\s*(" + NUM + ")", text).group(1))
    return {"nlayers": nl, "D_band": [d1, d2], "DT_band": [t1, t2],
            "reference_tol": fnum(re.search(r"tol\s*=\s*(" + NUM + ")", text).group(1))}


def cma_scaledadd(text: str) -> dict:
    nl = int(re.search(r"nlayers\s*=\s*(\d+)_i_def", text).group(1))
    mu = fnum(re.search(r"mu\s*=\s*(" + NUM + ")_r_solver", text).group(1))
    nu = fnum(re.search(r"nu\s*=\s*(" + NUM + ")_r_solver", text).group(1))
    dtd = [fnum(re.search(r"clm_mat_DTD\(%d,i,cell\)\s*=\s*(" % k + NUM + ")", text).group(1))
           for k in (1, 2, 3)]
    m1 = fnum(re.search(r"clm_mat_M\(1,i,cell\)\s*=\s*(" + NUM + ")", text).group(1))
    return {"nlayers": nl, "mu": mu, "nu": nu, "DTD_band": dtd, "M_band": [m1],
            "reference_tol": fnum(re.search(r"tol\s*=\s*(" + NUM + ")", text).group(1))}


def cma_m2v_lumped_inv(text: str) -> dict:
    nl = int(re.search(r"nlayers\s*=\s*(\d+)", text).group(1))
    assert re.search(r"reshape\(\s*\(/\s*1\.0_r_solver/3\.0_r_solver,\s*1\.0_r_solver/6\.0_r_solver",
                     text), "m2v stencil not found"
    ends = fnum(re.search(r"answer\s*=\s*(" + NUM + r")_r_solver\s*\n", text).group(1))
    inner = re.search(r"answer\s*=\s*\((" + NUM + r")_r_solver/(" + NUM + r")_r_solver\)", text)
    return {"nlayers": nl, "local_stencil": [[1 / 3, 1 / 6], [1 / 6, 1 / 3]],
            "answer_end_rows": ends, "answer_interior_rows": fnum(inner.group(1)) / fnum(inner.group(2)),
            "reference_tol": fnum(re.search(r"tol\s*=\s*(" + NUM + ")", text).group(1))}


def cma_diag_hmht(text: str) -> dict:
    nl = int(re.search(r"nlayers\s*=\s*(\d+)", text).group(1))
    rho = [fnum(re.search(r"rho\(%d\)\s*=\s*(" % k + NUM + ")", text).group(1)) for k in range(1, 5)]
    sig = [fnum(re.search(r"sigma\(%d\)\s*=\s*(" % k + NUM + ")", text).group(1)) for k in range(1, 5)]
    return {"nlayers": nl, "rho": rho, "sigma": sig,
            "answer": sum(r * r / s for r, s in zip(rho, sig)),
            "reference_tol": fnum(re.search(r"tol\s*=\s*(" + NUM + ")", text).group(1))}


def operator_x_plus_ay(text: str) -> dict:
    # test_x_plus_ay: x(1,:,j) and y(1,:,j) constant per column j, scalar a,
    # answers per column
    body = text.split("subroutine test_x_plus_ay")[1].split("end subroutine test_x_plus_ay")[0]
    ndf1 = int(re.search(r"ndf1\s*=\s*(\d+)", body).group(1))
    ndf2 = int(re.search(r"ndf2\s*=\s*(\d+)", body).group(1))
    xs = {int(j): fnum(v) for j, v in re.findall(r"\bx\(1,:,(\d)\)\s*=\s*(" + NUM + ")", body)}
    ys = {int(j): fnum(v) for j, v in re.findall(r"\by\(1,:,(\d)\)\s*=\s*(" + NUM + ")", body)}
    a = fnum(re.search(r"::\s*a\s*=\s*(" + NUM + ")", body).group(1))
    ans = [fnum(v) for v in re.findall(r"answer\s*=\s*(" + NUM + ")", body)]
    return {"ndf1": ndf1, "ndf2": ndf2, "x": [xs[j + 1] for j in range(ndf2)],
            "y": [ys[j + 1] for j in range(ndf2)], "a": a, "answer": ans,
            "tol": fnum(re.search(r"tol\s*=\s*(" + NUM + ")", body).group(1))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference checkout")
    ap.add_argument("--out", default=str(Path(__file__).with_name("kernel_goldens.json")))
    a = ap.parse_args()
    ut = Path(a.ref) / "components/science/unit-test/kernel"
    src = {
        "matrix_vector": ut / "algebra/matrix_vector_mod_test.pf",
        "tri_solve": ut / "solver/sci_tri_solve_kernel_mod_test.pf",
        "cma_appinv": ut / "columnwise_operators/columnwise_op_appinv_kernel_mod_test.pf",
        "cma_app": ut / "columnwise_operators/columnwise_op_app_kernel_mod_test.pf",
        "cma_asm": ut / "columnwise_operators/columnwise_op_asm_kernel_mod_test.pf",
        "cma_mul": ut / "columnwise_operators/columnwise_op_mul_kernel_mod_test.pf",
        "cma_scaledadd": ut / "columnwise_operators/columnwise_op_scaledadd_kernel_mod_test.pf",
        "cma_m2v_lumped_inv":
            ut / "columnwise_operators/columnwise_op_asm_m2v_lumped_inv_kernel_mod_test.pf",
        "cma_diag_hmht": ut / "columnwise_operators/columnwise_op_asm_diag_hmht_kernel_mod_test.pf",
        "operator_x_plus_ay": ut / "algebra/operator_algebra_kernel_mod_test.pf",
    }
    out = {
        "matrix_vector": matrix_vector(src["matrix_vector"].read_text()),
        "tri_solve": tri_solve(src["tri_solve"].read_text()),
        "cma_appinv": cma_band(src["cma_appinv"].read_text()),
        "cma_app": cma_band(src["cma_app"].read_text()),
        "cma_asm": cma_asm(src["cma_asm"].read_text()),
        "cma_mul": cma_mul(src["cma_mul"].read_text()),
        "cma_scaledadd": cma_scaledadd(src["cma_scaledadd"].read_text()),
        "cma_m2v_lumped_inv": cma_m2v_lumped_inv(src["cma_m2v_lumped_inv"].read_text()),
        "cma_diag_hmht": cma_diag_hmht(src["cma_diag_hmht"].read_text()),
        "operator_x_plus_ay": operator_x_plus_ay(src["operator_x_plus_ay"].read_text()),
    }
    for k, p in src.items():
        out[k]["source"] = str(p.relative_to(Path(a.ref)))
    Path(a.out).write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", a.out)


if __name__ == "__main__":
    main()
