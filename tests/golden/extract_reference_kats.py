"""Extract the known-answer tests of veret-v/parallel_ds into reference_kats.json.

Sources (read as text; the reference's gtest targets do not build):
  * tests/simple_tests_DS.cpp:12-145 -- four small LPs with analytic optima
    (EXPECT_NEAR tolerance 1e-8, 1e-4 for Test4).
  * tests/test_math.cpp:12-49 -- 3x3 LU solve known answers (plain and transposed).

Run where the reference sources are:
    python tests/golden/extract_reference_kats.py REFERENCE_ROOT
The JSON it writes is committed; nothing at test time reads the reference.
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: extract_reference_kats.py REFERENCE_ROOT (the checkout of veret-v/parallel_ds)")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")

TYPES = {"Fixed": 0, "Free": 1, "Boxed": 2, "Upper": 3, "Lower": 4}


def vec(block, name, kind="double"):
    pat = (r"%s\s*\(\s*std::vector<%s>\{([^}]*)\}\s*\)" % (re.escape(name), kind))
    mm = re.search(pat, block)
    if not mm:
        raise ValueError(f"{name} not found")
    return [float(t) for t in mm.group(1).split(",")]


def types(block, name):
    mm = re.search(r"BoundaryTypeVector\s+%s\s*\{([^}]*)\}" % name, block, re.S)
    return [TYPES[t.strip().split("::")[1]] for t in mm.group(1).split(",")]


def matrix(block):
    mm = re.search(r"Matrix A\(\s*std::vector<double>\{([^}]*)\},\s*std::vector<MKL_INT>\{([^}]*)\},"
                   r"\s*std::vector<MKL_INT>\{([^}]*)\}", block, re.S)
    val = [float(t) for t in mm.group(1).split(",")]
    rp = [int(t) for t in mm.group(2).split(",")]
    ci = [int(t) for t in mm.group(3).split(",")]
    return val, rp, ci


def lps():
    path = os.path.join(REF, "tests", "simple_tests_DS.cpp")
    src = open(path).read()
    out = []
    for mm in re.finditer(r"TEST\(DualSimplexSimple, (Test\d)\)\s*\{(.*?)\n\}", src, re.S):
        name, block = mm.group(1), mm.group(2)
        line = src[:mm.start()].count("\n") + 1
        dims = re.search(r"int m = (\d+), n\s*=\s*(\d+);", block)
        m, n = int(dims.group(1)), int(dims.group(2))
        val, rp, ci = matrix(block)
        z = float(re.search(r"true_solution\.Z = ([-\d.]+);", block).group(1))
        tol = float(re.search(r"EXPECT_NEAR\(solution\.Z, true_solution\.Z, ([\de.-]+)\)", block).group(1))
        xs = vec(block, "true_solution.x = ValuesVector")
        out.append(dict(
            name=name, source=f"tests/simple_tests_DS.cpp:{line}", m=m, n=n,
            c=vec(block, "ValuesVector costs"),
            row_lb=vec(block, "ValuesVector lower_range"), row_ub=vec(block, "ValuesVector upper_range"),
            col_lb=vec(block, "ValuesVector lower_bound"), col_ub=vec(block, "ValuesVector upper_bound"),
            col_type=types(block, "bound_type"), row_type=types(block, "range_type"),
            val=val, row_ptr=rp, col_idx=ci, z=z, tol=tol, x=xs))
    return out


def lu_kats():
    path = os.path.join(REF, "tests", "test_math.cpp")
    src = open(path).read()
    out = []
    for mm in re.finditer(r"TEST\(Math, (Test[12])\)\s*\{(.*?)\n\}", src, re.S):
        name, block = mm.group(1), mm.group(2)
        line = src[:mm.start()].count("\n") + 1
        rhs = [float(t) for t in re.search(r"rhs1\(std::vector<double>\{([^}]*)\}", block).group(1).split(",")]
        exp = [float(t) for t in re.search(r"expected = \{([^}]*)\}", block).group(1).split(",")]
        val, rp, ci = matrix(block)
        transpose = "A.solve(rhs1, sol1, true)" in block
        out.append(dict(name=name, source=f"tests/test_math.cpp:{line}", n=3, val=val, row_ptr=rp,
                        col_idx=ci, rhs=rhs, expected=exp, transpose=transpose))
    return out


if __name__ == "__main__":
    data = dict(lps=lps(), lu=lu_kats())
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print(f"wrote {OUT}: {len(data['lps'])} LPs, {len(data['lu'])} LU KATs")
