"""Extract the reference's golden vectors into tests/golden/reference_unit_tests.json.

The reference pins its hot-path arithmetic with GoogleTest unit tests whose
expected values were computed in Mathematica (Tests/*/Test_*.cpp).  The
reference itself cannot be built in this environment (Eigen, MyCEL, SerAr,
Boost and GSL are absent), so the tests are read as text: every TEST_F body is
turned into an ordered list of simple operations (assign a vector, prepare,
call a problem method, expect approximate equality, ...) that
tests/test_oracle_golden.py replays against the oracle.  Fixture parameters
(temperature, radius, K, problem settings, Euler angles) are read from the
matching fixture headers.

Usage (only where the reference sources are present):
    python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import json
import math
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "reference_unit_tests.json"

# (test source, fixture header, problem kind) relative to the reference root
SOURCES = [
    ("Tests/Neel_Problem_Test/Test_Problem_Neel.cpp", "Tests/Neel_Problem_Test/Test_Problem_Neel.h", "neel"),
    ("Tests/Neel_Spherical_Test/Test_Neel_Spherical_Problem.cpp",
     "Tests/Neel_Spherical_Test/Test_Neel_Spherical_Problem.h", "neel_spherical"),
    ("Tests/BrownAndNeel_Relaxation_Test/Test_BrownAndNeel_Relaxation.cpp",
     "Tests/BrownAndNeel_Relaxation_Test/Test_BrownAndNeel_Relaxation.h", "brown_neel"),
    ("Tests/NeelSpherical_BrownEuler_Relaxation_Test/Test_NeelSpherical_BrownEuler_Problem.cpp",
     "Tests/NeelSpherical_BrownEuler_Relaxation_Test/Test_NeelSpherical_BrownEuler_Problem.h", "brown_neel_euler"),
    ("Tests/Neel_Problem_Test/Test_Uniaxial_Anisotropy.cpp", "Tests/Neel_Problem_Test/Test_Uniaxial_Anisotropy.h",
     "uniaxial"),
    ("Tests/Neel_Problem_Test/Test_ParamCalc_Neel.cpp", "Tests/Neel_Problem_Test/Test_ParamCalc_Neel.h", "param_neel"),
]

PI_PAT = re.compile(r"math::(?:constants|coordinates)::pi<Precision>")
TWO_PI_PAT = re.compile(r"math::constants::two_pi<Precision>")
EPS_PAT = re.compile(r"std::numeric_limits<Precision>::epsilon\(\)")
NUM_EXPR = re.compile(r"^[0-9eE+\-*/. ()piPIepsTWO_]*$")


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return "\n".join(line.split("//", 1)[0] for line in text.splitlines())


def evaluate(expr: str):
    e = PI_PAT.sub("pi", expr)
    e = TWO_PI_PAT.sub("TWO_PI", e)
    e = EPS_PAT.sub("eps", e)
    e = e.strip()
    if not NUM_EXPR.match(e.replace(" ", "")):
        return None
    try:
        return float(eval(e, {"__builtins__": {}}, {"pi": math.pi, "TWO_PI": 2 * math.pi,
                                                     "eps": sys.float_info.epsilon}))
    except Exception:  # noqa: BLE001 - anything unparsable is reported as None
        return None


def split_args(s: str) -> list[str]:
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def test_blocks(text: str):
    """Yield (fixture, name, body, line) for every TEST_F in text."""
    for m in re.finditer(r"TEST_F\(\s*(\w+)\s*,\s*(\w+)\s*\)", text):
        i = text.index("{", m.end())
        depth, j = 0, i
        while True:
            if text[j] == "{":
                depth += 1
            elif text[j] == "}":
                depth -= 1
                if depth == 0:
                    break
            j += 1
        yield m.group(1), m.group(2), text[i + 1:j], text.count("\n", 0, m.start()) + 1


KNOWN_CALLS = {
    "getDeterministicVector", "getStochasticMatrix", "getDrift", "getJacobiDeterministic",
    "getJacobiStochastic", "getStochasticMatrixSimplified", "getStratonovichtoItoSimplified",
}


def parse_statement(st: str):
    st = st.strip()
    if not st:
        return None
    m = re.match(r"^(\w+)\s*<<\s*(\w+)$", st)
    if m and evaluate(m.group(2)) is None:
        return {"op": "copy", "var": m.group(1), "src": m.group(2)}
    m = re.match(r"^(\w+)\s*<<\s*(.+)$", st, flags=re.S)
    if m:
        vals = [evaluate(x) for x in split_args(m.group(2))]
        return {"op": "assign", "var": m.group(1), "values": vals}
    m = re.match(r"^(?:const\s+)?(?:Vec\dD|Vec3D|Vec2D|Vec5D|Vec6D)\s+(\w+)\s*\((.*)\)$", st, flags=re.S)
    if m:
        args = split_args(m.group(2))
        if len(args) == 1 and re.match(r"^\w+$", args[0]) and evaluate(args[0]) is None:
            return {"op": "copy", "var": m.group(1), "src": args[0]}
        return {"op": "assign", "var": m.group(1), "values": [evaluate(x) for x in args]}
    m = re.match(r"^(\w+)\((\d+)\)\s*=\s*(.+)$", st)
    if m:
        return {"op": "setitem", "var": m.group(1), "index": int(m.group(2)), "value": evaluate(m.group(3))}
    m = re.match(r"^(?:const\s+)?Precision\s+(\w+)\s*=\s*(.+)$", st)
    if m:
        return {"op": "scalar", "var": m.group(1), "value": evaluate(m.group(2))}
    m = re.match(r"^constexpr\s+auto\s+(\w+)\s*=\s*(.+)$", st)
    if m:
        return {"op": "scalar", "var": m.group(1), "value": evaluate(m.group(2))}
    m = re.match(r"^(\w+)\s*\*=\s*(\w+)$", st)
    if m:
        return {"op": "scale", "var": m.group(1), "by": m.group(2)}
    m = re.match(r"^math::approximateJacobian\((\w+)\s*,\s*(\w+)\s*,\s*(\w+)\s*,\s*(\w+)\)$", st)
    if m:
        return {"op": "approx_jacobian", "func": m.group(1), "x": m.group(2), "dx": m.group(3), "out": m.group(4)}
    m = re.match(r"^finishJacobiCalculations\((\w+)\)$", st)
    if m:
        return {"op": "finish_jacobi", "var": m.group(1)}
    m = re.match(r"^prepareJacobiCalculations\((\w+)\)$", st)
    if m:
        return {"op": "prepare_jacobi", "var": m.group(1)}
    m = re.match(r"^(\w+)\.normalize\(\)$", st)
    if m:
        return {"op": "normalize", "var": m.group(1)}
    m = re.match(r"^(\w+)\s*=\s*math::coordinates::Wrap2DSphericalCoordinates\((\w+)\)$", st)
    if m:
        return {"op": "wrap", "var": m.group(1), "src": m.group(2)}
    m = re.match(r"^(?:Vec\dD|auto)\s+(\w+)\s*=\s*(\w+)$", st)
    if m:
        return {"op": "copy", "var": m.group(1), "src": m.group(2)}
    m = re.match(r"^(\w+)\s*=\s*(\w+)$", st)
    if m:
        return {"op": "copy", "var": m.group(1), "src": m.group(2)}
    m = re.match(r"^prepareCalculations\((\w+)\)$", st)
    if m:
        return {"op": "prepare", "var": m.group(1)}
    m = re.match(r"^finishCalculations\((\w+)\)$", st)
    if m:
        return {"op": "finish", "var": m.group(1)}
    m = re.match(r"^(?:const\s+)?(?:auto&?|[\w:<>]+)\s+(\w+)\s*=\s*(?:mProblem\.)?(\w+)\((.*)\)$", st, flags=re.S)
    if m and m.group(2) in KNOWN_CALLS:
        return {"op": "call", "out": m.group(1), "fn": m.group(2), "args": split_args(m.group(3))}
    m = re.match(r"^(\w+)\s*=\s*(?:mProblem\.)?(\w+)\((.*)\)$", st, flags=re.S)
    if m and m.group(2) in KNOWN_CALLS:
        return {"op": "call", "out": m.group(1), "fn": m.group(2), "args": split_args(m.group(3))}
    m = re.match(r"^EXPECT_(TRUE|FALSE)\((!?)([\w.]*isRotated)\)$", st)
    if m:
        val = (m.group(1) == "TRUE") != (m.group(2) == "!")
        return {"op": "expect_flag", "flag": m.group(3), "value": val}
    m = re.match(r"^EXPECT_TRUE\((\w+)\.isApprox\((\w+)(?:\s*,\s*(.+))?\)\)$", st)
    if m:
        tol = evaluate(m.group(3)) if m.group(3) else 1e-12  # Eigen dummy_precision<double>
        return {"op": "expect_approx", "a": m.group(1), "b": m.group(2), "tol": tol}
    m = re.match(r"^EXPECT_TRUE\(\(*\s*\((\w+)\s*-\s*(\w+)\)\.norm\(\)\s*<\s*([^)]+)\)*$", st)
    if m:
        return {"op": "expect_normdiff", "a": m.group(1), "b": m.group(2), "tol": evaluate(m.group(3))}
    m = re.match(r"^EXPECT_DOUBLE_EQ\((\w+)\((\d+)\)\s*,\s*(\w+)\((\d+)\)\)$", st)
    if m:
        return {"op": "expect_double_eq", "a": m.group(1), "ia": int(m.group(2)), "b": m.group(3),
                "ib": int(m.group(4))}
    return None


def parse_body(body: str):
    ops = []
    # the wrap-negative loops after finishCalculations in the Euler tests
    loop = re.compile(r"for\s*\(int i = (\d+); i < (\d+); i\+\+\)\s*\{\s*if\s*\((\w+)\(i\) < 0\)\s*\{\s*\w+\(i\)\s*="
                      r"\s*math::constants::two_pi<Precision>\s*\+\s*\w+\(i\);\s*\}\s*\}")
    funcs = []
    lam = re.compile(r"const\s+auto\s+(\w+)\s*=\s*\[&\]\s*\(auto\s*&\s*val\)\s*\{(.*?)\};", flags=re.S)
    for m in lam.finditer(body):
        ret = re.search(r"return\s+(.*?);", m.group(2), flags=re.S).group(1)
        funcs.append({"op": "define_func", "name": m.group(1), "expr": " ".join(ret.split())})
    body = lam.sub(";", body)
    ops.extend(funcs)
    pieces, last = [], 0
    for m in loop.finditer(body):
        pieces.append(("code", body[last:m.start()]))
        pieces.append(("loop", m))
        last = m.end()
    pieces.append(("code", body[last:]))
    for kind, item in pieces:
        if kind == "loop":
            ops.append({"op": "wrap_negative", "var": item.group(3), "lo": int(item.group(1)),
                        "hi": int(item.group(2))})
            continue
        # drop the diagnostic if-blocks that only print
        code = re.sub(r"if\s*\(![^{;]*\)\s*\{[^{}]*\}", "", item)
        for st in code.replace("{", ";").replace("}", ";").split(";"):
            op = parse_statement(" ".join(st.split()))
            if op is not None:
                ops.append(op)
    return ops


def parse_fixture(text: str):
    text = strip_comments(text)
    fx = {}
    for m in re.finditer(r"const\s+Precision\s+(\w+)\s*=\s*([^;]+);", text):
        fx[m.group(1)] = evaluate(m.group(2))
    settings = {}
    for m in re.finditer(r"ProbSet\.(m\w+)\s*=\s*([^;]+);", text):
        v = m.group(2).strip()
        settings[m.group(1)] = True if v == "true" else False if v == "false" else evaluate(v)
    fx["settings"] = settings
    m = re.search(r"Orientation\s*<<\s*([^;]+);", text) or re.search(r"Vec3D\s+Orientation\(([^)]*)\)", text)
    if m:
        fx["orientation"] = [evaluate(x) for x in split_args(m.group(1))]
    return fx


def main(ref_root: Path) -> None:
    doc = {"generated_by": "tests/golden/make_golden.py", "reference_root_relative": True, "suites": []}
    for src, hdr, kind in SOURCES:
        text = (ref_root / src).read_text(encoding="latin-1")
        clean = strip_comments(text)
        fixture = parse_fixture((ref_root / hdr).read_text(encoding="latin-1"))
        tests = []
        for fixname, name, body, _ in test_blocks(clean):
            line = next(i + 1 for i, l in enumerate(text.splitlines())
                        if re.search(rf"TEST_F\(\s*{fixname}\s*,\s*{name}\s*\)", l) and not l.strip().startswith("//"))
            tests.append({"name": name, "line": line, "ops": parse_body(body)})
        doc["suites"].append({"kind": kind, "source": src, "fixture_header": hdr, "fixture": fixture,
                              "tests": tests})
    OUT.write_text(json.dumps(doc, indent=1))
    print(f"wrote {OUT} ({sum(len(s['tests']) for s in doc['suites'])} tests)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the StochasticPhysics source tree>")
    main(Path(sys.argv[1]))
