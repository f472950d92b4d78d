"""Extract SimiLie's known-answer tests for the DEC path into JSON fixtures.

Run in a checkout that has the reference sources (path in SIMILIE_REF or the
first argument).  It reads the reference's GTest files as text and writes:

  derivative_kat.json   every EXPECT_EQ of tests/exterior/derivative.cpp:
                        fixture N, layout, input/output rank, dims, node,
                        output component (lexicographic index) and value.
  exterior_kat.json     scalar known answers of codifferential.cpp,
                        hodge_star.cpp and laplacian.cpp (tolerances too).

The fixtures are committed; the tests never need the reference at run time.
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIMILIE_REF")
if not REF:
    sys.exit("usage: make_golden.py <path of a SimiLie checkout>  (or set SIMILIE_REF)")
HERE = os.path.dirname(os.path.abspath(__file__))

DIM_TAGS = {"DDimT": "T", "DDimX": "X", "DDimY": "Y", "DDimZ": "Z"}


def rank_of(index_expr):
    """Rank of a test index type: AntisymmetricIndex<...> counts its members,
    a bare natural index (Mu2) is a 1-form."""
    index_expr = index_expr.strip()
    m = re.match(r"sil::tensor::TensorAntisymmetricIndex<(.*)>$", index_expr)
    if m:
        inner = m.group(1).strip()
        return 0 if inner == "" else len([s for s in inner.split(",") if s.strip()])
    if index_expr.startswith("sil::tensor::TensorNaturalIndex<>"):
        return 0
    return 1


def parse_derivative(path):
    src = open(path).read()
    tests = []
    # split into TEST blocks
    for m in re.finditer(r"TEST\(ExteriorDerivative, (\w+)\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        if "Spects" in name:
            continue  # handled separately below
        # each test_derivative<...>() call binds a variable name
        calls = list(re.finditer(
            r"auto \[(\w+), (\w+)\]\s*=\s*test_derivative<\s*(\d+),\s*(true|false),\s*(.*?)>\(\);", body, re.S))
        for ci, c in enumerate(calls):
            var = c.group(2)
            n_fix = int(c.group(3))
            coalescent = c.group(4) == "true"
            args = c.group(5)
            # split top-level template args
            depth, cur, parts = 0, "", []
            for ch in args:
                if ch == "<":
                    depth += 1
                elif ch == ">":
                    depth -= 1
                if ch == "," and depth == 0:
                    parts.append(cur.strip())
                    cur = ""
                else:
                    cur += ch
            parts.append(cur.strip())
            in_index, out_index, ddims = parts[0], parts[1], parts[2:]
            dims = [DIM_TAGS[d] for d in ddims]
            k_in = rank_of(in_index)
            k_out = rank_of(out_index)
            start = c.end()
            stop = calls[ci + 1].start() if ci + 1 < len(calls) else len(body)
            checks = []
            for e in re.finditer(
                    r"EXPECT_EQ\(\s*" + var + r"\(\s*ddc::DiscreteElement<[^>]*>\s*\{([^}]*)\},\s*"
                    + var + r"\.accessor\(\)\.access_element<([^>]*)>\(\)\),\s*([-0-9.]+)\)",
                    body[start:stop]):
                node = [int(v) for v in e.group(1).split(",")]
                comp_tags = [t.strip() for t in e.group(2).split(",")]
                comp_dims = sorted(dims.index(t) for t in comp_tags)
                value = float(e.group(3))
                checks.append({"node": node, "comp_dims": comp_dims, "value": value})
            tests.append({"name": name, "variant": ci, "N": n_fix, "component_first": coalescent,
                          "dims": dims, "k_in": k_in, "k_out": k_out, "checks": checks,
                          "source": f"tests/exterior/derivative.cpp ({name})"})
    # 2D rotational with a spectator lattice dim and a spectator tensor index
    m = re.search(r"TEST\(ExteriorDerivative, 2DRotationalWithSpects\)\s*\{(.*?)\n\}", src, re.S)
    if m:
        body = m.group(1)
        checks = []
        for e in re.finditer(r"ddc::DiscreteElement<DDimX, DDimY>\s*\{([^}]*)\},.*?access_element<X, Y>\(\)\),\s*([-0-9.]+)\)",
                             body, re.S):
            node = [int(v) for v in e.group(1).split(",")]
            checks.append({"node": node, "comp_dims": [0, 1], "value": float(e.group(2))})
        tests.append({"name": "2DRotationalWithSpects", "variant": 0, "N": 3, "component_first": True,
                      "dims": ["X", "Y"], "k_in": 1, "k_out": 2, "checks": checks,
                      "spectators": {"lattice": 3, "index": 10},
                      "out_extent": [3, 2, 2],
                      "source": "tests/exterior/derivative.cpp (2DRotationalWithSpects)"})
    return tests


def parse_exterior(ref):
    out = {}
    cod = open(os.path.join(ref, "tests/exterior/codifferential.cpp")).read()
    m = re.search(r"ddc::DiscreteVector<DDimX, DDimY> nb_cells\((\d+), (\d+)\)", cod)
    lo = re.search(r"lower_bounds\(([-0-9.]+), ([-0-9.]+)\)", cod)
    hi = re.search(r"upper_bounds\(([-0-9.]+), ([-0-9.]+)\)", cod)
    tol = re.search(r"expected_codifferential,\s*([0-9.e-]+)\)", cod)
    n = int(m.group(1))
    out["codifferential_2d_1form"] = {
        "points": n, "lower": float(lo.group(1)), "upper": float(hi.group(1)),
        "cochain_scale": (float(hi.group(1)) - float(lo.group(1))) / n,
        "expected": -(n - 1) / n - (n - 1) / n, "tolerance": float(tol.group(1)),
        "check_region": "interior (first and last node removed per axis)",
        "source": "tests/exterior/codifferential.cpp:38-118"}
    hs_all = open(os.path.join(ref, "tests/exterior/hodge_star.cpp")).read()
    hs = re.search(r"TEST\(DiscreteHodgeStar, Metric3D\)\s*\{(.*?)\n\}", hs_all, re.S).group(1)
    metric = {}
    for e in re.finditer(r"metric\(elem, metric\.accessor\(\)\.access_element<([XYZ]), ([XYZ])>\(\)\) = ([0-9.]+);", hs):
        metric[e.group(1) + e.group(2)] = float(e.group(3))
    form = re.search(r"form\(elem, form\.accessor\(\)\.access_element<X, Y>\(\)\) = ([0-9.]+);", hs)
    expect = re.search(r"access_element<Z>\(\)\),\s*([0-9.]+) \* std::sqrt\(([0-9.]+) / ([0-9.]+)\)\)", hs)
    out["hodge_star_3d_metric"] = {
        "metric": metric, "lower": 0.0, "upper": 2.0, "points": 2,
        "form_xy": float(form.group(1)),
        "expected_dual_z": float(expect.group(1)) * (float(expect.group(2)) / float(expect.group(3))) ** 0.5,
        "expected_round_trip_xy": float(form.group(1)),
        "tolerance_ulps": 4,
        "source": "tests/exterior/hodge_star.cpp:66-181"}
    lap = open(os.path.join(ref, "tests/exterior/laplacian.cpp")).read()
    gates = []
    for m in re.finditer(r"TEST\(Laplacian, (\w+)\)\s*\{(.*?)\n\}", lap, re.S):
        name, body = m.group(1), m.group(2)
        cells = re.search(r"nb_cells\(([0-9, ]+)\)", body)
        alpha = re.search(r"double const alpha = ([0-9.]+);", body)
        R = re.search(r"double const R = ([0-9.]+);", body)
        tols = re.findall(r"EXPECT_NEAR\([^;]*?,\s*([01])\.,\s*([0-9.e-]+)\)", body, re.S)
        gates.append({"name": name, "points": int(cells.group(1).split(",")[0]),
                      "alpha": float(alpha.group(1)) if alpha else None, "R": float(R.group(1)) if R else None,
                      "tolerance": float(tols[0][1]) if tols else None,
                      "source": f"tests/exterior/laplacian.cpp ({name})"})
    out["laplacian_gates"] = gates
    return out


def main():
    der = parse_derivative(os.path.join(REF, "tests/exterior/derivative.cpp"))
    with open(os.path.join(HERE, "derivative_kat.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "tests": der}, f, indent=1)
    ext = parse_exterior(REF)
    with open(os.path.join(HERE, "exterior_kat.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", **ext}, f, indent=1)
    print(f"{sum(len(t['checks']) for t in der)} derivative checks in {len(der)} cases")


if __name__ == "__main__":
    main()
