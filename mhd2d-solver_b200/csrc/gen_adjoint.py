"""Writes mhd_adjoint_gen.cuh: reverse-mode (adjoint) code of the ENO-Roe
interface algebra with every branch frozen.

    python gen_adjoint.py > mhd_adjoint_gen.cuh

The formulas below restate the midpoint eigen-system of getEigensF
(spatialmethodeno.cpp:288-571; the same arithmetic as mhd_eigen.cuh) and the
physical fluxes of updateFluxes (spatialmethodeno.cpp:89-127) as straight
-line programs.  Each program is differentiated in reverse mode: for every
statement t = f(x, y, ...) in reverse order the generator emits
    x_b += (df/dx) * t_b, ...
walking the expression tree (sum, difference, product, quotient, square
root, negation).  Clamps and degenerate-case branches are frozen: a
statement whose frozen condition held in the forward evaluation passes no
adjoint on (its value was a constant there), and neither does a statement
whose adjoint is exactly zero (degenerate midpoints, e.g. a pressure clamped
to zero, give infinite partial derivatives that a zero seed must not turn
into NaN).  The derivative of sqrt(v) is
taken as 0 at v = 0, the one-sided convention of a frozen branch (it only
arises where the forward value is exactly zero, e.g. B_x = 0).
"""
import ast
import re
import sys

# --------------------------------------------------------------------------
# Expression-tree reverse mode


def _src(node):
    return ast.unparse(node)


def acc(target, coef):
    """The statement target += coef.  A coefficient that is a product P * Q
    is accumulated with one fused multiply-add, target = fma(P, Q, target):
    one rounding instead of two, and one FP64 instruction."""
    try:
        node = ast.parse(coef, mode="eval").body
    except SyntaxError:
        node = None
    if isinstance(node, ast.BinOp) and isinstance(node.op, ast.Mult):
        # ast.unparse writes a double negation as "--", a C decrement
        left, right = (re.sub(r"-(?=-)", "- ", _src(x)) for x in (node.left, node.right))
        return f"{target} = fma({left}, {right}, {target});"
    return f"{target} += {coef};"


class Rcp:
    """Reciprocals of the denominators met in one reverse sweep: each distinct
    denominator is divided once (rcpN = 1 / d) and the adjoints multiply."""

    def __init__(self, prefix="rcp"):
        self.map = {}
        self.known = set()  # names that already hold the reciprocal
        self.prefix = prefix

    def name(self, src):
        if src not in self.map:
            self.map[src] = f"{self.prefix}{len(self.map)}"
        return self.map[src]

    def alias(self, src, name):
        """`name` is 1 / src already (a statement t = 1.0 / (src))."""
        self.map[src] = name
        self.known.add(name)

    def defs(self, indent, names=None):
        return [f"{indent}[[maybe_unused]] const double {n} = "
                f"1.0 / ({c_expr(src, names) if names else src});"
                for src, n in self.map.items() if n not in self.known]


def _rev(node, seed, out, rcp=None):
    """Append (variable, coefficient * seed) pairs for the leaves of `node`."""
    if isinstance(node, ast.Name):
        out.append((node.id, seed))
    elif isinstance(node, ast.Constant):
        pass
    elif isinstance(node, ast.UnaryOp):
        if isinstance(node.op, ast.USub):
            _rev(node.operand, f"-({seed})", out, rcp)
        elif isinstance(node.op, ast.UAdd):
            _rev(node.operand, seed, out, rcp)
        else:
            raise ValueError(ast.dump(node))
    elif isinstance(node, ast.BinOp):
        a, b = node.left, node.right
        if isinstance(node.op, ast.Add):
            _rev(a, seed, out, rcp)
            _rev(b, seed, out, rcp)
        elif isinstance(node.op, ast.Sub):
            _rev(a, seed, out, rcp)
            _rev(b, f"-({seed})", out, rcp)
        elif isinstance(node.op, ast.Mult):
            _rev(a, f"({seed}) * ({_src(b)})", out, rcp)
            _rev(b, f"({seed}) * ({_src(a)})", out, rcp)
        elif isinstance(node.op, ast.Div):
            if rcp is None:
                _rev(a, f"({seed}) / ({_src(b)})", out, rcp)
                _rev(b, f"-({seed}) * ({_src(a)}) / (({_src(b)}) * ({_src(b)}))", out, rcp)
            else:
                r = rcp.name(_src(b))
                _rev(a, f"({seed}) * {r}", out, rcp)
                _rev(b, f"-({seed}) * ({_src(a)}) * {r} * {r}", out, rcp)
        else:
            raise ValueError(ast.dump(node))
    elif isinstance(node, ast.Call) and node.func.id == "sqrt":
        _rev(node.args[0], f"({seed}) * inv2sqrt({_src(node.args[0])})", out, rcp)
    else:
        raise ValueError(ast.dump(node))


def reverse_of(expr, seed, rcp=None):
    out = []
    _rev(ast.parse(expr, mode="eval").body, seed, out, rcp)
    return out


def c_expr(expr, names):
    """Python expression -> C expression, renaming variables."""
    tree = ast.parse(expr, mode="eval").body

    class R(ast.NodeTransformer):
        def visit_Name(self, n):
            return ast.copy_location(ast.Name(id=names.get(n.id, n.id), ctx=n.ctx), n)

    return ast.unparse(R().visit(tree))


# --------------------------------------------------------------------------
# Midpoint state and eigen-system scalars (getEigensF; midpoint() of
# mhd_eigen.cuh).  Statements: (target, expr), (target, expr, frozen_cond,
# frozen_value) or ("#", raw C line).  U1 -> a0..a7 (a2_ for U1[2]), U2 -> b0..b7.

MID = [
    ("r", "0.5 * (a0 + b0)"),
    ("u", "0.5 * (a1 / a0 + b1 / b0)"),
    ("v", "0.5 * (a2_ / a0 + b2 / b0)"),
    ("w", "0.5 * (a3 / a0 + b3 / b0)"),
    ("bx", "0.5 * (a4 + b4)"),
    ("by", "0.5 * (a5 + b5)"),
    ("bz", "0.5 * (a6 + b6)"),
    ("uu", "u * u + v * v + w * w"),
    ("bb", "bx * bx + by * by + bz * bz"),
    ("mml", "a1 * a1 + a2_ * a2_ + a3 * a3"),
    ("bbl", "a4 * a4 + a5 * a5 + a6 * a6"),
    ("mmr", "b1 * b1 + b2 * b2 + b3 * b3"),
    ("bbr", "b4 * b4 + b5 * b5 + b6 * b6"),
    ("ptl", "gm1 * (a7 - 0.5 * mml / a0 - 0.5 * bbl) + 0.5 * bbl"),
    ("ptr", "gm1 * (b7 - 0.5 * mmr / b0 - 0.5 * bbr) + 0.5 * bbr"),
    ("pt", "0.5 * (ptl + ptr)"),
    ("p", "pt - 0.5 * bb", "p < 0.0", "0.0"),
    ("a2", "gm * p / r", "a2 < 0.0", "0.0"),
    ("a", "sqrt(a2)"),
    ("ca2", "bx * bx / r"),
    ("ca", "sqrt(ca2)"),
    ("c2", "0.5 * (bb / r + a2)"),
    ("ct", "c2 * c2 - a2 * ca2", "ct < 0.0", "0.0"),
    ("sct", "sqrt(ct)"),
    ("cs2", "c2 - sct", "cs2 < 0.0", "SMALL"),
    ("cf2", "c2 + sct", "cf2 < 0.0", "SMALL"),
    ("cs", "sqrt(cs2)"),
    ("cf", "sqrt(cf2)"),
    ("rr", "sqrt(r)"),
    ("bp2", "by * by + bz * bz"),
    ("#", "const bool deg = (bp2 < SMALL) && (fabs(ca2 - a2) < SMALL);"),
    ("af2", "(cf2 - ca2) / (cf2 - cs2)", "deg || af2 < 0.0", "deg ? 1.0 : 0.0"),
    ("as2", "(cf2 - a2) / (cf2 - cs2)", "deg || as2 < 0.0", "deg ? 1.0 : 0.0"),
    ("af", "sqrt(af2)"),
    ("as_", "sqrt(as2)"),
    ("sbp", "sqrt(bp2)", "!(bp2 > SMALL)", "1.0"),
    ("bty", "by / sbp", "!(bp2 > SMALL)", "G.rs2"),
    ("btz", "bz / sbp", "!(bp2 > SMALL)", "G.rs2"),
    ("th1", "1.0 / (af2 * a2 * (cf2 - g21 * a2) + as2 * cf2 * (cs2 - g21 * a2))"),
    ("th2", "1.0 / (sb * af2 * cf * a + sb * as2 * cs * ca)"),
    ("vb", "bty * v + btz * w"),
]
MID_INPUTS = [f"a{k}" if k != 2 else "a2_" for k in range(8)] + [f"b{k}" for k in range(8)]
# Mid fields whose adjoints the row code produces
MID_FIELDS = ["u", "v", "w", "uu", "a2", "a", "ca2", "ca", "cs2", "cs", "cf2", "cf", "rr", "af2",
              "af", "as2", "as_", "bty", "btz", "th1", "th2", "vb"]

# --------------------------------------------------------------------------
# Eigenvector rows (spatialmethodeno.cpp:392-568 with the continuity sign
# factors): sb = sgn(Bx), fcf = cffactor, fcs = csfactor, all +-1.

L0 = {
    0: "fcf * (0.25 * th1 * af * a2 * uu + 0.5 * th2 * (sb * af * a * u - as_ * cs * vb))",
    1: "fcf * (-0.5 * th1 * af * a2 * u - sb * 0.5 * th2 * af * a)",
    2: "fcf * (-0.5 * th1 * af * a2 * v + 0.5 * th2 * as_ * bty * cs)",
    3: "fcf * (-0.5 * th1 * af * a2 * w + 0.5 * th2 * as_ * btz * cs)",
    5: "fcf * (0.5 * th1 * as_ * bty * cf * rr * (cs2 - g21 * a2))",
    6: "fcf * (0.5 * th1 * as_ * btz * cf * rr * (cs2 - g21 * a2))",
    7: "fcf * (0.5 * th1 * af * a2)",
}
L6 = dict(L0)
L6.update({
    0: "fcf * (0.25 * th1 * af * a2 * uu - 0.5 * th2 * (sb * af * a * u - as_ * cs * vb))",
    1: "fcf * (-0.5 * th1 * af * a2 * u + sb * 0.5 * th2 * af * a)",
    2: "fcf * (-0.5 * th1 * af * a2 * v - 0.5 * th2 * as_ * bty * cs)",
    3: "fcf * (-0.5 * th1 * af * a2 * w - 0.5 * th2 * as_ * btz * cs)",
})
L1 = {0: "sb * (-0.5 * (btz * v - bty * w))", 2: "sb * (0.5 * btz)", 3: "sb * (-0.5 * bty)",
      5: "0.5 * btz * rr", 6: "-0.5 * bty * rr"}
L5 = {0: "sb * (0.5 * (btz * v - bty * w))", 2: "sb * (-0.5 * btz)", 3: "sb * (0.5 * bty)",
      5: "0.5 * btz * rr", 6: "-0.5 * bty * rr"}
L2 = {
    0: "fcs * (0.25 * th1 * as_ * cf2 * uu + 0.5 * th2 * (sb * as_ * ca * u + af * cf * vb))",
    1: "fcs * (-0.5 * th1 * as_ * cf2 * u - sb * 0.5 * th2 * as_ * ca)",
    2: "fcs * (-0.5 * th1 * as_ * cf2 * v - 0.5 * th2 * af * bty * cf)",
    3: "fcs * (-0.5 * th1 * as_ * cf2 * w - 0.5 * th2 * af * btz * cf)",
    5: "fcs * (-0.5 * th1 * af * bty * cf * rr * (cf2 - g21 * a2))",
    6: "fcs * (-0.5 * th1 * af * btz * cf * rr * (cf2 - g21 * a2))",
    7: "fcs * (0.5 * th1 * as_ * cf2)",
}
L4 = dict(L2)
L4.update({
    0: "fcs * (0.25 * th1 * as_ * cf2 * uu - 0.5 * th2 * (sb * as_ * ca * u + af * cf * vb))",
    1: "fcs * (-0.5 * th1 * as_ * cf2 * u + sb * 0.5 * th2 * as_ * ca)",
    2: "fcs * (-0.5 * th1 * as_ * cf2 * v + 0.5 * th2 * af * bty * cf)",
    3: "fcs * (-0.5 * th1 * as_ * cf2 * w + 0.5 * th2 * af * btz * cf)",
})
L3 = {0: "1.0 - 0.5 * th1 * uu * (af2 * a2 + as2 * cf2)",
      1: "th1 * (af2 * a2 + as2 * cf2) * u", 2: "th1 * (af2 * a2 + as2 * cf2) * v",
      3: "th1 * (af2 * a2 + as2 * cf2) * w",
      5: "th1 * af * as_ * bty * cf * rr * (cf2 - cs2)",
      6: "th1 * af * as_ * btz * cf * rr * (cf2 - cs2)",
      7: "-th1 * (af2 * a2 + as2 * cf2)"}
LROWS = [L0, L1, L2, L3, L4, L5, L6]

R0 = {0: "fcf * af", 1: "fcf * (af * (u - cf))", 2: "fcf * (af * v + sb * as_ * bty * ca)",
      3: "fcf * (af * w + sb * as_ * btz * ca)", 5: "fcf * (as_ * bty * cf / rr)",
      6: "fcf * (as_ * btz * cf / rr)",
      7: "fcf * (0.5 * af * uu + af * cf2 / g1 - af * cf * u + sb * as_ * ca * vb"
         " + g21 * af * (cf2 - a2))"}
R6 = dict(R0)
R6.update({1: "fcf * (af * (u + cf))", 2: "fcf * (af * v - sb * as_ * bty * ca)",
           3: "fcf * (af * w - sb * as_ * btz * ca)",
           7: "fcf * (0.5 * af * uu + af * cf2 / g1 + af * cf * u - sb * as_ * ca * vb"
              " + g21 * af * (cf2 - a2))"})
R1 = {2: "sb * btz", 3: "-(sb * bty)", 5: "btz / rr", 6: "-bty / rr", 7: "sb * (btz * v - bty * w)"}
R5 = {2: "-(sb * btz)", 3: "sb * bty", 5: "btz / rr", 6: "-bty / rr",
      7: "-(sb * (btz * v - bty * w))"}
R2 = {0: "fcs * as_", 1: "fcs * (as_ * (u - cs))", 2: "fcs * (as_ * v - sb * af * bty * a)",
      3: "fcs * (as_ * w - sb * af * btz * a)", 5: "fcs * (-af * bty * a2 / (cf * rr))",
      6: "fcs * (-af * btz * a2 / (cf * rr))",
      7: "fcs * (0.5 * as_ * uu + as_ * cs2 / g1 - as_ * cs * u - sb * af * a * vb"
         " + g21 * as_ * (cs2 - a2))"}
R4 = dict(R2)
R4.update({1: "fcs * (as_ * (u + cs))", 2: "fcs * (as_ * v + sb * af * bty * a)",
           3: "fcs * (as_ * w + sb * af * btz * a)",
           7: "fcs * (0.5 * as_ * uu + as_ * cs2 / g1 + as_ * cs * u + sb * af * a * vb"
              " + g21 * as_ * (cs2 - a2))"})
R3 = {0: "1.0", 1: "u", 2: "v", 3: "w", 7: "0.5 * uu"}
RROWS = [R0, R1, R2, R3, R4, R5, R6]

# The same rows split by pair: rows k and 6 - k (k = 0, 1, 2) are A + B and
# A - B (left) and C + D and C - D (right).  Row 3 is its own "pair" (A, C).
# The adjoint of both rows of a pair is then one pass over A, B, C, D with
# the seeds lb_k + lb_{6-k} (A), lb_k - lb_{6-k} (B), and likewise for C, D.
PAIRS = [
    (0, 6,
     {0: "fcf * (0.25 * th1 * af * a2 * uu)", 1: "fcf * (-0.5 * th1 * af * a2 * u)",
      2: "fcf * (-0.5 * th1 * af * a2 * v)", 3: "fcf * (-0.5 * th1 * af * a2 * w)",
      5: "fcf * (0.5 * th1 * as_ * bty * cf * rr * (cs2 - g21 * a2))",
      6: "fcf * (0.5 * th1 * as_ * btz * cf * rr * (cs2 - g21 * a2))",
      7: "fcf * (0.5 * th1 * af * a2)"},
     {0: "fcf * (0.5 * th2 * (sb * af * a * u - as_ * cs * vb))",
      1: "fcf * (-(sb * 0.5 * th2 * af * a))", 2: "fcf * (0.5 * th2 * as_ * bty * cs)",
      3: "fcf * (0.5 * th2 * as_ * btz * cs)"},
     {0: "fcf * af", 1: "fcf * (af * u)", 2: "fcf * (af * v)", 3: "fcf * (af * w)",
      5: "fcf * (as_ * bty * cf / rr)", 6: "fcf * (as_ * btz * cf / rr)",
      7: "fcf * (0.5 * af * uu + af * cf2 / g1 + g21 * af * (cf2 - a2))"},
     {1: "fcf * (-(af * cf))", 2: "fcf * (sb * as_ * bty * ca)",
      3: "fcf * (sb * as_ * btz * ca)", 7: "fcf * (-(af * cf * u) + sb * as_ * ca * vb)"}),
    (2, 4,
     {0: "fcs * (0.25 * th1 * as_ * cf2 * uu)", 1: "fcs * (-0.5 * th1 * as_ * cf2 * u)",
      2: "fcs * (-0.5 * th1 * as_ * cf2 * v)", 3: "fcs * (-0.5 * th1 * as_ * cf2 * w)",
      5: "fcs * (-0.5 * th1 * af * bty * cf * rr * (cf2 - g21 * a2))",
      6: "fcs * (-0.5 * th1 * af * btz * cf * rr * (cf2 - g21 * a2))",
      7: "fcs * (0.5 * th1 * as_ * cf2)"},
     {0: "fcs * (0.5 * th2 * (sb * as_ * ca * u + af * cf * vb))",
      1: "fcs * (-(sb * 0.5 * th2 * as_ * ca))", 2: "fcs * (-0.5 * th2 * af * bty * cf)",
      3: "fcs * (-0.5 * th2 * af * btz * cf)"},
     {0: "fcs * as_", 1: "fcs * (as_ * u)", 2: "fcs * (as_ * v)", 3: "fcs * (as_ * w)",
      5: "fcs * (-af * bty * a2 / (cf * rr))", 6: "fcs * (-af * btz * a2 / (cf * rr))",
      7: "fcs * (0.5 * as_ * uu + as_ * cs2 / g1 + g21 * as_ * (cs2 - a2))"},
     {1: "fcs * (-(as_ * cs))", 2: "fcs * (-(sb * af * bty * a))",
      3: "fcs * (-(sb * af * btz * a))", 7: "fcs * (-(as_ * cs * u) - sb * af * a * vb)"}),
    (1, 5,
     {5: "0.5 * btz * rr", 6: "-0.5 * bty * rr"},
     {0: "sb * (-0.5 * (btz * v - bty * w))", 2: "sb * (0.5 * btz)", 3: "sb * (-0.5 * bty)"},
     {5: "btz / rr", 6: "-bty / rr"},
     {2: "sb * btz", 3: "-(sb * bty)", 7: "sb * (btz * v - bty * w)"}),
    (3, 3, L3, {}, R3, {}),
]


def check_pairs():
    """The pair tables restate the rows: L_k = A + B, L_{6-k} = A - B, R likewise."""
    import math
    import random
    rnd = random.Random(5)
    for _ in range(20):
        env = {n: rnd.uniform(0.3, 2.0) for n in MID_FIELDS + ["g21", "g1", "uu"]}
        env.update({"sb": rnd.choice((-1.0, 1.0)), "fcf": rnd.choice((-1.0, 1.0)),
                    "fcs": rnd.choice((-1.0, 1.0)), "sqrt": math.sqrt})
        for k, k2, A, B, C, D in PAIRS:
            for rows, P, Q in ((LROWS, A, B), (RROWS, C, D)):
                for m in range(8):
                    pa = eval(P[m], env) if m in P else 0.0
                    pb = eval(Q[m], env) if m in Q else 0.0
                    for kk, s in ((k, 1.0), (k2, -1.0)):
                        if kk == k2 and s < 0 and k == k2:
                            continue
                        want = eval(rows[kk][m], env) if m in rows[kk] else 0.0
                        got = pa + s * pb
                        assert abs(got - want) <= 1e-12 * (1.0 + abs(want)), (k, kk, m, got, want)

# --------------------------------------------------------------------------
# Physical x flux of one cell (updateFluxes); q0..q7 the conserved state.

FLUX = [
    ("fu", "q1 / q0"), ("fv", "q2 / q0"), ("fw", "q3 / q0"),
    ("fuu", "fu * fu + fv * fv + fw * fw"),
    ("fub", "fu * q4 + fv * q5 + fw * q6"),
    ("fbb", "q4 * q4 + q5 * q5 + q6 * q6"),
    ("fp", "gm1 * (q7 - 0.5 * q0 * fuu - 0.5 * fbb)"),
    ("fpt", "fp + 0.5 * fbb"),
]
FLUX_OUT = {0: "q1", 1: "q1 * fu - q4 * q4 + fpt", 2: "q2 * fu - q4 * q5", 3: "q3 * fu - q4 * q6",
            5: "q5 * fu - q4 * fv", 6: "q6 * fu - q4 * fw", 7: "(q7 + fpt) * fu - q4 * fub"}

# --------------------------------------------------------------------------
# Code emission

MID_NAMES = {f: f"e.{'as' if f == 'as_' else f}" for f in MID_FIELDS}
MID_NAMES.update({"g21": "G.g21", "g1": "G.g1"})
CONSTS = ("gm", "gm1", "g21", "sb", "g1", "SMALL", "fcf", "fcs")


def emit_pairs():
    o = []
    o.append("// Adds the adjoint of rows k and 6 - k of the pair pi (k = 0, 2, 1, 3 for")
    o.append("// pi = 0..3) to mb: LS = lb_k + lb_{6-k}, LD = lb_k - lb_{6-k} (left rows,")
    o.append("// columns 0-3, 5-7 in slots 0-6), and right-row seeds (fS +- fD) * lF.")
    o.append("__device__ __forceinline__ void pair_adjoint(const Mid& e, const Gas& G, int pi,")
    o.append("                                             const double* LS, const double* LD,")
    o.append("                                             double fS, double fD,")
    o.append("                                             const double* lF, MidBar& mb) {")
    o.append("  const double sb = (e.sbxm ? -1.0 : 1.0), fcf = (e.fcfm ? -1.0 : 1.0),")
    o.append("               fcs = (e.fcsm ? -1.0 : 1.0);")
    o.append("  (void)fcf; (void)fcs; (void)sb;")
    o.append("  switch (pi) {")
    for pi, (k, k2, A, B, C, D) in enumerate(PAIRS):
        o.append(f"    case {pi}: {{  // rows {k} and {k2}")
        rcp = Rcp()
        body = []
        for table, seed_of in ((A, lambda m: f"LS[{m if m < 4 else m - 1}]"),
                               (B, lambda m: f"LD[{m if m < 4 else m - 1}]"),
                               (C, lambda m: f"rs{m}"), (D, lambda m: f"rd{m}")):
            for m, expr in sorted(table.items()):
                seed = seed_of(m)
                lines = []
                for var, coef in reverse_of(expr, seed, rcp):
                    if var in CONSTS:
                        continue
                    assert var in MID_FIELDS, var
                    field = "as" if var == "as_" else var
                    lines.append("        " + acc(f"mb.{field}", c_expr(coef, MID_NAMES)))
                if not lines:
                    continue
                if seed.startswith("rs") or seed.startswith("rd"):
                    src = "fS" if seed.startswith("rs") else "fD"
                    body.append(f"      {{ const double {seed} = {src} * lF[{m}];")
                    body.append(f"      if ({seed} != 0.0) {{")
                    body.extend(lines)
                    body.append("      } }")
                else:
                    body.append(f"      if ({seed} != 0.0) {{")
                    body.extend(lines)
                    body.append("      }")
        o.extend(rcp.defs("      ", MID_NAMES))
        o.extend(body)
        o.append("      break;")
        o.append("    }")
    o.append("    default:")
    o.append("      break;")
    o.append("  }")
    o.append("}")
    return o


def emit_program(name, decl, stmts, inputs, prologue, seeds, epilogue, subst=None):
    """Forward sweep (values, frozen-branch flags) then reverse sweep.  subst
    maps a target to an expression that already holds its (final) value; its
    frozen flag, if any, must not depend on the target itself."""
    subst = subst or {}
    o = [f"__device__ __forceinline__ void {name}({', '.join(decl)}) {{"]
    o.extend(prologue)
    targets = []
    for st in stmts:
        if st[0] == "#":
            o.append("  " + st[1])
            continue
        t, expr = st[0], st[1]
        targets.append(t)
        if t in subst:
            o.append(f"  [[maybe_unused]] double {t} = {subst[t]};")
            if len(st) > 2:
                assert not re.search(r"\b" + t + r"\b", st[2]), t
                o.append(f"  const bool {t}_fz = {st[2]};")
            continue
        o.append(f"  [[maybe_unused]] double {t} = {expr};")
        if len(st) > 2:
            o.append(f"  const bool {t}_fz = {st[2]};")
            o.append(f"  if ({t}_fz) {t} = {st[3]};")
    rcp = Rcp()
    for st in stmts:
        if st[0] == "#":
            continue
        node = ast.parse(st[1], mode="eval").body
        if (isinstance(node, ast.BinOp) and isinstance(node.op, ast.Div)
                and isinstance(node.left, ast.Constant) and node.left.value == 1.0):
            rcp.alias(_src(node.right), st[0])
    rev = []
    for st in reversed(stmts):
        if st[0] == "#":
            continue
        t, expr = st[0], st[1]
        lines = []
        for var, coef in reverse_of(expr, f"{t}_b", rcp):
            if var in CONSTS:
                continue
            lines.append("    " + acc(f"{var}_b", coef))
        if not lines:
            continue
        rev.append(f"  if (!{t}_fz && {t}_b != 0.0) {{" if len(st) > 2 else f"  if ({t}_b != 0.0) {{")
        rev.extend(lines)
        rev.append("  }")
    o.append("  // reverse sweep (one division per distinct denominator)")
    o.extend(rcp.defs("  "))
    for v in targets + inputs:
        o.append(f"  double {v}_b = 0.0;")
    o.extend(seeds)
    o.extend(rev)
    o.extend(epilogue)
    o.append("}")
    return o


def emit_mid():
    decl = ["const Gas& G", "const Mid& e", "const double* U1", "const double* U2",
            "const MidBar& mb", "double* U1b", "double* U2b"]
    pro = [f"  const double {MID_INPUTS[k]} = U1[{k}];" for k in range(8)]
    pro += [f"  const double {MID_INPUTS[8 + k]} = U2[{k}];" for k in range(8)]
    pro.append("  const double gm = G.gm, gm1 = gm - 1.0, g21 = G.g21;")
    pro.append("  const double sb = (e.sbxm ? -1.0 : 1.0);")
    seeds = []
    for f in MID_FIELDS:
        field = "as" if f == "as_" else f
        seeds.append(f"  {f}_b += mb.{field};")
    epi = ["  " + " ".join(f"U1b[{k}] += {MID_INPUTS[k]}_b;" for k in range(8)),
           "  " + " ".join(f"U2b[{k}] += {MID_INPUTS[8 + k]}_b;" for k in range(8))]
    # the midpoint scalars the forward already holds in e (bit-identical
    # arithmetic); frozen statements whose flag needs their raw value are
    # recomputed
    subst = {f: f"e.{'as' if f == 'as_' else f}" for f in
             ("u", "v", "w", "uu", "a", "ca2", "ca", "cs", "cf", "rr", "af", "as_", "bty", "btz",
              "th1", "th2", "vb")}
    return emit_program("midpoint_adjoint", decl, MID, MID_INPUTS, pro, seeds, epi, subst)


def emit_flux():
    decl = ["double gm", "const double* q", "const double* Fb", "double* qb"]
    pro = [f"  const double q{k} = q[{k}];" for k in range(8)]
    pro.append("  const double gm1 = gm - 1.0;")
    stmts = list(FLUX) + [(f"fo{m}", expr) for m, expr in sorted(FLUX_OUT.items())]
    seeds = [f"  fo{m}_b = Fb[{m}];" for m in sorted(FLUX_OUT)]
    epi = [f"  qb[{k}] += q{k}_b;" for k in range(8)]
    return emit_program("flux_x_adjoint", decl, stmts, [f"q{k}" for k in range(8)], pro, seeds,
                        epi)


def main():
    o = []
    o.append("// GENERATED by gen_adjoint.py from the formulas restated there; do not edit.")
    o.append("// Reverse-mode adjoints of the ENO-Roe interface algebra with frozen branches.")
    o.append("#pragma once")
    o.append("")
    o.append('#include "mhd_eigen.cuh"')
    o.append("")
    o.append("namespace mhd {")
    o.append("namespace MHD_KNS {")
    o.append("")
    o.append("// d sqrt(v) / dv, 0 at v = 0 (frozen one-sided branch)")
    o.append("__device__ __forceinline__ double inv2sqrt(double v) {")
    o.append("  return v > 0.0 ? 0.5 * rsqrt(v) : 0.0;")
    o.append("}")
    o.append("")
    o.append("// Adjoints of the Mid scalars.")
    o.append("struct MidBar {")
    o.append("  double " + ", ".join("as" if f == "as_" else f for f in MID_FIELDS) + ";")
    o.append("};")
    o.append("")
    check_pairs()
    o.extend(emit_pairs())
    o.append("")
    o.append("// Adds d(Mid)/d(U1, U2)^T mb to U1b, U2b (midpoint() of mhd_eigen.cuh).")
    o.extend(emit_mid())
    o.append("")
    o.append("// Adds (dF/dq)^T Fb to qb for the physical x flux F(q) (F[4] = 0).")
    o.extend(emit_flux())
    o.append("")
    o.append("}  // namespace MHD_KNS")
    o.append("}  // namespace mhd")
    sys.stdout.write("\n".join(o) + "\n")


if __name__ == "__main__":
    main()
