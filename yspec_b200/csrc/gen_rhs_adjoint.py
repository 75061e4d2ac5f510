"""Generate ysg_rhs_adjoint.cuh: transposes and coefficient gradients of the
right-hand sides in ysg_ode.cuh.

    python yspec_b200/csrc/gen_rhs_adjoint.py        # rewrites ysg_rhs_adjoint.cuh

Every right-hand side of the radial systems is bilinear: each output
component d[i] is a sum of terms (coefficient-matrix entry) x (state
component) x (constant), written in ysg_ode.cuh as nests of cmac / cmsc
(d += x y / d -= x y) over the entries of the system's coefficient struct.
This script parses those nests (they are valid Python expressions) into
term lists and emits, for every system, two functions the reverse sweep
needs at each Cash-Karp stage:

    tr(a, k, g)       g = A^T k      (A the system matrix built from a)
    cgrad(k, y, s)    s_e += k . (dA/da_e) y  for every entry e of a

so they follow the forward right-hand sides term for term and never drift
from them.  The output is committed; the build does not run this script.
"""
from __future__ import annotations

import ast
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "ysg_ode.cuh"
OUT = HERE / "ysg_rhs_adjoint.cuh"

# system struct -> (coefficient struct, state array name)
SYSTEMS = ["TorSys", "RadSys", "MinorSolidG", "MinorFluidG", "BvecSolidG",
           "MinorSolidNC", "MinorFluidNC", "BvecSolidNC"]
COEF_FIELDS = {
    "TorCoef": ["t", "k", "s"],
    "RadCoef": ["t", "k", "s"],
    "SolidCoef": ["t11", "t12", "k11", "k22", "s11", "s12", "s22", "t21", "t22", "t31", "t33", "k33",
                  "s13", "s23"],
    "FluidCoef": ["t11", "t12", "k11", "s11", "s12", "s22", "t21", "t22", "k22"],
}


class Lin:
    """Linear form: {atom: factor}; atoms are ('c', field) or ('y', index)."""

    def __init__(self, terms=None, const=0.0):
        self.t = dict(terms or {})
        self.const = const

    def kind(self):
        kinds = {a[0] for a in self.t}
        assert len(kinds) <= 1, kinds
        return kinds.pop() if kinds else None

    def scale(self, f):
        return Lin({a: f * v for a, v in self.t.items()}, f * self.const)

    def add(self, o, sign=1.0):
        t = dict(self.t)
        for a, v in o.t.items():
            t[a] = t.get(a, 0.0) + sign * v
        return Lin(t, self.const + sign * o.const)


class Bil:
    """Sum of (coefficient field, state index, factor)."""

    def __init__(self, terms=None):
        self.t = list(terms or [])

    def add(self, o, sign=1.0):
        return Bil(self.t + [(c, j, sign * f) for c, j, f in o.t])

    def scale(self, f):
        return Bil([(c, j, f * v) for c, j, v in self.t])


def product(x, y):
    if isinstance(x, float):
        return y.scale(x)
    if isinstance(y, float):
        return x.scale(y)
    assert isinstance(x, Lin) and isinstance(y, Lin) and x.const == 0 and y.const == 0
    if x.kind() == "y":
        x, y = y, x
    assert x.kind() == "c" and y.kind() == "y", (x.t, y.t)
    return Bil([(cx[1], yy[1], fx * fy) for cx, fx in x.t.items() for yy, fy in y.t.items()])


def evaluate(node, env, state):
    if isinstance(node, ast.Constant):
        return float(node.value)
    if isinstance(node, ast.Name):
        return env[node.id]
    if isinstance(node, ast.Attribute):            # a.field
        assert isinstance(node.value, ast.Name) and node.value.id == "a"
        return Lin({("c", node.attr): 1.0})
    if isinstance(node, ast.Subscript):            # m[3]
        assert isinstance(node.value, ast.Name) and node.value.id == state
        return Lin({("y", int(node.slice.value)): 1.0})
    if isinstance(node, ast.UnaryOp) and isinstance(node.op, ast.USub):
        v = evaluate(node.operand, env, state)
        return -v if isinstance(v, float) else v.scale(-1.0)
    if isinstance(node, ast.BinOp):
        a, b = evaluate(node.left, env, state), evaluate(node.right, env, state)
        if isinstance(node.op, ast.Mult):
            return product(a, b)
        sign = 1.0 if isinstance(node.op, ast.Add) else -1.0
        assert isinstance(node.op, (ast.Add, ast.Sub))
        if isinstance(a, float) and isinstance(b, float):
            return a + sign * b
        return a.add(b, sign)
    if isinstance(node, ast.Call):
        name = node.func.id
        assert name in ("cmac", "cmsc"), name
        s, x, y = (evaluate(n, env, state) for n in node.args)
        return s.add(product(x, y), 1.0 if name == "cmac" else -1.0)
    raise ValueError(ast.dump(node))


def parse_system(src: str, name: str):
    m = re.search(r"struct " + name + r" \{(.*?)\n\};", src, re.S)
    body = m.group(1)
    n = int(re.search(r"static constexpr int N = (\d+)", body).group(1))
    coef_type = re.search(r"(\w+Coef) a = ", body).group(1)
    state = re.search(r"const mcplx\* (\w+), Out d", body).group(1)
    env = {}
    outs = {}
    for line in body.splitlines():
        line = line.strip()
        md = re.match(r"(?:const )?(?:mcplx|mreal) (.*);$", line)
        if md:
            for part in re.split(r",\s*(?=\w+ = )", md.group(1)):
                lhs, rhs = part.split(" = ", 1)
                env[lhs.strip()] = evaluate(ast.parse(rhs, mode="eval").body, env, state)
            continue
        mo = re.match(r"d\[(\d+)\] = (.*);$", line)
        if mo:
            v = evaluate(ast.parse(mo.group(2), mode="eval").body, env, state)
            assert isinstance(v, Bil)
            outs[int(mo.group(1))] = v
    assert sorted(outs) == list(range(n)), (name, sorted(outs))
    return n, coef_type, outs


def fmt(f):
    return repr(float(f))


def emit(name, n, coef_type, outs):
    fields = COEF_FIELDS[coef_type]
    L = [f"// {name}: {n} components, coefficients {coef_type}",
         f"struct {name}Adj {{",
         f"    static constexpr int N = {n};",
         f"    using Coef = {coef_type};",
         f"    using Bar = {coef_type}Bar;",
         "    // g = A^T k",
         f"    __device__ static __forceinline__ void tr(const {coef_type}& a, const cd* k, cd* g)",
         "    {"]
    by_in = {}
    for i, b in outs.items():
        for c, j, f in b.t:
            by_in.setdefault(j, []).append((c, i, f))
    for j in range(n):
        terms = by_in.get(j, [])
        if not terms:
            L.append(f"        g[{j}] = mk(0.0);")
            continue
        parts = [f"({fmt(f)} * a.{c}) * k[{i}]" if f != 1.0 else f"a.{c} * k[{i}]" for c, i, f in terms]
        L.append(f"        g[{j}] = " + " + ".join(parts) + ";")
    L.append("    }")
    L.append("    // s.e += k . (dA/da_e) y")
    L.append(f"    __device__ static __forceinline__ void cgrad(const cd* k, const cd* y, {coef_type}Bar& s)")
    L.append("    {")
    by_c = {}
    for i, b in outs.items():
        for c, j, f in b.t:
            by_c.setdefault(c, []).append((i, j, f))
    for c in fields:
        terms = by_c.get(c, [])
        if not terms:
            continue
        parts = [f"{fmt(f)} * (k[{i}] * y[{j}])" if f != 1.0 else f"k[{i}] * y[{j}]" for i, j, f in terms]
        L.append(f"        s.{c} += " + " + ".join(parts) + ";")
    L.append("    }")
    L.append("};")
    return "\n".join(L)


def main() -> int:
    src = SRC.read_text()
    parts = ["// ysg_rhs_adjoint.cuh -- GENERATED by gen_rhs_adjoint.py from the right-hand",
             "// sides of ysg_ode.cuh; do not edit.  For each system: tr() applies the",
             "// transposed system matrix, cgrad() accumulates the gradient of k . A y",
             "// with respect to each entry of the coefficient struct (complex, in the",
             "// convention dL = Re(sum s_e da_e)).",
             "#pragma once",
             '#include "ysg_ode.cuh"',
             "",
             "namespace ysg {",
             "inline namespace YSG_VARIANT {",
             ""]
    for ct, fields in COEF_FIELDS.items():
        parts.append(f"struct {ct}Bar {{")
        parts.append("    cd " + ", ".join(fields) + ";")
        parts.append(f"    __device__ void zero() {{ " + " ".join(f"{f} = mk(0.0);" for f in fields) + " }")
        parts.append("};")
        parts.append("")
    for name in SYSTEMS:
        n, ct, outs = parse_system(src, name)
        parts.append(emit(name, n, ct, outs))
        parts.append("")
    parts += ["}  // namespace YSG_VARIANT", "}  // namespace ysg", ""]
    OUT.write_text("\n".join(parts))
    print(f"wrote {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
