"""Generate jac_adjoint.cuh: reverse-mode derivatives of the flux Jacobians a, b, c.

Reads the Jacobian functions of fdv_physics.cuh (jac_a_2d/3d, jac_b_rows_2d/3d,
jac_c_rows_2d/3d), evaluates their straight-line bodies symbolically with sympy for every
direction i, and emits, for each function, the gradient of sum_entries W_entry * entry with
respect to the Gauss-point state it reads (E, U, dU, v, mu, k, tau) and to the gas constant Cv
(through which the Mach number enters).  The weights W are the
adjoint of the entries in the element functional (adjoint.cuh); the generated code is the
reverse sweep of the same formulas, with common subexpressions shared (sympy cse).

Run:  python gen_jac_adjoint.py   (the Makefile reruns it when fdv_physics.cuh changes)
"""
import os
import re

import sympy as sp
from sympy.printing.c import C99CodePrinter

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "fdv_physics.cuh")
OUT = os.path.join(HERE, "jac_adjoint.cuh")

# Gauss-point state fields a Jacobian may read, as (C access, symbol name)
STATE = ([("f.E", "E")] + [(f"f.U[{q}]", f"U{q}") for q in range(5)] +
         [(f"f.dU[{q}][{c}]", f"dU{q}{c}") for q in range(5) for c in range(3)] +
         [(f"f.v[{c}]", f"v{c}") for c in range(3)] + [("f.mu", "mu"), ("f.k", "k")] +
         [(f"f.tau[{a}][{b}]", f"tau{a}{b}") for a in range(3) for b in range(3)])
GAS = ["gamma", "gamm1", "gm1d2", "gamm3", "gm3d2", "Cv", "creyn"]


def function_body(src, name):
    """The text between the braces of `name(`'s definition."""
    m = re.search(r"\n[^\n]*\b" + re.escape(name) + r"\(", src)
    i = src.index("{", m.end())
    depth, j = 0, i
    while True:
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[i + 1:j]
        j += 1


def statements(body):
    """Split a body into a tree: ('stmt', text) | ('if', [(cond, block), ...])."""
    body = re.sub(r"//[^\n]*", "", body)
    body = re.sub(r"#pragma[^\n]*", "", body)
    s = body.strip()

    def parse_block(s, k):
        items = []
        while k < len(s):
            while k < len(s) and s[k].isspace():
                k += 1
            if k >= len(s):
                break
            if s[k] == "}":
                return items, k + 1
            if s.startswith("if", k) and s[k + 2:k + 3] in " (":
                branches = []
                while True:
                    c0 = s.index("(", k)
                    depth, c1 = 0, c0
                    while True:
                        if s[c1] == "(":
                            depth += 1
                        elif s[c1] == ")":
                            depth -= 1
                            if depth == 0:
                                break
                        c1 += 1
                    cond = s[c0 + 1:c1]
                    b0 = s.index("{", c1)
                    blk, k = parse_block(s, b0 + 1)
                    branches.append((cond, blk))
                    m = re.match(r"\s*else\s*", s[k:])
                    if not m:
                        break
                    k += m.end()
                    if s.startswith("if", k):
                        continue
                    b0 = s.index("{", k)
                    blk, k = parse_block(s, b0 + 1)
                    branches.append(("1", blk))
                    break
                items.append(("if", branches))
                continue
            if s.startswith("for", k):
                e = s.index(";", s.index(")", k))
                items.append(("for", s[k:e + 1]))
                k = e + 1
                continue
            e = s.index(";", k)
            items.append(("stmt", s[k:e].strip()))
            k = e + 1
        return items, k

    tree, _ = parse_block(s, 0)
    return tree


def split_top(s, sep=","):
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return [p.strip() for p in parts]


class Interp:
    def __init__(self, ndim, i):
        self.ndim, self.i = ndim, i
        self.sym = {n: sp.Symbol(n) for _, n in STATE}
        self.gas = {g: sp.Symbol("th_" + g) for g in GAS}
        self.locals = {}
        self.entries = {}
        self.scale = None

    def expr(self, e):
        e = e.strip()
        for acc, n in sorted(STATE, key=lambda t: -len(t[0])):
            e = e.replace(acc, f"S['{n}']")
        e = re.sub(r"\bth\.(\w+)", lambda m: f"G['{m.group(1)}']", e)
        # tau alias: const auto& t = f.tau  ->  t[a][b]
        e = re.sub(r"\bt\[(\d)\]\[(\d)\]", lambda m: f"S['tau{m.group(1)}{m.group(2)}']", e)

        def name(m):
            w = m.group(0)
            if w in self.locals:
                return f"L['{w}']"
            if w in ("S", "G", "L"):
                return w
            return w

        e = re.sub(r"(?<![\['\w.])[A-Za-z_]\w*(?![\w'])", name, e)
        e = re.sub(r"(\d+)\.(?!\d)", r"\1.0", e).replace("\n", " ")
        v = eval("(" + e + ")", {"S": self.sym, "G": self.gas, "L": self.locals, "sp": sp})
        return sp.nsimplify(v, rational=False) if isinstance(v, (int, float)) else v

    def run(self, tree):
        for kind, item in tree:
            if kind == "if":
                for cond, blk in item:
                    c = cond.replace("i", str(self.i)) if cond != "1" else "1"
                    if eval(c):
                        self.run(blk)
                        break
            elif kind == "for":
                if "*=" in item:
                    m = re.search(r"\*=\s*(\w+)", item)
                    self.scale = self.locals[m.group(1)]
            else:
                self.stmt(item)

    def stmt(self, st):
        if st.startswith("S* blk") or "= 0.0" in st and st.startswith("m["):
            return
        m = re.match(r"const auto& t = f\.tau", st)
        if m:
            return
        m = re.match(r"const S (\w+)\[(\d+)\] = \{(.*)\}$", st, re.S)
        if m:
            self.locals[m.group(1)] = [self.expr(x) for x in split_top(m.group(3))]
            return
        m = re.match(r"const S (.*)$", st, re.S)
        if m:
            for decl in split_top(m.group(1)):
                n, e = decl.split("=", 1)
                self.locals[n.strip()] = self.expr(e)
            return
        m = re.match(r"JA\((\w+),\s*(\d+),\s*(\d+),\s*(\d+)\)\s*=\s*(.*)$", st, re.S)
        if m:
            ii = self.i if m.group(1) == "blk" else int(m.group(2))
            self.entries[(ii, int(m.group(3)), int(m.group(4)))] = self.expr(m.group(5))
            return
        m = re.match(r"JC\((\w+),\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)\)\s*=\s*(.*)$", st, re.S)
        if m:
            self.entries[(self.i, int(m.group(3)), int(m.group(4)), int(m.group(5)))] = self.expr(m.group(6))
            return
        raise ValueError("unhandled statement: " + st)


def entries_of(src, fname, ndim, i):
    it = Interp(ndim, i)
    it.run(statements(function_body(src, fname)))
    if it.scale is not None:
        it.entries = {k: v * it.scale for k, v in it.entries.items()}
    return it


def emit(fname, out_name, ndim, per_row, src):
    """Reverse code: g += d/dstate sum W[idx] entry[idx]."""
    lines = []
    rows = range(ndim) if per_row else [None]
    for i in rows:
        it = entries_of(src, fname, ndim, 0 if i is None else i)
        ents = it.entries
        W = {}
        total = 0
        for key, e in ents.items():
            if e == 0:
                continue
            if len(key) == 3:
                idx = key[0] * 25 + key[1] * 5 + key[2] if i is None else key[1] * 5 + key[2]
            else:
                idx = key[1] * 25 + key[2] * 5 + key[3]
            w = sp.Symbol(f"W[{idx}]")
            W[idx] = w
            total += w * e
        used = [n for _, n in STATE if it.sym[n] in total.free_symbols]
        grads = [sp.diff(total, it.sym[n]) for n in used]
        names = [gname(n) for n in used]
        cv = it.gas["Cv"]
        if cv in total.free_symbols:  # the Mach number enters the Jacobians through Cv
            grads.append(sp.diff(total, cv))
            names.append("gCv")
        reps, red = sp.cse(grads, symbols=sp.numbered_symbols("t"), optimizations="basic")
        body = []
        for s_, e in reps:
            body.append(f"    const double {s_} = {ccode(e)};")
        for n, e in zip(names, red):
            body.append(f"    {n} += {ccode(e)};")
        cond = "" if i is None else f"  if (i == {i}) {{\n"
        lines.append(cond + "\n".join(body) + ("\n  }" if i is not None else ""))
    sig_i = ", int i" if per_row else ""
    return (f"// reverse of {fname}: g += d/d(state) of sum_idx W[idx] * entry[idx], gCv += d/dCv of it\n"
            f"template <class WA>\n"
            f"CFDV_HD CFDV_INLINE void {out_name}(const GasParams& th, const GpState& f{sig_i}, const WA& W, "
            f"GpState& g, double& gCv) {{\n" + "\n".join(lines) + "\n  (void)gCv;\n}\n")


def gname(n):
    if n == "E":
        return "g.E"
    if n in ("mu", "k"):
        return "g." + n
    m = re.match(r"U(\d)$", n)
    if m:
        return f"g.U[{m.group(1)}]"
    m = re.match(r"dU(\d)(\d)$", n)
    if m:
        return f"g.dU[{m.group(1)}][{m.group(2)}]"
    m = re.match(r"v(\d)$", n)
    if m:
        return f"g.v[{m.group(1)}]"
    m = re.match(r"tau(\d)(\d)$", n)
    if m:
        return f"g.tau[{m.group(1)}][{m.group(2)}]"
    raise ValueError(n)


class _Printer(C99CodePrinter):
    """Integer powers as products and quotients instead of pow()."""

    def _print_Pow(self, e):
        b, x = e.as_base_exp()
        if x.is_Integer and 1 <= abs(int(x)) <= 3:
            p = "*".join([self.parenthesize(b, 100)] * abs(int(x)))
            return f"({p})" if x > 0 else f"(1.0/({p}))"
        return super()._print_Pow(e)


def ccode(e):
    s = _Printer().doprint(e)
    s = re.sub(r"\bth_(\w+)", r"th.\1", s)
    rep = {n: acc for acc, n in STATE}
    s = re.sub(r"\b(E|U\d|dU\d\d|v\d|mu|k|tau\d\d)\b", lambda m: rep[m.group(1)], s)
    return s


def main():
    src = open(SRC).read()
    parts = [
        "// GENERATED by gen_jac_adjoint.py from fdv_physics.cuh -- do not edit.",
        "// Reverse-mode derivatives of the flux Jacobians: for weights W on the entries (the",
        "// adjoint of the entries in the element functional), g += d/d(state) sum W * entry and",
        "// gCv += d/dCv sum W * entry.  W is any type with operator[](int): an array, or an",
        "// accessor that forms each weight where the code reads it.",
        "#pragma once",
        '#include "fdv_physics.cuh"',
        "",
        "namespace cfdv {",
        "",
    ]
    for nd in (2, 3):
        parts.append(emit(f"jac_a_{nd}d", f"jac_a_adj_{nd}d", nd, False, src))
        parts.append(emit(f"jac_b_rows_{nd}d", f"jac_b_rows_adj_{nd}d", nd, True, src))
        parts.append(emit(f"jac_c_rows_{nd}d", f"jac_c_rows_adj_{nd}d", nd, True, src))
    parts.append("}  // namespace cfdv\n")
    with open(OUT, "w") as f:
        f.write("\n".join(parts))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
