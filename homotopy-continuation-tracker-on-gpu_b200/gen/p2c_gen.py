"""Native table and coefficient-expression generator for homotopy problems.

Replaces, for the tracker's purposes, the MATLAB generator of the reference
(auto-data-gen-tools/autogen_gpuhc.m:128-708 and createUnivPoly4Coeffs.m).
Two modes:

* derive  -- for a problem the reference already ships: read its polynomial
  system (``sys_<p>.m``) and its shipped ``dHdt_indx.txt``; recover every
  unique coefficient c_k(p) (a polynomial in the parameters) in the shipped
  table's numbering, and check that both shipped tables reproduce H and
  dH/dx of the system exactly.  Writes ``p2c_terms.txt``.
* generate -- for a new problem: from the polynomial system alone, number the
  unique coefficients, and write ``dHdx_indx.txt`` / ``dHdt_indx.txt`` in the
  reference layout plus ``p2c_terms.txt``.

``p2c_terms.txt`` lists c_k(p) = sum_terms (num/den) * prod_j p_j and is what
the product's coefficient builders (host: csrc/problem.cpp p2c_host, device:
csrc/p2c.cu) expand into the per-hypothesis tables c_k(t) = c_k(q + t (p - q)).

Table layout (reference, GPU-HC/magmaHC/gpu-idx-evals/dev-eval-indxing-P3P.cuh:69-120):
  dHdx[row][col][term][part], part = [scale, k, var_0 .. var_{Px-3}]
  dHdt[row][term][part],      part = [scale, k, var_0 .. var_{Pt-3}]
  var index N is the constant 1; padding term = [0, M, N, ...];
  coefficient index M is the constant-1 sentinel for parameter-free monomials.
"""
import os
import re
import sys
from fractions import Fraction

import sympy as sp


# ----------------------------------------------------------------------------
# parsing
# ----------------------------------------------------------------------------

def parse_matlab_system(path):
    """Return (xs, ps, eqs) from a reference sys_<p>.m file.

    The files declare ``syms x1 .. xN`` and ``syms p1 .. pP`` and list
    ``f(i) = <polynomial>;`` one per line.
    """
    text = open(path).read()
    syms = []
    for m in re.finditer(r"^\s*syms\s+([^\n%]+)", text, re.M):
        syms.append(m.group(1).split())
    xs_names = [s for group in syms for s in group if re.fullmatch(r"x\d+", s)]
    ps_names = [s for group in syms for s in group if re.fullmatch(r"p\d+", s)]
    xs = [sp.Symbol(n) for n in sorted(xs_names, key=lambda s: int(s[1:]))]
    ps = [sp.Symbol(n) for n in sorted(ps_names, key=lambda s: int(s[1:]))]
    loc = {str(s): s for s in xs + ps}
    eqs = {}
    for m in re.finditer(r"^\s*f\((\d+)\)\s*=\s*([^;]+);", text, re.M):
        expr = m.group(2).replace("^", "**")
        eqs[int(m.group(1))] = sp.expand(sp.sympify(expr, locals=loc))
    ordered = [eqs[i] for i in sorted(eqs)]
    return xs, ps, ordered


def read_ints(path):
    return [int(v) for v in open(path).read().split()]


def read_yaml_flat(path):
    """The flat ``key: value`` subset of the reference's gpuhc_settings.yaml."""
    out = {}
    for line in open(path):
        line = line.split("#", 1)[0]
        m = re.match(r"\s*([A-Za-z_][A-Za-z0-9_]*)\s*:\s*(\S+)", line)
        if m:
            out[m.group(1)] = m.group(2)
    return out


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------

def _monomial_key(vars_, N):
    """exponent tuple of prod x[v] over the variable slots (slot N == 1)."""
    e = [0] * N
    for v in vars_:
        if v != N:
            e[v] += 1
    return tuple(e)


def _poly_in_x(expr, xs):
    return sp.Poly(expr, *xs).as_dict()


def _terms_of(expr, ps):
    """c(p) as [(Fraction, [param indices with repetition])]."""
    expr = sp.expand(expr)
    if expr == 0:
        return []
    poly = sp.Poly(expr, *ps)
    out = []
    for exps, coef in poly.terms():
        fac = []
        for j, e in enumerate(exps):
            fac += [j] * int(e)
        c = sp.Rational(coef)
        out.append((Fraction(int(c.p), int(c.q)), fac))
    return out


# ----------------------------------------------------------------------------
# derive mode: recover c_k in the shipped numbering
# ----------------------------------------------------------------------------

def derive(problem_dir, sys_m_path):
    y = read_yaml_flat(os.path.join(problem_dir, "gpuhc_settings.yaml"))
    if y.get("GPUHC_Type") != "P2C":
        raise ValueError("derive: only P2C problems carry coefficient tables")
    N = int(y["Num_Of_Vars"])
    P = int(y["Num_Of_Params"])
    M = int(y["Num_Of_Coeffs_From_Params"])
    K = int(y["Max_Order_Of_T"])
    Tx, Px = int(y["dHdx_Max_Terms"]), int(y["dHdx_Max_Parts"])
    Tt, Pt = int(y["dHdt_Max_Terms"]), int(y["dHdt_Max_Parts"])
    xs, ps, eqs = parse_matlab_system(sys_m_path)
    # a system may declare trailing parameters its equations never use (optimal_PnP_quat declares
    # p1..p85 and uses p1..p81, as its YAML's Num_Of_Params says): drop those
    used = set().union(*[e.free_symbols for e in eqs]) if eqs else set()
    while len(ps) > P and ps[-1] not in used:
        ps = ps[:-1]
    if len(xs) != N or len(ps) != P or len(eqs) != N:
        raise ValueError("system %s: %d vars %d params %d eqs, yaml says N=%d P=%d"
                         % (sys_m_path, len(xs), len(ps), len(eqs), N, P))
    ht = read_ints(os.path.join(problem_dir, "dHdt_indx.txt"))
    hx = read_ints(os.path.join(problem_dir, "dHdx_indx.txt"))
    if len(ht) != N * Tt * Pt or len(hx) != N * N * Tx * Px:
        raise ValueError("table sizes do not match the YAML")

    coef = [None] * M
    for r in range(N):
        fdict = _poly_in_x(eqs[r], xs)
        seen = {}
        for j in range(Tt):
            e = ht[(r * Tt + j) * Pt:(r * Tt + j + 1) * Pt]
            s, k, vars_ = e[0], e[1], e[2:]
            if s == 0:
                continue
            key = _monomial_key(vars_, N)
            if key in seen:
                raise ValueError("row %d: monomial %s appears twice" % (r, key))
            seen[key] = (s, k)
        if set(seen) != set(fdict):
            raise ValueError("row %d: table monomials %s != system monomials %s"
                             % (r, sorted(seen), sorted(fdict)))
        for key, (s, k) in seen.items():
            val = sp.expand(fdict[key] / s)
            if k == M:
                if val != 1:
                    raise ValueError("row %d: sentinel term with coefficient %s" % (r, val))
                continue
            if coef[k] is None:
                coef[k] = val
            elif sp.expand(coef[k] - val) != 0:
                raise ValueError("coefficient %d inconsistent across rows" % k)
    missing = [k for k in range(M) if coef[k] is None]
    if missing:
        raise ValueError("coefficients never referenced by dHdt: %s" % missing)

    # cross-check dH/dx: sum of table terms == d f_r / d x_i
    cs = coef + [sp.Integer(1)]
    for r in range(N):
        for i in range(N):
            expect = sp.expand(sp.diff(eqs[r], xs[i]))
            got = 0
            for j in range(Tx):
                base = ((r * N + i) * Tx + j) * Px
                e = hx[base:base + Px]
                if e[0] == 0:
                    continue
                mono = 1
                for v in e[2:]:
                    if v != N:
                        mono *= xs[v]
                got += e[0] * cs[e[1]] * mono
            if sp.expand(got - expect) != 0:
                raise ValueError("dHdx row %d col %d does not match d f/dx" % (r, i))
    for k in range(M):
        deg = sp.Poly(coef[k], *ps).total_degree() if coef[k].free_symbols else 0
        if deg > K:
            raise ValueError("coefficient %d has degree %d > K=%d" % (k, deg, K))
    return dict(N=N, P=P, M=M, K=K, coefs=[_terms_of(c, ps) for c in coef])


# ----------------------------------------------------------------------------
# generate mode: number coefficients and emit the two tables
# ----------------------------------------------------------------------------

def generate(xs, ps, eqs):
    """Tables for a new P2C problem from its polynomial system.

    Unique coefficients are numbered in order of first appearance (rows in
    order, monomials in sympy's graded order); a coefficient equal to another
    up to an integer factor is shared with that factor moved into the scale.
    """
    N = len(xs)
    coefs = []          # sympy expressions in ps
    ht_rows = []        # per row: list of (scale, k, [vars])
    hx_entries = {}     # (r, i) -> list of (scale, k, [vars])

    def index_of(c):
        for k, old in enumerate(coefs):
            q = sp.simplify(c / old)
            if q.is_Integer:
                return k, int(q)
        coefs.append(c)
        return len(coefs) - 1, 1

    M_sentinel = None
    rows = []
    for r in range(N):
        d = sp.Poly(eqs[r], *xs)
        terms = []
        for exps, c in d.terms():
            c = sp.expand(c)
            vars_ = []
            for v, e in enumerate(exps):
                vars_ += [v] * int(e)
            if not c.free_symbols:
                terms.append(("const", int(c), vars_))
            else:
                k, s = index_of(c)
                terms.append(("coef", (k, s), vars_))
        rows.append(terms)
    M = len(coefs)
    M_sentinel = M
    for r in range(N):
        out = []
        for kind, val, vars_ in rows[r]:
            if kind == "const":
                out.append((val, M_sentinel, vars_))
            else:
                k, s = val
                out.append((s, k, vars_))
        ht_rows.append(out)
    # dH/dx: derivative of each monomial term
    for r in range(N):
        for i in range(N):
            lst = []
            for s, k, vars_ in ht_rows[r]:
                e = vars_.count(i)
                if e == 0:
                    continue
                rest = list(vars_)
                rest.remove(i)
                lst.append((s * e, k, rest))
            # merge equal (k, vars)
            merged = {}
            for s, k, rest in lst:
                key = (k, tuple(sorted(rest)))
                merged[key] = merged.get(key, 0) + s
            hx_entries[(r, i)] = [(s, k, list(v)) for (k, v), s in merged.items() if s != 0]
    Tt = max(len(t) for t in ht_rows)
    Pt = 2 + max(len(v) for t in ht_rows for _, _, v in t)
    Tx = max(1, max(len(v) for v in hx_entries.values()))
    Px = 2 + max([len(v) for lst in hx_entries.values() for _, _, v in lst] + [1])
    ht = []
    for r in range(N):
        for j in range(Tt):
            if j < len(ht_rows[r]):
                s, k, v = ht_rows[r][j]
                ht += [s, k] + v + [N] * (Pt - 2 - len(v))
            else:
                ht += [0, M] + [N] * (Pt - 2)
    hx = []
    for r in range(N):
        for i in range(N):
            lst = hx_entries[(r, i)]
            for j in range(Tx):
                if j < len(lst):
                    s, k, v = lst[j]
                    hx += [s, k] + v + [N] * (Px - 2 - len(v))
                else:
                    hx += [0, M] + [N] * (Px - 2)
    K = max([sp.Poly(c, *ps).total_degree() for c in coefs] + [1])
    return dict(N=N, P=len(ps), M=M, K=K, Tx=Tx, Px=Px, Tt=Tt, Pt=Pt, hx=hx, ht=ht,
                coefs=[_terms_of(c, ps) for c in coefs])


# ----------------------------------------------------------------------------
# output
# ----------------------------------------------------------------------------

def write_p2c_terms(path, info, source):
    with open(path, "w") as f:
        f.write("# coefficient expressions c_k(p) = sum num/den * prod p_j (0-based p_j)\n")
        f.write("# generated by gen/p2c_gen.py from %s\n" % source)
        f.write("# header: M K P ; then per term: k num den nfactors j_1 .. j_n\n")
        f.write("%d %d %d\n" % (info["M"], info["K"], info["P"]))
        for k, terms in enumerate(info["coefs"]):
            for c, fac in terms:
                f.write("%d %d %d %d%s\n" % (k, c.numerator, c.denominator, len(fac),
                                            "".join(" %d" % j for j in fac)))


def write_table(path, vals, per_line):
    with open(path, "w") as f:
        for i in range(0, len(vals), per_line):
            f.write("\t".join(str(v) for v in vals[i:i + per_line]) + "\t\n")


if __name__ == "__main__":
    if len(sys.argv) != 3:
        print("usage: p2c_gen.py <problem_dir> <sys_p.m>")
        sys.exit(2)
    info = derive(sys.argv[1], sys.argv[2])
    write_p2c_terms(os.path.join(sys.argv[1], "p2c_terms.txt"), info, os.path.basename(sys.argv[2]))
    print("M=%d K=%d P=%d terms=%d" % (info["M"], info["K"], info["P"],
                                      sum(len(t) for t in info["coefs"])))
