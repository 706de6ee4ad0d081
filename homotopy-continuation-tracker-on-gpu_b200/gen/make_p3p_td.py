"""Generate the problem folder P3P_TD: P3P by a total-degree homotopy.

Unknowns: the depths d1, d2, d3 of three points along unit bearings b1, b2, b3.
Equations, one per point pair (i, j) in (1,2), (1,3), (2,3):
    a_ii d_i^2 + a_jj d_j^2 + a_ij d_i d_j + a_0 = 0
with 12 coefficient parameters [a_ii, a_jj, a_ij, a_0] per equation.  The
target is the P3P system (1, 1, -2 c_ij, -s_ij) with c_ij = b_i . b_j and
s_ij = |X_i - X_j|^2; the start system gamma (x_k^2 - 1) (one x_k per
equation) uses the same monomials, so the straight-line parameter homotopy
is exactly H = (1 - t) gamma G + t F with the 8 start solutions (+-1, +-1, +-1).
gamma is a unit-modulus complex number (the gamma trick keeps paths regular).

The tables are produced by p2c_gen.generate in the reference layout and the
folder can be read by anything that reads the reference's problem folders.

usage: python make_p3p_td.py [gamma_angle_rad]
"""
import itertools
import math
import os
import sys

import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import p2c_gen  # noqa: E402

DEST = os.path.join(os.path.dirname(HERE), "problems", "P3P_TD")
PAIRS = [(0, 1), (0, 2), (1, 2)]
# the unknown whose square forms the start equation of each pair
START_VAR = [0, 2, 1]


def system():
    xs = sp.symbols("x1:4")
    ps = sp.symbols("p1:13")
    eqs = []
    for e, (i, j) in enumerate(PAIRS):
        a_ii, a_jj, a_ij, a_0 = ps[4 * e:4 * e + 4]
        eqs.append(sp.expand(a_ii * xs[i] ** 2 + a_jj * xs[j] ** 2 + a_ij * xs[i] * xs[j] + a_0))
    return list(xs), list(ps), eqs


def start_params(gamma):
    """gamma (x_k^2 - 1) written in the [a_ii, a_jj, a_ij, a_0] slots of each equation."""
    out = []
    for e, (i, j) in enumerate(PAIRS):
        k = START_VAR[e]
        out += [gamma if k == i else 0.0, gamma if k == j else 0.0, 0.0, -gamma]
    return out


def target_params(c, s):
    """c, s: dicts (i, j) -> cosine of the bearings, squared distance of the points."""
    out = []
    for (i, j) in PAIRS:
        out += [1.0, 1.0, -2.0 * c[(i, j)], -s[(i, j)]]
    return out


def write(gamma_angle=0.7853981633974483):
    xs, ps, eqs = system()
    info = p2c_gen.generate(xs, ps, eqs)
    os.makedirs(DEST, exist_ok=True)
    g = complex(math.cos(gamma_angle), math.sin(gamma_angle))
    yaml = """%%YAML:1.0

#> P3P by a total-degree homotopy (generated by gen/make_p3p_td.py)
problem_name: P3P_TD
problem_print_out_name: P3P depths by a total-degree homotopy

GPUHC_Type: P2C
GPUHC_Max_Steps: 200
GPUHC_Max_Correction_Steps: 5
GPUHC_Num_Of_Steps_to_Increase_Delta_t: 3

Num_Of_Vars: 3
Num_Of_Params: 12
Num_Of_Tracks: 8
dHdx_Max_Terms: %d
dHdx_Max_Parts: %d
dHdt_Max_Terms: %d
dHdt_Max_Parts: %d
Max_Order_Of_T: %d
Num_Of_Coeffs_From_Params: %d

RANSAC_Dataset: None
""" % (info["Tx"], info["Px"], info["Tt"], info["Pt"], info["K"], info["M"])
    open(os.path.join(DEST, "gpuhc_settings.yaml"), "w").write(yaml)
    with open(os.path.join(DEST, "start_params.txt"), "w") as f:
        for v in start_params(g):
            v = complex(v)
            f.write("%.17g\t%.17g\n" % (v.real, v.imag))
    # a default target: the unit-cube P3P scene of scenes.p3p_td(seed=0)
    sys.path.insert(0, os.path.dirname(HERE))
    import scenes
    (_, tg), _ = scenes.p3p_td(1, seed=0)
    with open(os.path.join(DEST, "target_params.txt"), "w") as f:
        for v in tg[0][:12]:
            f.write("%.17g\t%.17g\n" % (v.real, v.imag))
    with open(os.path.join(DEST, "start_sols.txt"), "w") as f:
        for signs in itertools.product([1.0, -1.0], repeat=3):
            for sgn in signs:
                f.write("%.17g\t%.17g\n" % (sgn, 0.0))
    p2c_gen.write_table(os.path.join(DEST, "dHdx_indx.txt"), info["hx"], info["Tx"] * info["Px"] * 3)
    p2c_gen.write_table(os.path.join(DEST, "dHdt_indx.txt"), info["ht"], info["Tt"] * info["Pt"])
    p2c_gen.write_p2c_terms(os.path.join(DEST, "p2c_terms.txt"), info, "gen/make_p3p_td.py")
    return info


if __name__ == "__main__":
    info = write(float(sys.argv[1]) if len(sys.argv) > 1 else 0.7853981633974483)
    print("P3P_TD: M=%d K=%d Tx=%d Px=%d Tt=%d Pt=%d" % (info["M"], info["K"], info["Tx"], info["Px"],
                                                      info["Tt"], info["Pt"]))
