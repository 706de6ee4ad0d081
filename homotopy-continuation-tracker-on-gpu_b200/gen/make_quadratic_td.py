"""Generate synthetic P2C problem folders of any size: coupled quadratics by a total-degree homotopy.

Used as test fixtures for the system sizes that no shipped problem has (the tracker is compiled for
P2C N in {3, 4, 5, 6, 8, 10, 11, 12, 16, 18}).  Equation i of N (indices mod N):

    a_i0 x_i^2 + a_i1 x_{i+1} x_{i+2} + a_i2 x_{i+3} + a_i3 = 0

with 4N coefficient parameters.  The start parameters (a_i0, a_i1, a_i2, a_i3) = (g, 0, 0, -g) give
g (x_i^2 - 1) = 0, solved by every sign pattern (+-1, ..., +-1); g is a unit-modulus complex number,
so the straight-line parameter homotopy is the gamma-trick total-degree homotopy.  The folder keeps
`paths` of the 2^N start solutions (enough for parity tests; the full total degree is not needed),
and a seeded random real target.  Tables and p2c_terms.txt come from p2c_gen.generate in the
reference's layout.

usage: python make_quadratic_td.py <dest_root> <N> [paths] [seed]
"""
import cmath
import itertools
import os
import sys

import numpy as np
import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import p2c_gen  # noqa: E402


def system(N):
    xs = list(sp.symbols("x1:%d" % (N + 1)))
    ps = list(sp.symbols("p1:%d" % (4 * N + 1)))
    eqs = []
    for i in range(N):
        a0, a1, a2, a3 = ps[4 * i:4 * i + 4]
        eqs.append(sp.expand(a0 * xs[i] ** 2 + a1 * xs[(i + 1) % N] * xs[(i + 2) % N] + a2 * xs[(i + 3) % N] + a3))
    return xs, ps, eqs


def write(dest_root, N, paths=64, seed=0, name=None):
    name = name or "QTD_%d" % N
    dest = os.path.join(dest_root, name)
    paths = min(paths, 2 ** N)
    xs, ps, eqs = system(N)
    info = p2c_gen.generate(xs, ps, eqs)
    os.makedirs(dest, exist_ok=True)
    rng = np.random.default_rng(seed)
    g = cmath.exp(1j * rng.uniform(0, 2 * np.pi))
    yaml = """%%YAML:1.0

#> coupled quadratics by a total-degree homotopy, N = %d (generated by gen/make_quadratic_td.py)
problem_name: %s
problem_print_out_name: coupled quadratics N = %d

GPUHC_Type: P2C
GPUHC_Max_Steps: 200
GPUHC_Max_Correction_Steps: 5
GPUHC_Num_Of_Steps_to_Increase_Delta_t: 3

Num_Of_Vars: %d
Num_Of_Params: %d
Num_Of_Tracks: %d
dHdx_Max_Terms: %d
dHdx_Max_Parts: %d
dHdt_Max_Terms: %d
dHdt_Max_Parts: %d
Max_Order_Of_T: %d
Num_Of_Coeffs_From_Params: %d

RANSAC_Dataset: None
""" % (N, name, N, N, 4 * N, paths, info["Tx"], info["Px"], info["Tt"], info["Pt"], info["K"], info["M"])
    open(os.path.join(dest, "gpuhc_settings.yaml"), "w").write(yaml)
    start = []
    for i in range(N):
        start += [g, 0.0, 0.0, -g]
    target = list(rng.normal(size=4 * N))
    for fname, vals in (("start_params.txt", start), ("target_params.txt", target)):
        with open(os.path.join(dest, fname), "w") as f:
            for v in vals:
                v = complex(v)
                f.write("%.17g\t%.17g\n" % (v.real, v.imag))
    with open(os.path.join(dest, "start_sols.txt"), "w") as f:
        for k, signs in enumerate(itertools.product([1.0, -1.0], repeat=N)):
            if k == paths:
                break
            for s in signs:
                f.write("%.17g\t%.17g\n" % (s, 0.0))
    p2c_gen.write_table(os.path.join(dest, "dHdx_indx.txt"), info["hx"], info["Tx"] * info["Px"] * N)
    p2c_gen.write_table(os.path.join(dest, "dHdt_indx.txt"), info["ht"], info["Tt"] * info["Pt"])
    p2c_gen.write_p2c_terms(os.path.join(dest, "p2c_terms.txt"), info, "gen/make_quadratic_td.py")
    return dest, info


if __name__ == "__main__":
    root, N = sys.argv[1], int(sys.argv[2])
    paths = int(sys.argv[3]) if len(sys.argv) > 3 else 64
    seed = int(sys.argv[4]) if len(sys.argv) > 4 else 0
    d, info = write(root, N, paths, seed)
    print(d, "M=%d K=%d Tx=%d Px=%d Tt=%d Pt=%d" % (info["M"], info["K"], info["Tx"], info["Px"], info["Tt"],
                                                   info["Pt"]))
