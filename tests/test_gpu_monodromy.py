"""The monodromy start-system solver on the generalized 3-view 4-point problem (needs a B200).

The reference's start system (problems/generalized_3views_4pts/start_sols.txt, 583 roots from its
Julia monodromy run) is one set of roots of the system at generic parameters; the solver here,
started from one seeded scene solution, finds 3,071.  Evidence that they are all genuine,
isolated roots of one system F(x; q) = 0: residual at rounding level, Jacobian condition numbers
far from singular, pairwise distinct, a count that further loops do not change; and the
reference's 583, continued from its start parameters to q, are all among them."""
import numpy as np
import pytest

import ghc
import monodromy
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_monodromy_roots_are_regular_distinct_and_contain_the_reference_set():
    pb = ghc.Problem("generalized_3views_4pts")
    q, Sq, S = monodromy.start_system(pb, seed=0)
    assert len(S) == len(Sq) == 3071
    ob = O.Problem("generalized_3views_4pts")
    hx, ht = O.p2c_tables(ob.terms, q, q)   # c_k(0) = c_k(q): the system F(x; q)
    worst, conds = 0.0, []
    for x in Sq:
        H, _, Hx = O.eval_system(ob, x, 0.0, hx=hx, ht=ht)
        worst = max(worst, np.abs(H).max() / max(1.0, np.abs(x).max()) ** 2)
        conds.append(np.linalg.cond(Hx))
    assert worst < 1e-12
    assert max(conds) < 1e7
    from scipy.spatial import cKDTree
    Z = np.concatenate([Sq.real, Sq.imag], axis=1)
    dist, _ = cKDTree(Z).query(Z, k=2)
    assert dist[:, 1].min() > 1e-3
    # further loops at q add nothing
    more = monodromy.monodromy_solve(pb, Sq, q, max_loops=4, stall_loops=4, seed=99)
    assert len(more) == len(Sq)
    # the reference's start system continued from its start parameters to q
    s, _ = pb.params()
    R = monodromy.track_leg(pb, pb.start_sols(), s, q, polish_iters=3)
    R = monodromy._merge(np.zeros((0, pb.N), dtype=complex), R)
    assert len(R) == 583
    for x in R:
        d = np.abs(Sq - x).max(axis=1) / max(1.0, np.abs(x).max())
        assert d.min() <= 1e-8
