"""The compiled H_x tables against the reference's index tables (no GPU).

Row block: every non-padding term of the dHdx table (GPU-HC/magmaHC/gpu-idx-evals/
dev-eval-indxing-P3P.cuh:70-84 reads it term by term) appears once, in table order, with its
scale, coefficient (or parameter pair), every variable slot including the constant slot N, its
column and the last-term-of-entry flag.  Balanced block: every entry's terms are walked by one
lane, in the same order, and stored to the entry's row and slot; the lanes' lengths are what the
walk runs.
"""
import numpy as np
import pytest

import ghc

PROBLEMS = ["P3P", "P3P_TD", "5pt_rel_pos_alg_form_quat", "generalized_3views_4pts",
            "uncalibrated_trifocal_rel_pos_CY", "trifocal_2op1p_30x30"]
LOW49 = np.uint64((1 << 49) - 1)


def width(N):
    return 4 if N <= 4 else 8 if N <= 8 else 16 if N <= 16 else 32


def raw_terms(pb, hx):
    """[(row, col, [parts])] of the non-padding terms, table order per (row, col)."""
    N, Tx, Px = pb.N, pb.Tx, pb.Px
    out = {}
    for r in range(N):
        for i in range(N):
            terms = []
            for j in range(Tx):
                if pb.kind == ghc.KIND_P2C:
                    e = [int(hx[((r * N + i) * Tx + j) * Px + q]) for q in range(Px)]
                else:
                    e = [int(hx[((i * Tx * Px) + j * Px + q) * N + r]) for q in range(Px)]
                if e[0] != 0:
                    terms.append(e)
            out[(r, i)] = terms
    return out


@pytest.mark.parametrize("name", PROBLEMS)
def test_row_block_encodes_the_reference_table(name):
    pb = ghc.Problem(name)
    N = pb.N
    words, off = pb.compiled_hx()
    hx, _ = pb.raw_tables()
    raw = raw_terms(pb, hx)
    ncs = 2 if pb.kind == ghc.KIND_PH else 1
    nv = pb.Px - 1 - ncs
    assert len(off) == N * N + 2 + width(N)
    for r in range(N):
        base = int(off[r * N])
        for i in range(N):
            j0, j1 = int(off[r * N + i]), int(off[r * N + i + 1])
            assert j1 - j0 == len(raw[(r, i)])
            for k, j in enumerate(range(j0, j1)):
                w = int(words[(j - base) * N + r])
                e = raw[(r, i)][k]
                assert ((w & 0xFF) ^ 0x80) - 0x80 == e[0]                 # scale (int8)
                assert (w >> 8) & 7 == nv                               # every slot kept
                if pb.kind == ghc.KIND_P2C:
                    assert (w >> 11) & 0x3FF == e[1]
                else:
                    assert ((w >> 11) & 0x3F, (w >> 17) & 0x3F) == (e[1], e[2])
                assert [(w >> (24 + 5 * q)) & 31 for q in range(nv)] == e[1 + ncs:]  # slot N included
                assert w >> 59 == i
                assert bool(w & (1 << 23)) == (j == j1 - 1)             # last term of its entry


@pytest.mark.parametrize("name", PROBLEMS)
def test_balanced_block_walks_every_entry_once_in_order(name):
    pb = ghc.Problem(name)
    N, W = pb.N, width(pb.N)
    words, off = pb.compiled_hx()
    first = int(off[N * N + 1])
    lens = [int(x) for x in off[N * N + 2:]]
    assert first != 0xFFFF  # built at every size
    assert sum(lens) == int(off[N * N])
    want = {}
    for r in range(N):
        base, slot = int(off[r * N]), 0
        for i in range(N):
            j0, j1 = int(off[r * N + i]), int(off[r * N + i + 1])
            if j1 > j0:
                want[(r, slot)] = [int(words[(j - base) * N + r]) for j in range(j0, j1)]
                slot += 1
    got = {}
    for l in range(W):
        cur = []
        for q in range(lens[l]):
            w = int(words[first + q * W + l])
            cur.append(w & int(LOW49))
            if w & (1 << 23):
                key = ((w >> 49) & 31, (w >> 54) & 31)
                assert key not in got
                got[key] = cur
                cur = []
        assert cur == []  # a lane ends on an entry's last term
    assert got == {k: [w & int(LOW49) for w in v] for k, v in want.items()}
    longest_row = max(int(off[r * N + N]) - int(off[r * N]) for r in range(N))
    assert max(lens) <= longest_row


def test_sizes_and_errors():
    pb = ghc.Problem("generalized_3views_4pts")
    w, o = pb.compiled_hx()
    assert int(o[pb.N * pb.N]) == pb.info.n_hx_terms == 144
    lens = [int(x) for x in o[pb.N * pb.N + 2:]]
    assert len(w) == 12 * 12 + 16 * max(lens)  # row block (12 rows x 12 terms), then the balanced block
    assert max(lens) == 9  # the 144 terms dealt to 16 lanes
