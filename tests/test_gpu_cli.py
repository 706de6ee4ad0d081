"""The command-line solver end to end (needs a B200): ``ghc-main -p <problem>``, the reference's
``magmaHC-main -p`` (GPU-HC/cmd/magmaHC-main.cpp:30-111), reads the problem folder, solves its
shipped target on the GPU, writes GPU_Converged_HC_tracks.txt in the reference's format
(Evaluations::Write_Converged_Sols, GPU-HC/magmaHC/Evaluations.cpp:66-86) and prints the
reference's counts.  The file and the counts must equal the oracle's on the same coefficient
tables (the CLI builds them on the device)."""
import os
import re
import subprocess

import numpy as np
import pytest

import ghc
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(os.path.abspath(ghc.__file__)), "ghc-main")


def cx_t(a):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).cuda()


def to_cx(t):
    a = t.double().cpu().numpy()
    return a[..., 0] + 1j * a[..., 1]


def read_tracks(path, N):
    lines = open(path).read().split("\n")
    assert lines[0] == "-------------------- RANSAC Iteration 1 --------------------"
    rows = [l.split("\t") for l in lines if len(l.split("\t")) == 2]
    z = np.array(rows, dtype=float)
    return (z[:, 0] + 1j * z[:, 1]).reshape(-1, N)


@pytest.mark.parametrize("name,prec", [("P3P", "fp64"), ("generalized_3views_4pts", "fp64"),
                                       ("trifocal_2op1p_30x30", "fp64"), ("uncalibrated_trifocal_rel_pos_CY", "fp32"),
                                       ("4view_triangulation", "fp64")])
def test_cli_matches_oracle(name, prec, tmp_path):
    run = subprocess.run([CLI, "-p", name, "--root", ghc.PROBLEMS, "--precision", prec, "-o", str(tmp_path)],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    pb, ob = ghc.Problem(name), O.Problem(name)
    f32 = prec == "fp32"
    cast = (lambda a: a.astype(np.complex64)) if f32 else (lambda a: a)
    if pb.kind == ghc.KIND_P2C:
        dhx, dht = pb.p2c_device(cx_t(ob.start_params), cx_t(ob.target_params[None]))
        torch.cuda.synchronize()
        kw = dict(hx=cast(to_cx(dhx)), ht=cast(to_cx(dht)[:, :(pb.M + 1) * pb.K]))
    else:
        kw = dict(p_start=cast(ob.start_params), p_target=cast(ob.target_params[None]))
    r = O.track(ob, cast(ob.start_sols), precision="f" if f32 else "d", nthreads=os.cpu_count() or 1, **kw)
    G = read_tracks(os.path.join(str(tmp_path), "GPU_Converged_HC_tracks.txt"), pb.N)
    assert np.array_equal(G, r["endpoints"][r["conv"] == 1])
    c = O.count_results(r["endpoints"], r["conv"], r["inf"])
    got = {k: int(re.search(r"Number of %s Solutions:\s+(\d+)" % lab, run.stdout).group(1))
           for k, lab in (("converged", "Converged"), ("real", "Real"), ("infinity", "Infinity Failed"),
                          ("unique", "Unique"))}
    assert got == c


def test_cli_missing_problem_fails(tmp_path):
    run = subprocess.run([CLI, "-p", "no_such_problem", "--root", ghc.PROBLEMS, "-o", str(tmp_path)],
                         capture_output=True, text=True, timeout=60)
    assert run.returncode != 0 and "DATA LOAD ERROR" in run.stderr
