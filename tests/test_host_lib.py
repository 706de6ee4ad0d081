"""Host side of the C ABI (no GPU): symbols, loaders, P2C, counts, error paths, CLI."""
import ctypes
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import ghc
import oracle as O

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "ghc.h")
PROBLEMS = sorted(os.listdir(ghc.PROBLEMS))


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:ghc_|kernel_HC_Solver)\w*)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert len(names) >= 15
    lib = ctypes.CDLL(ghc.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("name", PROBLEMS)
def test_loader_matches_oracle_reader(name):
    pb = ghc.Problem(name)
    ob = O.Problem(name)
    assert (pb.kind, pb.N, pb.P, pb.M, pb.K, pb.paths) == (ob.kind, ob.N, ob.P, ob.M, ob.K, ob.paths)
    assert (pb.max_steps, pb.max_corr, pb.incr_steps) == (ob.max_steps, ob.max_corr, ob.incr)
    assert np.array_equal(pb.start_sols(), ob.start_sols)
    s, t = pb.params()
    assert np.array_equal(s, ob.start_params) and np.array_equal(t, ob.target_params)
    hx, ht = pb.raw_tables()
    assert np.array_equal(hx, ob.hx_idx) and np.array_equal(ht, ob.ht_idx)
    # compiled terms: one per non-padding table term
    if pb.kind == ghc.KIND_P2C:
        assert pb.n_hx_terms == int((ob.hx_idx.reshape(-1, ob.Px)[:, 0] != 0).sum())
        assert pb.n_ht_terms == int((ob.ht_idx.reshape(-1, ob.Pt)[:, 0] != 0).sum())
    else:
        assert pb.n_hx_terms == int((ob.hx_idx.reshape(ob.N, ob.Tx, ob.Px, ob.N)[:, :, 0, :] != 0).sum())
        assert pb.n_ht_terms == int((ob.ht_idx.reshape(ob.Tt, ob.Pt, ob.N)[:, 0, :] != 0).sum())


@pytest.mark.parametrize("name", [p for p in PROBLEMS if p != "trifocal_2op1p_30x30"])
@pytest.mark.parametrize("exact", [False, True])
def test_host_p2c_matches_oracle(name, exact):
    pb = ghc.Problem(name)
    ob = O.Problem(name)
    rng = np.random.default_rng(7)
    tgt = np.append(rng.normal(size=pb.P) + 1j * rng.normal(size=pb.P), 1.0)
    hx, ht = pb.p2c(ob.start_params, tgt, exact_ht=exact)
    ohx, oht = O.p2c_tables(ob.terms, ob.start_params, tgt, exact_ht=exact)
    assert np.allclose(hx, ohx, rtol=1e-13, atol=1e-13 * np.abs(ohx).max())
    assert np.allclose(ht, oht, rtol=1e-13, atol=1e-13 * max(1, np.abs(oht).max()))


def test_count_results_matches_oracle_on_golden():
    rows = [l.split() for l in open(os.path.join(REPO, "tests", "golden", "cy_golden_tracks.txt")) if len(l.split()) == 2]
    g = np.array(rows, dtype=float)
    G = (g[:, 0] + 1j * g[:, 1]).reshape(-1, 12)
    one = np.ones(len(G), np.uint8)
    zero = np.zeros(len(G), np.uint8)
    assert ghc.count_results(G, one, zero) == dict(converged=444, real=0, infinity=0, unique=441)


def test_count_results_matches_oracle_random_clusters():
    rng = np.random.default_rng(11)
    base = rng.normal(size=(20, 4)) + 1j * rng.normal(size=(20, 4))
    base[:5] = base[:5].real  # some real solutions
    idx = rng.integers(0, 20, size=60)
    z = base[idx] + 1e-6 * rng.normal(size=(60, 4))
    conv = (rng.random(60) > 0.2).astype(np.uint8)
    inf = ((1 - conv) * (rng.random(60) > 0.5)).astype(np.uint8)
    assert ghc.count_results(z, conv, inf) == O.count_results(z, conv, inf)


def _copy_problem(tmp_path, name="P3P"):
    dst = tmp_path / name
    shutil.copytree(os.path.join(ghc.PROBLEMS, name), dst)
    return dst


def test_error_missing_problem(tmp_path):
    with pytest.raises(ghc.GhcError, match=r"\(-2\)"):
        ghc.Problem("no_such_problem", root=str(tmp_path))


def test_error_malformed_yaml(tmp_path):
    d = _copy_problem(tmp_path)
    text = open(d / "gpuhc_settings.yaml").read().replace("Num_Of_Vars: 3", "Num_Of_Vars: three")
    open(d / "gpuhc_settings.yaml", "w").write(text)
    with pytest.raises(ghc.GhcError, match=r"\(-3\)"):
        ghc.Problem("P3P", root=str(tmp_path))


def test_error_table_index_out_of_range(tmp_path):
    d = _copy_problem(tmp_path)
    vals = open(d / "dHdx_indx.txt").read().split()
    vals[1] = "77"  # coefficient index beyond M
    open(d / "dHdx_indx.txt", "w").write(" ".join(vals))
    with pytest.raises(ghc.GhcError, match=r"\(-4\)"):
        ghc.Problem("P3P", root=str(tmp_path))


def test_error_term_scale_outside_int8(tmp_path):
    d = _copy_problem(tmp_path)
    vals = open(d / "dHdx_indx.txt").read().split()
    vals[0] = "300"  # the first term's integer scale: the term word holds it in 8 bits
    open(d / "dHdx_indx.txt", "w").write(" ".join(vals))
    with pytest.raises(ghc.GhcError, match=r"\(-4\).*int8"):
        ghc.Problem("P3P", root=str(tmp_path))


def test_error_variable_index_out_of_range(tmp_path):
    d = _copy_problem(tmp_path)
    vals = open(d / "dHdx_indx.txt").read().split()
    vals[2] = "9"  # the first term's variable slot: beyond N (slot N = 3 is the constant 1)
    open(d / "dHdx_indx.txt", "w").write(" ".join(vals))
    with pytest.raises(ghc.GhcError, match=r"\(-4\).*variable"):
        ghc.Problem("P3P", root=str(tmp_path))


def test_error_truncated_table(tmp_path):
    d = _copy_problem(tmp_path)
    vals = open(d / "dHdt_indx.txt").read().split()
    open(d / "dHdt_indx.txt", "w").write(" ".join(vals[:-3]))
    with pytest.raises(ghc.GhcError, match=r"\(-3\)"):
        ghc.Problem("P3P", root=str(tmp_path))


def test_error_truncated_start_sols(tmp_path):
    d = _copy_problem(tmp_path)
    lines = open(d / "start_sols.txt").read().splitlines()
    open(d / "start_sols.txt", "w").write("\n".join(lines[:5]))
    with pytest.raises(ghc.GhcError, match=r"\(-3\)"):
        ghc.Problem("P3P", root=str(tmp_path))


def test_error_too_many_unknowns(tmp_path):
    d = _copy_problem(tmp_path)
    text = open(d / "gpuhc_settings.yaml").read().replace("Num_Of_Vars: 3", "Num_Of_Vars: 40")
    open(d / "gpuhc_settings.yaml", "w").write(text)
    with pytest.raises(ghc.GhcError, match=r"\(-4\)"):
        ghc.Problem("P3P", root=str(tmp_path))


def test_target_params_missing_is_allowed(tmp_path):
    d = _copy_problem(tmp_path)
    os.remove(d / "target_params.txt")
    pb = ghc.Problem("P3P", root=str(tmp_path))
    s, t = pb.params()
    assert t[-1] == 1 and np.all(t[:-1] == 0)


def test_cli_help_and_missing_problem():
    exe = os.path.join(os.path.dirname(ghc.LIB_PATH), "ghc-main")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "-p" in r.stdout
    r = subprocess.run([exe, "-p", "no_such_problem"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "DATA LOAD ERROR" in r.stderr


def test_tuning_setters_validate():
    pb = ghc.Problem("generalized_3views_4pts")
    assert ghc.get_tuning(pb, ghc.PREC_FP64) == (0, -1)
    ghc.set_tuning(pb, ghc.PREC_MIXED, 1, 0)
    assert ghc.get_tuning(pb, ghc.PREC_FP64) == (1, 0) and ghc.get_tuning(pb, ghc.PREC_FP32) == (1, 0)
    ghc.set_tuning(pb, ghc.PREC_FP32, 0, 1)
    assert ghc.get_tuning(pb, ghc.PREC_FP64) == (1, 0) and ghc.get_tuning(pb, ghc.PREC_FP32) == (0, 1)
    ghc.set_tuning(pb, ghc.PREC_FP64, 0, 2)
    assert ghc.get_tuning(pb, ghc.PREC_FP64) == (0, 2)
    for bad in [(ghc.PREC_FP64, 2, 0), (ghc.PREC_FP64, 0, 3), (ghc.PREC_FP64, 0, -2), (7, 0, 0)]:
        with pytest.raises(ghc.GhcError):
            ghc.set_tuning(pb, *bad)


def test_no_alloc_rejects_tables_beyond_its_fixed_array(tmp_path):
    """ghc_track_noalloc keeps the compiled tables in a fixed 64 KiB device array: a problem whose
    tables need more is rejected with GHC_ERR_LIMIT (-8) and a message naming the sizes, before any
    device work (the pointers below are never used) and without binding the handle to a device."""
    import ctypes
    N, Tx, Px, Tt, Pt, M, P, paths = 18, 30, 3, 1, 4, 40, 40, 2
    d = tmp_path / "DENSE_18"
    d.mkdir()
    (d / "gpuhc_settings.yaml").write_text(
        "problem_name: DENSE_18\nGPUHC_Type: P2C\nGPUHC_Max_Steps: 10\nGPUHC_Max_Correction_Steps: 3\n"
        "GPUHC_Num_Of_Steps_to_Increase_Delta_t: 2\nNum_Of_Vars: %d\nNum_Of_Params: %d\nNum_Of_Tracks: %d\n"
        "dHdx_Max_Terms: %d\ndHdx_Max_Parts: %d\ndHdt_Max_Terms: %d\ndHdt_Max_Parts: %d\nMax_Order_Of_T: 1\n"
        "Num_Of_Coeffs_From_Params: %d\n" % (N, P, paths, Tx, Px, Tt, Pt, M))
    pairs = "".join("%d 0\n" % (k + 1) for k in range(P))
    (d / "start_params.txt").write_text(pairs)
    (d / "target_params.txt").write_text(pairs)
    (d / "start_sols.txt").write_text("1 0\n" * (N * paths))
    hx = [[1, k % M, k % (N + 1)] for k in range(N * N * Tx)]   # every term a real (non-padding) term
    (d / "dHdx_indx.txt").write_text("\n".join(" ".join(map(str, t)) for t in hx) + "\n")
    ht = [[1, r % M, r % N, N] for r in range(N * Tt)]
    (d / "dHdt_indx.txt").write_text("\n".join(" ".join(map(str, t)) for t in ht) + "\n")
    pb = ghc.Problem("DENSE_18", root=str(tmp_path))
    a = ghc.TrackArgs()
    a.n_hyp, a.precision = 1, ghc.PREC_FP64
    a.d_start_sols = a.d_endpoints = a.d_coef_hx = a.d_coef_ht = 256
    rc = ghc.ghc_track_noalloc(pb.h, ctypes.byref(a), None)
    assert rc == -8
    msg = ghc.ghc_last_error().decode()
    assert "65536" in msg and "ghc_track" in msg
    assert pb.bound_device() == -1


def test_serve_admission_rule():
    """Live admission: a batch starts only if its transient coefficient tables leave the reserve free."""
    import serve
    pb = ghc.Problem("generalized_3views_4pts")
    need = serve.transient_bytes(pb, 100)
    assert need == 16 * 100 * (pb.M + 1) * (2 * pb.K + 1)
    assert serve.transient_bytes(ghc.Problem("trifocal_2op1p_30x30"), 100) == 0  # PH: slot buffers only
    assert serve.admit(need + 1000, need, 1000) and not serve.admit(need + 999, need, 1000)
