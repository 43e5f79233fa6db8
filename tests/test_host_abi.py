"""CPU-side checks of libgslam: it loads, exports every declared entry point, and
its host-only integer work (log parsing, edge order, CSR pattern) is bit-exact
against the oracle and the reference build. No compute call needs a GPU here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, assert_bitwise, load_pkg, ref_data


def _declared_functions():
    names = set()
    for h in ("gslam.h", "gslam_dropin.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", src, flags=re.M):
            if m.group(1) not in ("if", "sizeof", "defined"):
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    G = load_pkg()
    L = G.abi.lib()
    declared = _declared_functions()
    assert len(declared) >= 30
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert set(G.abi.EXPORTS) <= declared | {"gslam_dropin_status"}
    assert b"sm_100a" in L.gslam_version()


def _oracle_graph_from(log, oracle):
    return oracle.Graph(log.delta, log.u_step, log.u, log.x_step, log.x, log.z_step, log.z_lm, log.z)


@pytest.mark.parametrize("n,seed", [(150, 1), (600, 2)])
def test_log_reader_matches_oracle(oracle, tmp_path, n, seed):
    G = load_pkg()
    cg = G.synth.city_grid(n, seed=seed)
    path = str(tmp_path / "g.txt")
    G.synth.write_log(path, G.synth.to_reference_log(cg))
    a = G.read_log(path)
    b = oracle.read_log(path)
    assert a.delta == b.delta
    for k in ("u_step", "x_step", "z_step", "z_lm"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    for k in ("u", "x", "z"):
        assert_bitwise(getattr(a, k), getattr(b, k), k)


def test_log_reader_reference_file(oracle):
    G = load_pkg()
    path = ref_data("cityTrees800.txt")
    a, b = G.read_log(path), oracle.read_log(path)
    assert_bitwise(a.x, b.x, "x")
    assert_bitwise(a.z, b.z, "z")
    assert np.array_equal(a.z_lm, b.z_lm)


def test_log_reader_errors(tmp_path):
    G = load_pkg()
    with pytest.raises(G.abi.GslamError):
        G.read_log(str(tmp_path / "missing.txt"))
    p = tmp_path / "trunc.txt"
    p.write_text("delta 1.0\nu 0 0.0 0.0\nx 0 0.0 0.0\n")
    with pytest.raises(G.abi.GslamError):
        G.read_log(str(p))


def _edge_order(z_lm):
    G = load_pkg()
    L = G.abi.lib()
    z_lm = np.ascontiguousarray(z_lm, np.uint32)
    n = C.c_int64()
    G.abi.check(L.gslam_obs_edge_order(len(z_lm), G.abi.ptr(z_lm, C.c_uint32), None, None, 0, C.byref(n)))
    pj = np.zeros(max(n.value, 1), np.uint32)
    pk = np.zeros(max(n.value, 1), np.uint32)
    G.abi.check(L.gslam_obs_edge_order(len(z_lm), G.abi.ptr(z_lm, C.c_uint32), G.abi.ptr(pj, C.c_uint32),
                                       G.abi.ptr(pk, C.c_uint32), n.value, C.byref(n)))
    return pj[:n.value], pk[:n.value]


def test_edge_order_matches_oracle():
    import oracle as O
    rng = np.random.default_rng(4)
    for trial in range(20):
        z_lm = rng.integers(0, rng.integers(1, 40), size=rng.integers(0, 120)).astype(np.uint32)
        a = _edge_order(z_lm)
        b = O.obs_pairs(z_lm)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_edge_order_matches_reference_make_edges(oracle):
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    g = oracle.read_log(ref_data("cityTrees800.txt"))
    t1, t2, *_ = oracle.ref_round(g, g.x, 0.1)
    pj, pk = _edge_order(g.z_lm)
    n_obs = len(pj)
    assert np.array_equal(g.z_step[pj], t1[:n_obs]) and np.array_equal(g.z_step[pk], t2[:n_obs])


def _pattern(n_poses, t1, t2):
    G = load_pkg()
    L = G.abi.lib()
    t1 = np.ascontiguousarray(t1, np.uint32)
    t2 = np.ascontiguousarray(t2, np.uint32)
    nnz = C.c_int64()
    G.abi.check(L.gslam_csr_pattern(n_poses, len(t1), G.abi.ptr(t1, C.c_uint32), G.abi.ptr(t2, C.c_uint32),
                                    None, None, C.byref(nnz)))
    rp = np.zeros(3 * n_poses + 1, np.int32)
    ci = np.zeros(max(nnz.value, 1), np.int32)
    G.abi.check(L.gslam_csr_pattern(n_poses, len(t1), G.abi.ptr(t1, C.c_uint32), G.abi.ptr(t2, C.c_uint32),
                                    G.abi.ptr(rp, C.c_int), G.abi.ptr(ci, C.c_int), C.byref(nnz)))
    return rp, ci[:nnz.value]


@pytest.mark.parametrize("case", ["chain", "random", "bare_anchor", "single_pose", "self_loops"])
def test_csr_pattern_matches_oracle(oracle, case):
    rng = np.random.default_rng(hash(case) % 1000)
    if case == "chain":
        n = 50; t1 = np.arange(n - 1); t2 = t1 + 1
    elif case == "random":
        n = 80; t1 = rng.integers(0, n, 300); t2 = rng.integers(0, n, 300)
    elif case == "bare_anchor":
        n = 10; t1 = np.array([3, 4, 5]); t2 = np.array([4, 9, 5])
    elif case == "single_pose":
        n = 1; t1 = np.zeros(0); t2 = np.zeros(0)
    else:
        n = 6; t1 = np.array([0, 2, 2, 5]); t2 = np.array([1, 2, 3, 5])
    rp, ci = _pattern(n, t1, t2)
    rp2, ci2, _, _ = oracle.csr_build(3 * n, np.asarray(t1, np.uint32), np.asarray(t2, np.uint32),
                                      np.zeros((len(t1), 42)))
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2)


def test_csr_pattern_matches_reference_build(oracle):
    if not oracle.ref_available():
        pytest.skip("reference build absent")
    g = oracle.read_log(ref_data("cityTrees800.txt"))
    t1, t2, _, (rp, ci, _), _, _ = oracle.ref_round(g, g.x, 0.1)
    rp2, ci2 = _pattern(g.n_poses, t1, t2)
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2)


def test_csr_pattern_rejects_bad_edges():
    G = load_pkg()
    with pytest.raises(G.abi.GslamError):
        _pattern(5, [0, 7], [1, 2])


def test_cli_usage_and_header_match_the_reference_program(oracle, tmp_path):
    """The GSLAM program's argument handling and the two lines it prints before the first
    round (argument echo; delta and record counts, src/cpu_pcg_fp64/GSLAM.c:13-50) are the
    reference program's, byte for byte; both reject a wrong argument count with their usage
    line and exit status 1. (Runs one round: on a machine without a GPU our program stops
    there with an error, which this test does not look at.)"""
    import subprocess
    G = load_pkg()
    ref_exe = os.path.join(ROOT, "oracle", "_ref", "GSLAM")
    if not os.path.exists(ref_exe):
        pytest.skip("reference build absent (oracle/_ref)")
    cg = G.synth.city_grid(120, seed=4)
    path = str(tmp_path / "walk.txt")
    G.synth.write_log(path, G.synth.to_reference_log(cg))
    ours, ref = G.abi.CLI_PATH, ref_exe
    for args in ([], ["1", "0.1"]):
        a = subprocess.run([ours, *args], capture_output=True, text=True, timeout=60)
        b = subprocess.run([ref, *args], capture_output=True, text=True, timeout=60)
        assert a.returncode == b.returncode == 1
        assert a.stdout.replace(ours, "GSLAM") == b.stdout.replace(ref, "GSLAM")
    env = dict(os.environ, POSE_DUMP_FILE=str(tmp_path / "dump.txt"))
    a = subprocess.run([ours, "1", "0.1", "1", "0", path], capture_output=True, text=True, timeout=300, env=env)
    b = subprocess.run([ref, "1", "0.1", "1", "0", path], capture_output=True, text=True, timeout=300, env=env)
    assert a.stdout.splitlines()[:2] == b.stdout.splitlines()[:2]
    assert a.returncode in (0, 1) and b.returncode == 0


def test_entry_points_validate_arguments_before_the_gpu():
    """Bad arguments come back as status codes before any CUDA call (so these run without a
    GPU): null or empty inputs and out-of-range indices as GSLAM_ERR_BAD_INPUT, sizes past a
    fixed capacity as GSLAM_ERR_TOO_LARGE, each with a message in gslam_last_error."""
    G = load_pkg()
    A = G.abi
    L = A.lib()
    out = C.c_void_p()
    one = np.zeros(3)
    idx = np.array([0, 7], np.uint32)
    meas = np.zeros((2, 3))
    se2 = lambda n, ei, ej, ne: A.SE2GraphDesc(n, A.ptr(one), ne, A.ptr(ei, C.c_uint32),  # noqa: E731
                                               A.ptr(ej, C.c_uint32), A.ptr(meas), A.ptr(meas), 0.1, 1e6)
    assert L.gslam_create_se2(None, None, C.byref(out)) == A.ERR_BAD_INPUT
    assert L.gslam_create_se2(C.byref(se2(0, idx, idx, 0)), None, C.byref(out)) == A.ERR_BAD_INPUT
    assert L.gslam_create_se2(C.byref(se2(5, idx, idx, 2)), None, C.byref(out)) == A.ERR_BAD_INPUT
    assert b"out of range" in L.gslam_last_error()
    assert L.gslam_create_se2(C.byref(se2(0x40000000, idx, idx, 0)), None, C.byref(out)) == A.ERR_TOO_LARGE
    assert out.value is None
    # a batch: a graph without poses, an edge out of range, a non-positive lambda
    g_ok = se2(8, idx, idx, 2)
    for bad in (se2(0, idx, idx, 0), se2(5, idx, idx, 2)):
        arr = (A.SE2GraphDesc * 2)(g_ok, bad)
        assert L.gslam_create_se2_batch(arr, 2, None, C.byref(out)) == A.ERR_BAD_INPUT
    neg = se2(8, idx, idx, 2)
    neg.lam = -1.0
    assert L.gslam_create_se2_batch((A.SE2GraphDesc * 1)(neg), 1, None, C.byref(out)) == A.ERR_BAD_INPUT
    assert b"lambda" in L.gslam_last_error()
    assert L.gslam_create_se2_batch(None, 0, None, C.byref(out)) == A.ERR_BAD_INPUT
    # the reference's factor family: an observation step past the poses
    u = np.zeros((4, 2))
    steps = np.array([9], np.uint32)
    rd = A.ReferenceGraphDesc(4, A.ptr(np.zeros((4, 3))), A.ptr(u), 1.0, 1.0, A.ptr(np.zeros(4)), 1,
                              A.ptr(steps, C.c_uint32), A.ptr(steps, C.c_uint32), A.ptr(np.zeros((1, 2))))
    assert L.gslam_create_reference(C.byref(rd), None, C.byref(out)) == A.ERR_BAD_INPUT
    # dense path and the allocation-free solve (pointers are never dereferenced)
    dummy = C.c_void_p(16)
    assert L.gslam_gj_inverse(0, dummy, 0, None, None) == A.ERR_BAD_INPUT
    assert L.gslam_gj_solve(4, dummy, 2, dummy, dummy, None, None) == A.ERR_BAD_INPUT
    assert L.gslam_pcg_solve_static(7, dummy, dummy, dummy, dummy, dummy, 1e-6, 10, None, None) == A.ERR_BAD_INPUT
    assert L.gslam_pcg_solve_static(3 * 16385, dummy, dummy, dummy, dummy, dummy, 1e-6, 10, None,
                                    None) == A.ERR_TOO_LARGE
    assert b"16384" in L.gslam_last_error()
