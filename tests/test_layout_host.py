"""The device layout, checked on the CPU (gslam_layout_plan, no GPU).

libgslam renumbers the block rows (Cuthill-McKee for one graph, then a sort by
block count inside windows), cuts them into 32-row slices and builds, per block
slot, the list of edge contributions the assembly kernel sums. These tests read
that plan back through the C ABI and replay, in numpy, exactly what the device
kernels do with it (k_assemble, k_assemble_xi and the sliced SpMV: one IEEE add or
multiply at a time, in the plan's order). The replay must give the oracle's
Omega, xi and q = Omega p bit for bit (the reference's summation orders,
src/cpu_pcg_fp64/MatrixOps.c:224-272 and 349-353), so the host half of the
parity contract is pinned without a GPU.
"""
import numpy as np
import pytest

from conftest import assert_bitwise, load_pkg

ANCHOR = 1e6   # the reference's pose-0 anchor (MatrixOps.c:224-231)


def _plan(n, t1, t2, **kw):
    return load_pkg().abi.layout_plan(n, t1, t2, **kw)


def _slot_rows(P):
    """New row of every slot (-1 never happens: padding slots belong to a row too)."""
    sp = P["slice_ptr"]
    rows = np.empty(P["n_slots"], np.int64)
    for s in range(P["n_slices"]):
        k = np.arange(sp[s], sp[s + 1])
        rows[k] = 32 * s + (k - sp[s]) % 32
    return rows


def _row_len(P):
    rows = _slot_rows(P)
    real = P["col"] >= 0
    return np.bincount(rows[real], minlength=32 * P["n_slices"])


def _assemble(P, blocks, anchor):
    """k_assemble: per (slot, entry), +0.0, the anchor on block (0,0)'s diagonal, then
    every contribution in list order; the result scattered into the reference CSR."""
    ptr, ctr = P["ctr_ptr"], P["ctr"]
    cnt = np.diff(ptr)
    acc = np.zeros((P["n_slots"], 9))
    a = P["anchor_slot"]
    acc[a, [0, 4, 8]] = acc[a, [0, 4, 8]] + anchor
    ent = np.arange(9)
    for p in range(int(cnt.max(initial=0))):
        sl = np.nonzero(cnt > p)[0]
        code = ctr[ptr[sl] + p]
        acc[sl] = acc[sl] + blocks[(code >> 2)[:, None], (9 * (code & 3))[:, None] + ent[None, :]]
    rows = _slot_rows(P)
    rlen = _row_len(P)
    vals = np.zeros(P["csr_nnz"])
    base = P["slot_csr"]
    m = base >= 0
    for e in range(9):
        r, c = divmod(e, 3)
        vals[base[m] + r * 3 * rlen[rows[m]] + c] = acc[m, e]
    for slot in np.nonzero(base == -2)[0]:   # bare anchor: rows 0..2 hold only (d, d)
        for r in range(3):
            vals[r] = acc[slot, 4 * r]
    return acc, vals


def _assemble_xi(P, blocks):
    """k_assemble_xi: per (new row, component), contributions in list order from +0.0."""
    ptr, ctr = P["xi_ptr"], P["xi_ctr"]
    n = P["n_rows"]
    cnt = np.diff(ptr)
    acc = np.zeros((n, 3))
    for p in range(int(cnt.max(initial=0))):
        rw = np.nonzero(cnt > p)[0]
        code = ctr[ptr[rw] + p]
        acc[rw] = acc[rw] + blocks[(code >> 1)[:, None], (36 + 3 * (code & 1))[:, None] + np.arange(3)[None, :]]
    xi = np.zeros(3 * n)
    xi.reshape(n, 3)[P["perm"]] = acc
    return xi


def _spmv(P, acc, p):
    """The sliced SpMV (spmv_row): per new row, blocks in slot order, each scalar row
    q_r = ((0 + v_r0 p_0) + v_r1 p_1) + v_r2 p_2 + ... with no fused multiply-add."""
    n = P["n_rows"]
    rows = _slot_rows(P)
    rlen = _row_len(P)
    p_new = np.asarray(p).reshape(n, 3)[P["perm"]]
    q = np.zeros((n, 3))
    sp = P["slice_ptr"]
    for j in range(int(rlen.max(initial=0))):
        slot = np.array([sp[r // 32] + 32 * j + r % 32 for r in range(n) if rlen[r] > j], np.int64)
        if slot.size == 0:
            continue
        rw = rows[slot]
        pc = p_new[P["col"][slot]]
        for r in range(3):
            for c in range(3):
                q[rw, r] = q[rw, r] + acc[slot, 3 * r + c] * pc[:, c]
    out = np.zeros(3 * n)
    out.reshape(n, 3)[P["perm"]] = q
    return out


def _se2_case(oracle, n, seed, far=0.0, drop_pose0=False):
    G = load_pkg()
    cg = G.synth.city_grid(n, seed=seed, far_fraction=far)
    ei, ej, meas, lw = cg.edge_i, cg.edge_j, cg.meas, cg.log_w
    if drop_pose0:   # no edge touches pose 0: rows 0..2 hold only the anchor
        keep = (ei != 0) & (ej != 0)
        ei, ej, meas, lw = ei[keep], ej[keep], meas[keep], lw[keep]
    blocks, _ = oracle.se2_linearise(cg.init, ei, ej, meas, lw, 0.1)
    return n, ei.astype(np.uint32), ej.astype(np.uint32), blocks


def _reference_case(oracle, tmp_path, n, seed):
    G = load_pkg()
    cg = G.synth.city_grid(n, seed=seed, k_closures=3, radius=3.0)
    path = str(tmp_path / "g.txt")
    G.synth.write_log(path, G.synth.to_reference_log(cg))
    g = oracle.read_log(path)
    t1, t2, blocks = oracle.linearise(g, g.x, 1.0)
    return g.n_poses, t1, t2, blocks


def _cases(oracle, tmp_path):
    return {
        "se2_1500_far": _se2_case(oracle, 1500, 4, far=0.02),
        "se2_60_small": _se2_case(oracle, 60, 5),
        "se2_300_bare_anchor": _se2_case(oracle, 300, 6, drop_pose0=True),
        "reference_700": _reference_case(oracle, tmp_path, 700, 7),
    }


@pytest.mark.parametrize("window", [0, 1, 96])
def test_replayed_assembly_and_spmv_are_the_oracles(oracle, tmp_path, window):
    for name, (n, t1, t2, blocks) in _cases(oracle, tmp_path).items():
        P = _plan(n, t1, t2, sell_window=window)
        rp, ci, va, xi = oracle.csr_build_anchor(3 * n, t1, t2, blocks, ANCHOR)
        assert P["csr_nnz"] == len(va), name
        acc, vals = _assemble(P, blocks, ANCHOR)
        assert_bitwise(vals, va, f"{name}: Omega")
        assert_bitwise(_assemble_xi(P, blocks), xi, f"{name}: xi")
        p = np.random.default_rng(1).standard_normal(3 * n)
        assert_bitwise(_spmv(P, acc, p), oracle.spmv(rp, ci, va, p), f"{name}: Omega p")


def test_plan_invariants(oracle, tmp_path):
    for name, (n, t1, t2, blocks) in _cases(oracle, tmp_path).items():
        E = len(t1)
        for window in (0, 1, 96):
            P = _plan(n, t1, t2, sell_window=window)
            perm = P["perm"]
            assert np.array_equal(np.sort(perm), np.arange(n)), name
            # every block of the pattern once, in its row, ascending ORIGINAL column order
            keys = {(0, 0)}
            for a, b in zip(t1.tolist(), t2.tolist()):
                keys.update({(a, a), (a, b), (b, a), (b, b)})
            want = {}
            for a, b in keys:
                want.setdefault(a, []).append(b)
            sp, col = P["slice_ptr"], P["col"]
            rlen = _row_len(P)
            assert P["nnzb"] == len(keys)
            for s in range(P["n_slices"]):
                width = (sp[s + 1] - sp[s]) // 32
                assert width == rlen[32 * s: 32 * s + 32].max()
                for lane in range(32):
                    r = 32 * s + lane
                    cs = col[sp[s] + lane: sp[s + 1]: 32]
                    assert (cs[rlen[r]:] == -1).all()
                    if r < n:
                        got = perm[cs[: rlen[r]]].tolist()
                        assert got == sorted(want[int(perm[r])]), (name, r)
            # windows: rows sorted by block count, longest first
            w = 1024 if window <= 0 else window
            if w > 1:
                for w0 in range(0, n, w):
                    ln = rlen[w0: min(n, w0 + w)]
                    assert (np.diff(ln) <= 0).all(), (name, w0)
            # contribution lists: every edge's four sub-blocks once, each in its own block's
            # slot, in edge order; padding slots empty
            ptr, ctr = P["ctr_ptr"], P["ctr"]
            assert np.array_equal(np.sort(ctr), np.arange(4 * E))
            assert (np.diff(ptr)[col < 0] == 0).all()
            for slot in np.nonzero(np.diff(ptr))[0][:2000]:
                codes = ctr[ptr[slot]: ptr[slot + 1]]
                assert (np.diff(codes >> 2) > 0).all()
                r = perm[_slot_rows(P)[slot]]
                c = perm[col[slot]]
                for code in codes:
                    e, q = divmod(int(code), 4)
                    a, b = int(t1[e]), int(t2[e])
                    assert (r, c) == [(a, a), (a, b), (b, a), (b, b)][q]
            xp, xc = P["xi_ptr"], P["xi_ctr"]
            assert np.array_equal(np.sort(xc), np.arange(2 * E))
            for r in range(n):
                codes = xc[xp[r]: xp[r + 1]]
                assert (np.diff(codes) > 0).all()
                for code in codes:
                    e, wb = divmod(int(code), 2)
                    assert int((t1 if wb == 0 else t2)[e]) == perm[r]
            assert (P["slot_csr"][col < 0] == -1).all()
            assert P["bare_anchor"] == int(name.endswith("bare_anchor"))


def test_cuthill_mckee_order_is_breadth_first_and_local(oracle):
    """With the window sort off, a single graph's rows are a breadth-first order of its
    block pattern (every row after a component's first has a neighbour placed earlier),
    and the rows a 256-row range reaches outside itself (its halo) shrink against the
    input order on a walk with far loop closures."""
    n, t1, t2, _ = _se2_case(oracle, 6000, 9, far=0.02)
    P = _plan(n, t1, t2, sell_window=1)
    perm = P["perm"]
    iperm = np.empty(n, np.int64)
    iperm[perm] = np.arange(n)
    nbrs = [[] for _ in range(n)]
    for a, b in zip(t1.tolist(), t2.tolist()):
        nbrs[a].append(b)
        nbrs[b].append(a)
    starts = 0
    for pos in range(1, n):
        r = perm[pos]
        if not any(iperm[c] < pos for c in nbrs[r]):
            starts += 1
    assert starts == 0   # the walk is one component: its first row is the only start

    def halo(pos_of):
        """Median and largest count of distinct rows outside each 256-row range of an
        order that the range's rows have blocks with."""
        row_at = np.argsort(pos_of)
        sizes = []
        for c0 in range(0, n, 256):
            outside = {c for r in row_at[c0:c0 + 256] for c in nbrs[r]
                       if not c0 <= pos_of[c] < c0 + 256}
            sizes.append(len(outside))
        return np.median(sizes), max(sizes)

    med_cm, max_cm = halo(iperm)
    med_in, max_in = halo(np.arange(n))
    print(f"halo per 256 rows: input order median {med_in} max {max_in}; "
          f"Cuthill-McKee median {med_cm} max {max_cm}")
    assert med_cm <= med_in and max_cm < max_in, (med_cm, max_cm, med_in, max_in)


def test_batch_plan_keeps_each_graph_in_its_range(oracle):
    """A batch (segments at each graph's 32-aligned start, padding rows with their own
    diagonal block): rows never leave their graph's range, every slice belongs to one
    graph, and inside a window the rows keep their input order apart from the sort by
    block count (no Cuthill-McKee reordering)."""
    G = load_pkg()
    sizes = [100, 37, 700]
    t1, t2, segs, diag = [], [], [], []
    off = 0
    for k, nk in enumerate(sizes):
        cg = G.synth.city_grid(nk, seed=20 + k)
        segs.append(off)
        t1.append(cg.edge_i + off)
        t2.append(cg.edge_j + off)
        padded = (nk + 31) // 32 * 32
        diag.append(off)
        diag.extend(range(off + nk, off + padded))
        off += padded
    n = off
    t1 = np.concatenate(t1).astype(np.uint32)
    t2 = np.concatenate(t2).astype(np.uint32)
    for window in (0, 64):
        P = _plan(n, t1, t2, sell_window=window, segments=segs, diag_rows=diag)
        perm = P["perm"]
        bounds = segs + [n]
        rlen = _row_len(P)
        for q in range(len(segs)):
            a, b = bounds[q], bounds[q + 1]
            assert sorted(perm[a:b].tolist()) == list(range(a, b))
            w = 1024 if window <= 0 else window
            for w0 in range(a, b, w):
                w1 = min(b, w0 + w)
                assert (np.diff(rlen[w0:w1]) <= 0).all()
                # the stable sort of the window's input rows by block count, longest first
                count_of = {int(perm[i]): int(rlen[i]) for i in range(w0, w1)}
                assert perm[w0:w1].tolist() == sorted(range(w0, w1), key=lambda r: -count_of[r])
        for s in range(P["n_slices"]):
            g_of = np.searchsorted(bounds, perm[32 * s: 32 * s + 32], side="right") - 1
            assert (g_of == g_of[0]).all()


def test_plan_rejects_bad_input():
    G = load_pkg()
    L = G.abi.lib()
    t = np.array([0, 5], np.uint32)
    with pytest.raises(G.abi.GslamError):
        G.abi.layout_plan(3, t, t)            # pose index out of range
    with pytest.raises(G.abi.GslamError):
        G.abi.layout_plan(10, t, t, segments=[2, 5])    # first segment must start at 0
    with pytest.raises(G.abi.GslamError):
        G.abi.layout_plan(10, t, t, segments=[0, 5, 5])  # strictly ascending
    assert L.gslam_layout_plan(0, 0, None, None, 0, 0, None, 0, None, None, *([None] * 8)) == G.abi.ERR_BAD_INPUT


@pytest.mark.parametrize("n,t1,t2", [(1, [], []), (2, [0], [1]), (3, [1], [2]),
                                     (33, list(range(32)), list(range(1, 33)))],
                         ids=["one_pose_no_edges", "two_poses", "pose0_untouched", "33_rows_two_slices"])
def test_small_and_ragged_graphs(oracle, n, t1, t2):
    """Edge cases of the plan: a single pose with no edge (only the anchor block), a pose 0
    that no edge touches, a last slice with one row. Random block values: the replay is
    the same IEEE arithmetic whatever they are."""
    t1 = np.array(t1, np.uint32)
    t2 = np.array(t2, np.uint32)
    P = _plan(n, t1, t2)
    blocks = np.random.default_rng(n).standard_normal((len(t1), 42))
    rp, ci, va, xi = oracle.csr_build_anchor(3 * n, t1, t2, blocks, ANCHOR)
    acc, vals = _assemble(P, blocks, ANCHOR)
    assert_bitwise(vals, va, "Omega")
    assert_bitwise(_assemble_xi(P, blocks), xi, "xi")
    p = np.random.default_rng(2).standard_normal(3 * n)
    assert_bitwise(_spmv(P, acc, p), oracle.spmv(rp, ci, va, p), "Omega p")
    assert P["n_slices"] == (n + 31) // 32
    assert P["bare_anchor"] == int(not any(a == 0 or b == 0 for a, b in zip(t1, t2)))
