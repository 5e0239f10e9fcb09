"""CPU oracle pinned against the reference's own outputs (golden fixtures made
by tests/golden/make_golden.py from the reference's compiled host code) and
against independent brute-force checks.  No GPU needed."""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALGO_FIX = sorted(glob.glob(os.path.join(GOLD, "ref_algos_*.npz")))
PMA_FIX = sorted(glob.glob(os.path.join(GOLD, "ref_pma_*.npz")))


def _src_ids(row):
    return np.repeat(np.arange(len(row) - 1, dtype=np.uint32), np.diff(row).astype(np.int64))


def test_fixtures_present():
    assert len(ALGO_FIX) >= 4 and len(PMA_FIX) >= 3


@pytest.mark.parametrize("path", ALGO_FIX, ids=os.path.basename)
def test_sssp_matches_reference_host(path):
    """SSSPHostNaive (hybrid_sssp_host.cu:35-63): FIFO restatement bit-exact,
    and Dijkstra on the same (u+v)%128 weights gives the same distances."""
    f = np.load(path)
    nv, row, col = int(f["nv"]), f["row"], f["col"]
    w = ((_src_ids(row) + col) % 128).astype(np.uint32)
    for k in f.files:
        if not k.startswith("sssp_"):
            continue
        s = int(k.split("_")[1])
        ref = f[k]
        d_fifo, _ = O.sssp_fifo(nv, row, col, None, s)
        assert np.array_equal(d_fifo, ref)
        d, _ = O.sssp(nv, row, col, w, s)
        assert np.array_equal(d, ref)


@pytest.mark.parametrize("path", ALGO_FIX, ids=os.path.basename)
def test_bfs_matches_reference_host(path):
    """BFSHost (hybrid_bfs_host.cpp:33-60)."""
    f = np.load(path)
    nv, row, col = int(f["nv"]), f["row"], f["col"]
    for k in f.files:
        if not k.startswith("bfs_"):
            continue
        s = int(k.split("_")[1])
        d, _ = O.bfs(nv, row, col, s)
        assert np.array_equal(d, f[k])
        d2, _ = O.bfs_fifo(nv, row, col, s)
        assert np.array_equal(d2, f[k])


@pytest.mark.parametrize("path", ALGO_FIX, ids=os.path.basename)
def test_pagerank_matches_reference_host(path):
    """PageRankHost (hybrid_pr_host.cu:43-124): the float restatement is
    bit-exact; the FP64 fixed point agrees within the float path's error."""
    f = np.load(path)
    nv, row, col = int(f["nv"]), f["row"], f["col"]
    ref = f["pr"]
    assert np.array_equal(O.pr_host_float(nv, row, col, 0.85, 1e-6), ref)
    x = O.pagerank(nv, row, col)
    rel = np.abs(ref.astype(np.float64) - x) / x
    assert rel.max() < 1e-4


@pytest.mark.parametrize("path", PMA_FIX, ids=os.path.basename)
def test_snapshot_apply_matches_reference_pma(path):
    """host::PMAGraph insert + del_edge (csr_graph.cuh:658-811) per snapshot.

    apply_refexact reproduces the reference bit for bit (same lists, same
    order).  apply (the engine's semantics: delete removes every copy) agrees
    with it everywhere except where the reference's del_edge index slip
    leaves one of two adjacent copies of a deleted edge behind; the fixtures
    contain such cases on purpose and the difference is exactly those copies.
    """
    from collections import Counter

    f = np.load(path)
    nv, row, col = int(f["nv"]), f["row"], f["col"]
    r_all, c_all = row, col
    ever_deleted = set()
    for k in range(int(f["nsnap"])):
        ins, de = f[f"ins_{k}"], f[f"del_{k}"]
        row, col = O.apply_refexact(nv, row, col, ins[:, 0], ins[:, 1], de[:, 0], de[:, 1])
        assert np.array_equal(row, f[f"row_{k}"])
        assert np.array_equal(col, f[f"col_{k}"])
        r_all, c_all, _ = O.apply(nv, r_all, c_all, None, ins[:, 0], ins[:, 1], None,
                                  de[:, 0], de[:, 1])
        ever_deleted |= set(zip(de[:, 0].tolist(), de[:, 1].tolist()))
        for v in range(nv):
            ref_c = Counter(col[row[v]:row[v + 1]].tolist())
            all_c = Counter(c_all[r_all[v]:r_all[v + 1]].tolist())
            assert not (all_c - ref_c)
            assert all((v, x) in ever_deleted for x in (ref_c - all_c))


def test_readme_known_answers():
    """The 5-vertex example of the reference README (README.md:68-96), with
    the reference's synthesized weights (u+v)%128+1; values worked by hand."""
    src = np.array([0, 0, 1, 1, 2, 3], np.uint32)
    dst = np.array([1, 2, 2, 3, 4, 4], np.uint32)
    row, col, _ = O.csr_file_order(5, src, dst)
    w = ((_src_ids(row) + col) % 128 + 1).astype(np.uint32)
    d, p = O.sssp(5, row, col, w, 0)
    assert d.tolist() == [0, 2, 3, 7, 10]
    assert p.tolist() == [O.INF, 0, 0, 1, 2]
    b, bp = O.bfs(5, row, col, 0)
    assert b.tolist() == [0, 1, 1, 2, 2]
    assert bp.tolist() == [O.INF, 0, 0, 1, 2]
    assert O.cc(5, row, col).tolist() == [0, 0, 0, 0, 0]
    x = O.pagerank(5, row, col)
    hand = [0.15, 0.21375, 0.30459375, 0.24084375, 0.613621875]
    assert np.allclose(x, hand, atol=1e-12)
    # snapshot 0: +{03,04} -{01,02,12}; snapshot 1: +{14,23} -{13,24,34}
    r1, c1, _ = O.apply(5, row, col, None, [0, 0], [3, 4], None, [0, 0, 1], [1, 2, 2])
    w1 = ((_src_ids(r1) + c1) % 128 + 1).astype(np.uint32)
    assert O.sssp(5, r1, c1, w1, 0)[0].tolist() == [0, O.INF, O.INF, 4, 5]
    assert O.cc(5, r1, c1).tolist() == [0, 1, 2, 0, 0]
    r2, c2, _ = O.apply(5, r1, c1, None, [1, 2], [4, 3], None, [1, 2, 3], [3, 4, 4])
    assert sorted(zip(_src_ids(r2).tolist(), c2.tolist())) == [(0, 3), (0, 4), (1, 4), (2, 3)]
    assert O.cc(5, r2, c2).tolist() == [0, 1, 2, 0, 0]
    assert O.bfs(5, r2, c2, 0)[0].tolist() == [0, O.INF, O.INF, 1, 1]


def _reach_min_label(nv, row, col):
    lab = np.full(nv, O.INF, np.uint32)
    for r in range(nv):
        seen = {r}
        st = [r]
        while st:
            u = st.pop()
            for e in range(row[u], row[u + 1]):
                v = int(col[e])
                if v not in seen:
                    seen.add(v)
                    st.append(v)
        for v in seen:
            lab[v] = min(lab[v], r)
    return lab


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_cc_oracle_brute_force(seed):
    nv, row, col = O.rmat_csr(7, 4, seed)
    assert np.array_equal(O.cc(nv, row, col), _reach_min_label(nv, row, col))


@pytest.mark.parametrize("seed", [1, 2])
def test_pagerank_oracle_dense_solve(seed):
    nv, row, col = O.rmat_csr(7, 8, seed)
    A = np.zeros((nv, nv))
    deg = np.diff(row).astype(np.float64)
    for u in range(nv):
        for e in range(row[u], row[u + 1]):
            A[col[e], u] += 1.0 / deg[u]
    x_ref = np.linalg.solve(np.eye(nv) - 0.85 * A, np.full(nv, 0.15))
    x = O.pagerank(nv, row, col)
    assert np.max(np.abs(x - x_ref)) < 1e-10


@pytest.mark.parametrize("seed", [3, 4])
def test_pagerank_warm_start_and_stop_rule(seed):
    """The algebra of the engine's PageRank rounds, restated on the CPU: from
    any x0 (here the fixed point of the graph before a snapshot), residual
    r0 = (1-a) + a P^T x0 - x0, then rounds x += r, r <- a P^T r (absorb and
    sweep) until sum|r| < tol reach the fixed point of the new graph within
    tol / (1 - a) in L-inf, in fewer rounds than a start from x = 0,
    r = 1 - a; signed residuals included."""
    import scipy.sparse as sp

    a, tol = 0.85, 1.5e-7
    nv, row, col = O.rmat_csr(10, 8, seed)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, seed, 200, 200)
    row2, col2, _ = O.apply(nv, row, col, None, i_s, i_d, None, d_s, d_d)

    def pt(r_, c_):
        src = np.repeat(np.arange(nv), np.diff(r_.astype(np.int64)))
        deg = np.diff(r_.astype(np.int64)).astype(np.float64)
        val = 1.0 / deg[src]
        return sp.csr_matrix((val, (c_.astype(np.int64), src)), shape=(nv, nv))

    P2 = pt(row2, col2)

    def rounds(x, r):
        k = 0
        while True:
            l1 = np.abs(r).sum()
            x = x + r
            k += 1
            if l1 < tol:
                return x, k
            r = a * (P2 @ r)

    x_old = O.pagerank(nv, row, col)
    x_new = O.pagerank(nv, row2, col2)
    xw, kw = rounds(x_old.copy(), (1 - a) + a * (P2 @ x_old) - x_old)
    xc, kc = rounds(np.zeros(nv), np.full(nv, 1 - a))
    assert np.max(np.abs(xw - x_new)) <= tol / (1 - a)
    assert np.max(np.abs(xc - x_new)) <= tol / (1 - a)
    assert kw < kc


@pytest.mark.parametrize("seed", [5, 6, 7])
def test_incremental_sssp_repair_strategies(seed):
    """The engine's incremental SSSP after a snapshot, restated on the CPU:
    parent-tree invalidation of the deleted tree edges (every descendant
    reset), then either the reference's re-push from every reached vertex or
    the pull over the in-edges of the reset vertices plus the inserted edges,
    then rounds from the vertices that improved.  Both reach the distances of
    a from-scratch run on the new graph."""
    INF = 0xFFFFFFFF
    nv, row, col = O.rmat_csr(9, 8, seed)
    w = O.weights(nv, row, col, seed, 0)
    d0, p0 = O.sssp(nv, row, col, w, 0)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, seed, 150, 150)
    iw = np.array([O.weight_of(seed, u, v) for u, v in zip(i_s, i_d)], np.uint32)
    row2, col2, w2 = O.apply(nv, row, col, w, i_s, i_d, iw, d_s, d_d)
    want, _ = O.sssp(nv, row2, col2, w2, 0)

    src2 = np.repeat(np.arange(nv), np.diff(row2.astype(np.int64)))

    def relax_rounds(d, frontier):
        d = d.copy()
        while frontier:
            nxt = set()
            for u in frontier:
                if d[u] == INF:
                    continue
                for e in range(int(row2[u]), int(row2[u + 1])):
                    v, c = int(col2[e]), int(d[u]) + int(w2[e])
                    if c < d[v]:
                        d[v] = c
                        nxt.add(v)
            frontier = nxt
        return d

    # invalidation: deleted tree edges reset their child and its subtree
    d = d0.astype(np.int64).copy()
    par = p0.astype(np.int64)
    deleted = set(zip(d_s.tolist(), d_d.tolist()))
    children = {}
    for v in range(nv):
        if d0[v] != INF and par[v] != v:
            children.setdefault(int(par[v]), []).append(v)
    reset = set()
    stack = [v for (u, v) in deleted if d0[v] != INF and par[v] == u and v != 0]
    while stack:
        v = stack.pop()
        if v in reset:
            continue
        reset.add(v)
        stack.extend(children.get(v, []))
    for v in reset:
        d[v] = INF
    # (a) the reference's re-push from every reached vertex (and inserts)
    da = relax_rounds(d, {v for v in range(nv) if d[v] != INF})
    # (b) pull over the reset vertices' in-edges, then the inserted edges
    db = d.copy()
    improved = set()
    for e in range(len(col2)):
        u, v = int(src2[e]), int(col2[e])
        if v in reset and db[u] != INF and (u not in reset) and int(db[u]) + int(w2[e]) < db[v]:
            db[v] = int(db[u]) + int(w2[e])
            improved.add(v)
    for u, v, c in zip(i_s.tolist(), i_d.tolist(), iw.tolist()):
        if db[u] != INF and int(db[u]) + c < db[v]:
            db[v] = int(db[u]) + c
            improved.add(v)
    db = relax_rounds(db, improved)
    assert np.array_equal(da.astype(np.uint32), want)
    assert np.array_equal(db.astype(np.uint32), want)


def test_sssp_dijkstra_vs_fifo_explicit_weights():
    nv, row, col = O.rmat_csr(11, 16, 9)
    w = O.weights(nv, row, col, 3, 0)
    assert w.min() >= 1 and w.max() <= 64
    for s in [0, 5, 100]:
        d, p = O.sssp(nv, row, col, w, s)
        d2, _ = O.sssp_fifo(nv, row, col, w, s)
        assert np.array_equal(d, d2)
        assert O.check_tree(nv, row, col, w, s, d, p) == 0


def test_check_tree_detects_planted_mistakes():
    """Mistakes planted in oracle outputs (on the CPU) are caught."""
    nv, row, col = O.rmat_csr(10, 16, 4)
    w = O.weights(nv, row, col, 1, 0)
    d, p = O.sssp(nv, row, col, w, 0)
    assert O.check_tree(nv, row, col, w, 0, d, p) == 0
    reached = np.nonzero((d != O.INF) & (np.arange(nv) != 0))[0]
    v = int(reached[len(reached) // 2])
    d2 = d.copy()
    d2[v] += 1
    assert O.check_tree(nv, row, col, w, 0, d2, p) > 0
    p2 = p.copy()
    p2[v] = (p[v] + 1) % nv
    assert O.check_tree(nv, row, col, w, 0, d, p2) > 0
    lab = O.cc(nv, row, col)
    par = np.full(nv, O.INF, np.uint32)  # no parents at all: invalid
    assert O.check_cc_parent(nv, row, col, lab, par) > 0


def test_update_generator_properties():
    nv, row, col = O.rmat_csr(10, 16, 1)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 77, 500, 500)
    keys = set(zip(_src_ids(row).tolist(), col.tolist()))
    ins = list(zip(i_s.tolist(), i_d.tolist()))
    dels = list(zip(d_s.tolist(), d_d.tolist()))
    assert len(set(ins)) == 500 and len(set(dels)) == 500
    assert all(u != v and (u, v) not in keys for u, v in ins)
    assert all((u, v) in keys for u, v in dels)
    # deterministic
    again = O.gen_updates(nv, row, col, 77, 500, 500)
    assert all(np.array_equal(a, b) for a, b in zip(again, (i_s, i_d, d_s, d_d)))


def test_rmat_generator_shape():
    nv, row, col = O.rmat_csr(12, 16, 1)
    assert nv == 4096 and row[-1] == len(col)
    src = _src_ids(row)
    assert np.all(src != col)  # no self loops
    k = (src.astype(np.uint64) << np.uint64(32)) | col
    assert np.all(np.diff(k.astype(np.int64)) > 0)  # sorted, unique
    # skew: vertex 0 is the heaviest source for a > d
    deg = np.diff(row)
    assert deg[0] == deg.max()


def test_widest_path_oracle_brute_force():
    """The widest-path oracle (user functor parity) equals a brute-force
    fixed point of width[v] = max over in-edges of min(width[u], w)."""
    for scale, seed in ((7, 1), (9, 4)):
        nv, row, col = O.rmat_csr(scale, 8, seed)
        w = O.weights(nv, row, col, seed, 0)
        for src in (0, 3):
            got = O.widest(nv, row, col, w, src)
            b = np.zeros(nv, np.int64)
            b[src] = 2**32 - 1
            changed = True
            while changed:
                changed = False
                for u in range(nv):
                    if b[u] == 0:
                        continue
                    for e in range(row[u], row[u + 1]):
                        nb = min(b[u], int(w[e]))
                        if nb > b[col[e]]:
                            b[col[e]] = nb
                            changed = True
            assert np.array_equal(got, b.astype(np.uint32))
