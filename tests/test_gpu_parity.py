"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Integer algorithms (BFS depth, SSSP distance, CC label) must match bit for
bit.  Parents are not unique (any tight predecessor is a correct parent, and
the engine keeps the one whose strict improvement landed last), so they are
checked for validity: BFS/SSSP parents form a tree of tight existing edges
rooted at the source; CC parents have the same label, an existing edge and no
cycle.  PageRank must be within L-infinity 1e-6 of
the FP64 power iteration of the same fixed point.
"""
import numpy as np
import pytest

import oracle as O
import sgs

pytestmark = pytest.mark.gpu

PR_TOL = 1e-6  # L-infinity vs FP64 power iteration


def _src_ids(row):
    return np.repeat(np.arange(len(row) - 1, dtype=np.uint32), np.diff(row).astype(np.int64))


class Mirror:
    """Oracle-side copy of the graph, updated with the same batches."""

    def __init__(self, nv, row, col, w):
        self.nv, self.row, self.col, self.w = nv, row, col, w

    def apply(self, i_s, i_d, i_w, d_s, d_d):
        self.row, self.col, self.w = O.apply(self.nv, self.row, self.col, self.w,
                                             i_s, i_d, i_w, d_s, d_d)


def check_graph(eng, m):
    row, col, w = eng.export(weights=m.w is not None)
    assert np.array_equal(row, m.row)
    for v in range(m.nv):
        a = sorted(zip(col[row[v]:row[v + 1]].tolist(),
                       (w[row[v]:row[v + 1]] if w is not None else col[row[v]:row[v + 1]]).tolist()))
        b = sorted(zip(m.col[m.row[v]:m.row[v + 1]].tolist(),
                       (m.w[m.row[v]:m.row[v + 1]] if m.w is not None
                        else m.col[m.row[v]:m.row[v + 1]]).tolist()))
        assert a == b, v


def check_query(q, m, wmode):
    nv, row, col = m.nv, m.row, m.col
    if q.algo == sgs.PR:
        x = O.pagerank(nv, row, col)
        got = q.value()
        assert np.max(np.abs(got - x)) <= PR_TOL
        st = q.stats()
        assert st["converged"] == 1
        return
    val, par = q.value(), q.parent()
    if q.algo == sgs.CC:
        lab = O.cc(nv, row, col)
        assert np.array_equal(val, lab)
        assert O.check_cc_parent(nv, row, col, val, par) == 0
        return
    src = min(q.source, nv - 1)
    if q.algo == sgs.BFS:
        w = None
        d, _ = O.bfs(nv, row, col, src)
    else:
        w = m.w if wmode == sgs.W_EXPLICIT else O.weights(nv, row, col, 0, 1 if wmode == sgs.W_SYNTH else 2)
        d, _ = O.sssp(nv, row, col, w, src)
    assert np.array_equal(val, d)
    assert O.check_tree(nv, row, col, w, src, val, par) == 0


def test_device_generator_matches_oracle():
    nv, row, col = O.rmat_csr(12, 16, 5)
    w = O.weights(nv, row, col, 9, 0)
    with sgs.Engine() as e:
        e.load_rmat(12, 16, 5, wseed=9)
        r2, c2, w2 = e.export(weights=True)
    m = Mirror(nv, row, col, w)
    assert np.array_equal(r2, row)
    for v in range(0, nv, 7):
        a = sorted(zip(c2[r2[v]:r2[v + 1]].tolist(), w2[r2[v]:r2[v + 1]].tolist()))
        b = list(zip(col[row[v]:row[v + 1]].tolist(), w[row[v]:row[v + 1]].tolist()))
        assert a == b
    del m


@pytest.mark.parametrize("wmode", [sgs.W_EXPLICIT, sgs.W_SYNTH])
def test_static_queries(wmode):
    nv, row, col = O.rmat_csr(14, 16, 2)
    w = O.weights(nv, row, col, 4, 0 if wmode == sgs.W_EXPLICIT else 1)
    with sgs.Engine(weight_mode=wmode) as e:
        e.load_csr(nv, row, col, w if wmode == sgs.W_EXPLICIT else None)
        m = Mirror(nv, row, col, w if wmode == sgs.W_EXPLICIT else None)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.SSSP, 1234), e.add_query(sgs.BFS, 0),
              e.add_query(sgs.BFS, 77), e.add_query(sgs.CC), e.add_query(sgs.PR)]
        for q in qs:
            check_query(q, m, wmode)
            assert q.stats()["converged"] == 1


def test_readme_example_snapshots():
    """README.md:68-96 through the reference-style driver sequence."""
    src = np.array([0, 0, 1, 1, 2, 3], np.uint32)
    dst = np.array([1, 2, 2, 3, 4, 4], np.uint32)
    adds = [([0, 0], [3, 4]), ([1, 2], [4, 3])]
    dels = [([0, 0, 1], [1, 2, 2]), ([1, 2, 3], [3, 4, 4])]
    expect = {
        "sssp": [[0, 2, 3, 7, 10], [0, O.INF, O.INF, 4, 5], [0, O.INF, O.INF, 4, 5]],
        "bfs": [[0, 1, 1, 2, 2], [0, O.INF, O.INF, 1, 1], [0, O.INF, O.INF, 1, 1]],
        "cc": [[0, 0, 0, 0, 0], [0, 1, 2, 0, 0], [0, 1, 2, 0, 0]],
    }
    for algo, exp in expect.items():
        he = sgs.HybridEngine(algo, weight_mode=sgs.W_SYNTH)
        he.LoadGraph(src, dst)
        he.InitGraph(0)
        he.Start()
        assert he.GatherValue().tolist() == exp[0]
        for k in range(2):
            he.del_edge(*dels[k])
            he.add_edge(*adds[k])
            assert he.GatherValue().tolist() == exp[k + 1], (algo, k)
            assert he.GatherBuffer().tolist() == exp[k + 1]
        he.engine.close()
    he = sgs.HybridEngine("pr", weight_mode=sgs.W_SYNTH)
    he.LoadGraph(src, dst)
    he.InitGraph(1e-6)
    he.Start()
    assert np.allclose(he.GatherValue(), [0.15, 0.21375, 0.30459375, 0.24084375, 0.613621875],
                       atol=1e-6)
    row, col, _ = O.csr_file_order(5, src, dst)
    for k in range(2):
        he.Cancelation(*dels[k])
        he.Compensate(*adds[k])
        row, col, _ = O.apply(5, row, col, None, adds[k][0], adds[k][1], None, dels[k][0], dels[k][1])
        assert np.max(np.abs(he.GatherValue() - O.pagerank(5, row, col))) <= PR_TOL
    he.engine.close()


@pytest.mark.parametrize("scale,nsnap,nupd", [(11, 4, 300), (14, 4, 3000)])
def test_incremental_snapshots(scale, nsnap, nupd):
    nv, row, col = O.rmat_csr(scale, 16, 3)
    w = O.weights(nv, row, col, 2, 0)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 0), e.add_query(sgs.CC),
              e.add_query(sgs.PR), e.add_query(sgs.SSSP, 5)]
        i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 11, nsnap * nupd, nsnap * nupd)
        for k in range(nsnap):
            sl = slice(k * nupd, (k + 1) * nupd)
            iw = np.array([O.weight_of(2, u, v) for u, v in zip(i_s[sl], i_d[sl])], np.uint32)
            e.apply_batch(i_s[sl], i_d[sl], iw, d_s[sl], d_d[sl])
            m.apply(i_s[sl], i_d[sl], iw, d_s[sl], d_d[sl])
            check_graph(e, m)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        st = e.engine_stats()
        assert st["ne"] == len(m.col)


def test_messy_batches():
    """Duplicate inserts, insert+delete of one edge in a batch (delete wins),
    deletes of non-edges, self loops, repeated deletes, empty batches."""
    nv, row, col = O.rmat_csr(10, 8, 6)
    w = O.weights(nv, row, col, 1, 0)
    rng = np.random.default_rng(3)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 3), e.add_query(sgs.CC),
              e.add_query(sgs.PR)]
        srcs = _src_ids(row)
        for k in range(5):
            i_s = rng.integers(0, nv, 200).astype(np.uint32)
            i_d = rng.integers(0, nv, 200).astype(np.uint32)
            i_s = np.concatenate([i_s, i_s[:30], [7, 7]]).astype(np.uint32)
            i_d = np.concatenate([i_d, i_d[:30], [7, 9]]).astype(np.uint32)
            iw = rng.integers(1, 65, len(i_s)).astype(np.uint32)
            pick = rng.integers(0, len(m.col), 150)
            ms = _src_ids(m.row)
            d_s = np.concatenate([ms[pick], i_s[40:50], rng.integers(0, nv, 20), ms[pick[:10]]])
            d_d = np.concatenate([m.col[pick], i_d[40:50], rng.integers(0, nv, 20), m.col[pick[:10]]])
            d_s, d_d = d_s.astype(np.uint32), d_d.astype(np.uint32)
            e.apply_batch(i_s, i_d, iw, d_s, d_d)
            m.apply(i_s, i_d, iw, d_s, d_d)
            check_graph(e, m)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        e.apply_batch([], [], None, [], [])
        for q in qs:
            check_query(q, m, sgs.W_EXPLICIT)
        del srcs


@pytest.mark.parametrize("pull", [0, 1])
def test_hub_deletes(pull):
    """Sources losing hundreds of edges in one batch (the shared-memory hash
    path of the tombstoning), with parallel copies of deleted edges, repeated
    deletes and deletes of non-edges, next to sources losing one or two; the
    in-edge store (pull) gets the same deletes transposed."""
    rng = np.random.default_rng(11)
    nv = 3000
    hubs = [0, 1, 2]
    src = [np.full(1500, h) for h in hubs] + [rng.integers(0, nv, 20000)]
    dst = [rng.integers(0, nv, 1500) for _ in hubs] + [rng.integers(0, nv, 20000)]
    src = np.concatenate(src).astype(np.uint32)
    dst = np.concatenate(dst).astype(np.uint32)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]  # parallel copies kept
    row = np.zeros(nv + 1, np.uint64)
    np.add.at(row, src.astype(np.int64) + 1, 1)
    row = np.cumsum(row).astype(np.uint64)
    col = dst
    w = O.weights(nv, row, col, 4, 0)
    with sgs.Engine(pull=pull) as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 1), e.add_query(sgs.CC), e.add_query(sgs.PR)]
        for k in range(3):
            ms = _src_ids(m.row)
            hub_rows = np.nonzero(np.isin(ms, hubs))[0]
            pick = rng.choice(hub_rows, 900, replace=False)
            other = rng.integers(0, len(m.col), 300)
            d_s = np.concatenate([ms[pick], ms[pick[:50]], ms[other], [0] * 20]).astype(np.uint32)
            d_d = np.concatenate([m.col[pick], m.col[pick[:50]], m.col[other],
                                  rng.integers(0, nv, 20)]).astype(np.uint32)
            i_s = rng.integers(0, nv, 500).astype(np.uint32)
            i_d = rng.integers(0, nv, 500).astype(np.uint32)
            iw = rng.integers(1, 65, 500).astype(np.uint32)
            e.apply_batch(i_s, i_d, iw, d_s, d_d)
            m.apply(i_s, i_d, iw, d_s, d_d)
            check_graph(e, m)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)


def test_relocation_and_repack():
    """No slack and no headroom: every insert relocates a block and the arena
    is repacked; results stay identical."""
    nv, row, col = O.rmat_csr(11, 8, 8)
    w = O.weights(nv, row, col, 5, 0)
    with sgs.Engine(slack_div=0, arena_headroom=0.0) as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.PR)]
        i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 5, 3 * 4000, 3 * 100)
        for k in range(3):
            a, b = slice(k * 4000, (k + 1) * 4000), slice(k * 100, (k + 1) * 100)
            iw = np.array([O.weight_of(5, u, v) for u, v in zip(i_s[a], i_d[a])], np.uint32)
            e.apply_batch(i_s[a], i_d[a], iw, d_s[b], d_d[b])
            m.apply(i_s[a], i_d[a], iw, d_s[b], d_d[b])
            check_graph(e, m)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        st = e.engine_stats()
        assert st["repacks"] >= 1


def test_out_of_hbm_tier():
    """An HBM budget far below the graph: most blocks live in pinned host
    memory and are read over the host link; results are identical."""
    nv, row, col = O.rmat_csr(13, 16, 4)
    w = O.weights(nv, row, col, 6, 0)
    budget_gb = len(col) * 8 * 0.2 / 1e9
    with sgs.Engine(hbm_budget_gb=budget_gb, segments=64) as e:
        e.load_csr(nv, row, col, w)
        st = e.engine_stats()
        assert st["arena_bytes_host"] > 0
        assert st["hbm_resident_vertices"] < nv
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.CC), e.add_query(sgs.PR)]
        for q in qs:
            check_query(q, m, sgs.W_EXPLICIT)
        i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 9, 2000, 2000)
        iw = np.array([O.weight_of(6, u, v) for u, v in zip(i_s, i_d)], np.uint32)
        e.apply_batch(i_s, i_d, iw, d_s, d_d)
        m.apply(i_s, i_d, iw, d_s, d_d)
        check_graph(e, m)
        for q in qs:
            check_query(q, m, sgs.W_EXPLICIT)


def test_edge_cases():
    # single vertex, no edges
    with sgs.Engine() as e:
        e.load_csr(1, np.array([0, 0], np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
        q = e.add_query(sgs.SSSP, 0)
        assert q.value().tolist() == [0]
        c = e.add_query(sgs.CC)
        assert c.value().tolist() == [0]
        p = e.add_query(sgs.PR)
        assert np.allclose(p.value(), [0.15])
    # source out of range is clamped (hybrid_sssp.cu:213)
    nv, row, col = O.rmat_csr(8, 8, 1)
    w = O.weights(nv, row, col, 1, 0)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        q = e.add_query(sgs.BFS, 10 ** 6)
        assert q.source == 10 ** 6
        d, _ = O.bfs(nv, row, col, nv - 1)
        assert np.array_equal(q.value(), d)
        # isolated / sink source
        sink = int(np.nonzero(np.diff(row) == 0)[0][0])
        q2 = e.add_query(sgs.SSSP, sink)
        v = q2.value()
        assert v[sink] == 0 and np.all(np.delete(v, sink) == O.INF)


def test_errors_are_status_codes():
    nv, row, col = O.rmat_csr(8, 8, 1)
    w = O.weights(nv, row, col, 1, 0)
    with sgs.Engine() as e:
        with pytest.raises(sgs.SgsError) as ei:
            e.add_query(sgs.SSSP, 0)
        assert ei.value.code == -4  # no graph yet
        e.load_csr(nv, row, col, w)
        q = e.add_query(sgs.SSSP, 0)
        with pytest.raises(sgs.SgsError) as ei:
            e.apply_batch([nv + 5], [1], [3], [], [])
        assert ei.value.code == -1
        with pytest.raises(sgs.SgsError) as ei:
            e.apply_batch([1], [2], [0], [], [])
        assert ei.value.code == -1
        with pytest.raises(sgs.SgsError):
            e.gather(999, 0)
        # the engine is still usable after rejected batches
        d, p = O.sssp(nv, row, col, w, 0)
        assert np.array_equal(q.value(), d)
    with pytest.raises(sgs.SgsError):
        with sgs.Engine() as e:
            e.load_csr(4, np.array([0, 1, 1, 1, 1], np.uint64), np.array([9], np.uint32),
                       np.array([1], np.uint32))


def test_groups_match_single_lane_engine():
    """Queries relaxed together in a group give exactly what one-query-per-
    pass (group_size=1) gives, through static start and snapshots; lanes
    that join a running group and removed lanes do not disturb the others."""
    nv, row, col = O.rmat_csr(13, 16, 12)
    w = O.weights(nv, row, col, 3, 0)
    specs = [(sgs.SSSP, 0), (sgs.BFS, 0), (sgs.CC, 0), (sgs.SSSP, 77), (sgs.BFS, 901), (sgs.CC, 0)]
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 21, 3 * 1500, 3 * 1500)
    iw = np.array([O.weight_of(3, u, v) for u, v in zip(i_s, i_d)], np.uint32)
    res = {}
    for gs in (1, 4):
        with sgs.Engine(group_size=gs) as e:
            e.load_csr(nv, row, col, w)
            qs = [e.add_query(a, s) for a, s in specs[:4]]
            m = Mirror(nv, row, col, w)
            out = []
            for k in range(3):
                sl = slice(k * 1500, (k + 1) * 1500)
                if k == 1:  # a lane joins mid-stream, another leaves
                    qs.append(e.add_query(*specs[4]))
                    e.remove_query(qs[1])
                    qs[1] = e.add_query(*specs[5])
                e.apply_batch(i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
                m.apply(i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
                for q in qs:
                    check_query(q, m, sgs.W_EXPLICIT)
                out.append([q.value() for q in qs])
            res[gs] = out
    for k in range(3):
        for a, b in zip(res[1][k], res[4][k]):
            assert np.array_equal(a, b)


def test_staged_batches_pipeline():
    """sgs_stage_batch + sgs_apply_staged (batch k+1 copied while batch k is
    applied) give the same graph and results as sgs_apply_batch; misuse is a
    status code."""
    import ctypes as C

    nv, row, col = O.rmat_csr(12, 16, 21)
    w = O.weights(nv, row, col, 7, 0)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 3, 4 * 1500, 4 * 1500)
    iw = np.array([O.weight_of(7, u, v) for u, v in zip(i_s, i_d)], np.uint32)
    parts = [[np.ascontiguousarray(x[k * 1500:(k + 1) * 1500]) for x in (i_s, i_d, iw, d_s, d_d)]
             for k in range(4)]

    def ptrs(p):
        return [x.ctypes.data_as(C.c_void_p).value for x in p]

    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 2), e.add_query(sgs.CC), e.add_query(sgs.PR)]
        with pytest.raises(sgs.SgsError):
            e.apply_staged()  # nothing staged
        a = ptrs(parts[0])
        e.stage_batch_ptr(a[0], a[1], a[2], 1500, a[3], a[4], 1500, sgs.MEM_HOST)
        for k in range(4):
            if k + 1 < 4:
                b = ptrs(parts[k + 1])
                e.stage_batch_ptr(b[0], b[1], b[2], 1500, b[3], b[4], 1500, sgs.MEM_HOST)
                if k == 0:
                    with pytest.raises(sgs.SgsError):  # a third staged batch
                        e.stage_batch_ptr(b[0], b[1], b[2], 1500, b[3], b[4], 1500, sgs.MEM_HOST)
            e.apply_staged()
            m.apply(*parts[k])
            check_graph(e, m)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)


@pytest.mark.parametrize("gs", [4, 64])
def test_batched_summaries_equal_single(gs):
    """sgs_query_summaries (one read-back; a narrow group's lanes in one
    pass) equals sgs_query_summary query by query, PageRank and a repeated
    id included."""
    nv, row, col = O.rmat_csr(11, 16, 4)
    w = O.weights(nv, row, col, 2, 0)
    with sgs.Engine(group_size=gs) as e:
        e.load_csr(nv, row, col, w)
        qs = e.add_queries([(sgs.SSSP, 0), (sgs.BFS, 5), (sgs.CC, 0), (sgs.BFS, 9), (sgs.SSSP, 3)])
        qs.append(e.add_query(sgs.PR))
        order = qs + [qs[1]]
        got = e.summaries(order)
        want = np.stack([q.summary() for q in order])
        pr = [i for i, q in enumerate(order) if q.algo == sgs.PR]
        ints = [i for i in range(len(order)) if i not in pr]
        assert np.array_equal(got[ints], want[ints])
        # PageRank: out[1] is the FP64 sum of ranks (its bits), summed with
        # atomics in no fixed order, so equal to rounding
        for i in pr:
            assert got[i, 0] == want[i, 0]
            a, b = got[i, 1:2].view(np.float64)[0], want[i, 1:2].view(np.float64)[0]
            assert abs(a - b) <= 1e-12 * abs(b)
