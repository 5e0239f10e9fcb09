"""Pull kernels over the in-edge (CSC) store: PageRank sweeps as pulls and
direction-optimizing (bottom-up) BFS starts.

The in-edge store is built by transposing the graph when a pull first needs
it and is then updated by every snapshot with the batch's keys transposed
(tombstones, appends, relocations, rebuilds when relocations do not fit).
Results must be exactly those of the push path and the CPU oracle: BFS
depths bit-exact with valid parent trees, PageRank within 1e-6 of the FP64
power iteration."""
import numpy as np
import pytest

import oracle as O
import sgs
from test_gpu_parity import PR_TOL, Mirror, check_graph, check_query

pytestmark = pytest.mark.gpu


def _batch(m, seed, ni, nd, wseed):
    i_s, i_d, d_s, d_d = O.gen_updates(m.nv, m.row, m.col, seed, ni, nd)
    iw = np.array([O.weight_of(wseed, u, v) for u, v in zip(i_s, i_d)], np.uint32)
    return i_s, i_d, iw, d_s, d_d


@pytest.mark.parametrize("pull", [0, 1])
def test_pagerank_pull_and_push_agree(pull):
    nv, row, col = O.rmat_csr(13, 16, 3)
    w = O.weights(nv, row, col, 2, 0)
    with sgs.Engine(pull=pull) as e:
        e.load_csr(nv, row, col, w)
        e.kernel_timing(True)
        m = Mirror(nv, row, col, w)
        q = e.add_query(sgs.PR)
        check_query(q, m, sgs.W_EXPLICIT)
        st = e.engine_stats()
        assert (st["in_store_bytes"] > 0) == bool(pull)
        for k in range(3):
            b = _batch(m, 30 + k, 2000, 2000, 2)
            e.apply_batch(*b)
            m.apply(*b)
            check_query(q, m, sgs.W_EXPLICIT)
        ks = e.kernel_stats()
        assert (ks["pr_pull"]["launches"] > 0) == bool(pull)
        assert (ks["pr_push"]["launches"] > 0) == (not pull)


def test_pagerank_round_kernel_matches_launches():
    """PageRank's pull rounds as one cooperative launch (persistent bit 3,
    the default) or as a kernel pair per round: both within 1e-6 of the FP64
    power iteration after every snapshot, and they stop after the same
    rounds (up to one round: the residual sum's order differs)."""
    nv, row, col = O.rmat_csr(14, 16, 6)
    w = O.weights(nv, row, col, 2, 0)
    rounds = {}
    for pers in (6, 14):
        with sgs.Engine(persistent=pers) as e:
            e.load_csr(nv, row, col, w)
            e.kernel_timing(True)
            m = Mirror(nv, row, col, w)
            q = e.add_query(sgs.PR)
            check_query(q, m, sgs.W_EXPLICIT)
            rs = [q.stats()["rounds"]]
            for k in range(2):
                b = _batch(m, 70 + k, 3000, 3000, 2)
                e.apply_batch(*b)
                m.apply(*b)
                check_query(q, m, sgs.W_EXPLICIT)
                assert q.stats()["converged"] == 1
                rs.append(q.stats()["rounds"])
            # one launch per convergence with the round kernel, two per round without
            launches = e.kernel_stats()["pr_pull"]["launches"]
            assert (launches == 3) if pers == 14 else (launches >= sum(rs))
            rounds[pers] = rs
    assert all(abs(a - b) <= 1 for a, b in zip(rounds[6], rounds[14]))


def test_in_store_rebuild_and_host_tier():
    """No slack, no headroom: the in-store's relocations overflow and it is
    rebuilt from the updated graph; the out-store keeps most blocks in host
    memory.  PageRank stays exact through it."""
    nv, row, col = O.rmat_csr(11, 8, 8)
    w = O.weights(nv, row, col, 5, 0)
    gb = len(col) * 8 / 1e9
    with sgs.Engine(slack_div=0, arena_headroom=0.0, hbm_budget_gb=0.3 * gb, segments=16) as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.PR), e.add_query(sgs.SSSP, 0)]
        for k in range(3):
            b = _batch(m, 50 + k, 3000, 300, 5)
            e.apply_batch(*b)
            m.apply(*b)
            check_graph(e, m)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        st = e.engine_stats()
        assert st["in_store_builds"] >= 2 and st["arena_bytes_host"] > 0


@pytest.mark.parametrize("gs", [1, 4])
def test_direction_optimizing_bfs(gs):
    """BFS-only starts with pull bit 1: bottom-up rounds over the in-edge
    store for the large middle frontiers; depths equal the oracle's and the
    push-only engine's, parents are valid; snapshots afterwards stay exact."""
    nv, row, col = O.rmat_csr(14, 16, 6)
    w = O.weights(nv, row, col, 3, 0)
    rng = np.random.default_rng(gs)
    srcs = [0] + [int(x) for x in rng.integers(0, nv, 3)]
    with sgs.Engine(pull=3, group_size=gs) as e, sgs.Engine(pull=0, group_size=gs) as ref:
        e.load_csr(nv, row, col, w)
        ref.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = e.add_queries([(sgs.BFS, s) for s in srcs])
        rs = ref.add_queries([(sgs.BFS, s) for s in srcs])
        assert e.engine_stats()["bfs_bottom_up_rounds"] > 0
        for q, r in zip(qs, rs):
            check_query(q, m, sgs.W_EXPLICIT)
            assert np.array_equal(q.value(), r.value())
            assert q.stats()["edges_traversed"] == r.stats()["edges_traversed"]
        for k in range(2):
            b = _batch(m, 70 + k, 2000, 2000, 3)
            e.apply_batch(*b)
            m.apply(*b)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        # a fresh BFS on the updated graph runs over the updated in-store
        q2 = e.add_query(sgs.BFS, 5)
        check_query(q2, m, sgs.W_EXPLICIT)


def test_pagerank_pull_tolerance_on_skewed_graph():
    """Hub in-blocks (split across CTAs, combined by atomics) and empty
    in-blocks; L-inf within tolerance of the FP64 power iteration."""
    nv, row, col = O.rmat_csr(15, 16, 11)
    w = O.weights(nv, row, col, 1, 0)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        q = e.add_query(sgs.PR)
        x = O.pagerank(nv, row, col)
        assert np.max(np.abs(q.value() - x)) <= PR_TOL


@pytest.mark.parametrize("pull", [0, 1])
def test_pagerank_warm_start(pull):
    """A removed PageRank query leaves its vector; the next start after a
    snapshot continues from it (residual computed on the updated graph) and
    meets the same tolerance in fewer rounds."""
    nv, row, col = O.rmat_csr(13, 16, 9)
    w = O.weights(nv, row, col, 2, 0)
    with sgs.Engine(pull=pull) as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        q0 = e.add_query(sgs.PR)
        r0 = q0.stats()["rounds"]
        check_query(q0, m, sgs.W_EXPLICIT)
        e.remove_query(q0)
        b = _batch(m, 99, 300, 300, 2)
        e.apply_batch(*b)
        m.apply(*b)
        q1 = e.add_query(sgs.PR)
        check_query(q1, m, sgs.W_EXPLICIT)
        assert e.engine_stats()["pr_warm_starts"] == 1
        assert q1.stats()["rounds"] < r0
    with sgs.Engine(pull=pull, pr_warm=0) as e:
        e.load_csr(nv, row, col, w)
        e.remove_query(e.add_query(sgs.PR))
        q = e.add_query(sgs.PR)
        assert e.engine_stats()["pr_warm_starts"] == 0
        assert q.stats()["rounds"] == r0


@pytest.mark.parametrize("gs, wmode", [(4, sgs.W_EXPLICIT), (1, sgs.W_EXPLICIT), (4, sgs.W_SYNTH)])
def test_pull_repair_equals_the_sweep(gs, wmode):
    """repair = 1: after deletions a narrow group pulls over the in-edges of
    the vertices the invalidation reset (in-edge store with weights) instead
    of re-pushing from every reached vertex.  Values equal the oracle's and
    the sweep engine's; far fewer edges are read."""
    nv, row, col = O.rmat_csr(13, 16, 12)
    w = O.weights(nv, row, col, 6, 0) if wmode == sgs.W_EXPLICIT else None
    specs = [(sgs.SSSP, 0), (sgs.BFS, 7), (sgs.CC, 0), (sgs.SSSP, 11)]
    with sgs.Engine(repair=1, group_size=gs, weight_mode=wmode) as e, \
            sgs.Engine(repair=0, group_size=gs, weight_mode=wmode) as ref:
        e.load_csr(nv, row, col, w)
        ref.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs, rs = e.add_queries(specs), ref.add_queries(specs)
        for k in range(4):
            i_s, i_d, d_s, d_d = O.gen_updates(m.nv, m.row, m.col, 80 + k, 1500, 1500 if k != 2 else 0)
            iw = np.array([O.weight_of(6, u, v) for u, v in zip(i_s, i_d)], np.uint32) \
                if wmode == sgs.W_EXPLICIT else None
            e.apply_batch(i_s, i_d, iw, d_s, d_d)
            ref.apply_batch(i_s, i_d, iw, d_s, d_d)
            m.apply(i_s, i_d, iw, d_s, d_d)
            for q, r in zip(qs, rs):
                check_query(q, m, wmode)
                assert np.array_equal(q.value(), r.value())
            if k != 2:  # deletions: the pull reads a fraction of what the sweep reads
                assert sum(q.stats()["edges_traversed"] for q in qs) < \
                    sum(r.stats()["edges_traversed"] for r in rs)
        check_graph(e, m)
