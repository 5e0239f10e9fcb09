"""Served request loop (sgs_serve): update batches and one-shot queries with
Poisson arrivals, continuous batching of the queries.

Each query's result must be that of its graph version: values bit-exact
against the CPU oracle on that snapshot (PageRank within 1e-6), parents
valid, and identical to the same query run alone on the same snapshot.  The
version holds at least the updates that arrived before the query; exactly
those when updates may not preempt the queries in flight (serve_restarts =
0).  Preemption (an update restarting the queries in flight on the new
snapshot), slot admission, ordering and a failed update in the middle of
the trace are checked too."""
import numpy as np
import pytest

import oracle as O
import sgs
from test_gpu_parity import Mirror, check_query

pytestmark = pytest.mark.gpu


class Res:
    """A query result as check_query expects it (value/parent vectors)."""

    def __init__(self, algo, source, value, parent):
        self.algo, self.source, self._v, self._p = algo, source, value, parent

    def value(self):
        return self._v

    def parent(self):
        return self._p

    def stats(self):
        return {"converged": 1}


def _trace(nv, row, col, seed, n_upd=10, n_q=26, mean_gap=0.002, bad_update=None):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(10), np.log(1500), n_upd)).astype(int)
    tot = int(sizes.sum())
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, seed + 1, tot, tot)
    iw = np.array([O.weight_of(3, u, v) for u, v in zip(i_s, i_d)], np.uint32)
    kinds = ["update"] * n_upd + ["query"] * n_q
    rng.shuffle(kinds)
    t = np.cumsum(rng.exponential(mean_gap, len(kinds)))
    reqs, batches, off, u = [], [], 0, 0
    algos = [sgs.BFS, sgs.SSSP, sgs.CC, sgs.PR]
    for k, kind in enumerate(kinds):
        if kind == "update":
            n = sizes[u]
            sl = slice(off, off + n)
            off += n
            b = (i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
            if bad_update is not None and u == bad_update:
                b = (np.array([nv + 5], np.uint32), np.array([0], np.uint32),
                     np.array([1], np.uint32), d_s[:0], d_d[:0])
            batches.append(b)
            reqs.append({"kind": "update", "arrival_s": float(t[k]), "ins_src": b[0], "ins_dst": b[1],
                         "ins_w": b[2], "del_src": b[3], "del_dst": b[4]})
            u += 1
        else:
            a = algos[rng.integers(0, 4)]
            vo = np.empty(nv, np.float64 if a == sgs.PR else np.uint32)
            po = np.empty(nv, np.uint32)
            reqs.append({"kind": "query", "algo": a, "source": int(rng.integers(0, nv)),
                         "arrival_s": float(t[k]), "value_out": vo, "parent_out": po})
    return reqs, batches


def _snapshots(nv, row, col, w, batches, ok):
    m = Mirror(nv, row, col, w)
    snaps = [(m.row, m.col, m.w)]
    for b, good in zip(batches, ok):
        if good:  # versions count the updates that were applied
            m.apply(*b)
            snaps.append((m.row, m.col, m.w))
    return snaps


def _check_all(reqs, res, nv, snaps, slots, restarts=2):  # 2: the engine default
    upd_before = 0
    order = np.argsort([r["arrival_s"] for r in reqs], kind="stable")
    n_ok_upd = 0
    for i in order:
        r, c = reqs[i], res[i]
        if r["kind"] == "update":
            if c["status"] == 0:
                n_ok_upd += 1
                assert c["version"] == n_ok_upd
            continue
        assert c["status"] == 0
        if r["algo"] == sgs.PR or restarts:  # at least the updates that arrived before it
            assert n_ok_upd <= c["version"] <= len(snaps) - 1
        else:  # exactly the updates that arrived before it
            assert c["version"] == n_ok_upd
        if r["algo"] == sgs.PR:
            assert c["restarts"] == 0
        else:  # a restart moves the query to a later snapshot
            assert c["restarts"] <= restarts
            assert c["restarts"] == 0 or c["version"] > n_ok_upd
        # lanes in flight when it joined (slots bound them); PR: requests sharing its job
        assert 1 <= c["batch"] and (slots == 0 or r["algo"] == sgs.PR or c["batch"] <= slots)
        assert c["done_s"] >= c["start_s"] >= 0 and c["latency_s"] >= 0
        row, col, w = snaps[c["version"]]
        m = Mirror(nv, row, col, w)
        check_query(Res(r["algo"], r["source"], r["value_out"], r["parent_out"]), m, sgs.W_EXPLICIT)


@pytest.mark.parametrize("gs,slots,realtime,restarts",
                         [(4, 0, True, 1), (4, 3, False, 1), (64, 5, True, 1), (4, 0, True, 0),
                          (64, 0, False, 0), (64, 0, False, 3)])
def test_served_results_match_their_snapshot(gs, slots, realtime, restarts):
    nv, row, col = O.rmat_csr(12, 16, 3)
    w = O.weights(nv, row, col, 3, 0)
    reqs, batches = _trace(nv, row, col, 7 + gs + slots)
    with sgs.Engine(group_size=gs, serve_restarts=restarts) as e:
        e.load_csr(nv, row, col, w)
        res = e.serve(reqs, slots=slots, realtime=realtime)
    snaps = _snapshots(nv, row, col, w, batches, [True] * len(batches))
    _check_all(reqs, res, nv, snaps, slots, restarts)
    if slots == 0 and realtime:
        # some queries were batched together (continuous batching)
        assert max(c["batch"] for c, r in zip(res, reqs) if r["kind"] == "query") >= 1


def test_served_equals_alone():
    """A query served in the mix gives exactly what it gives alone on the
    same snapshot (integers bit-exact, PageRank within 1e-6)."""
    nv, row, col = O.rmat_csr(11, 16, 5)
    w = O.weights(nv, row, col, 3, 0)
    reqs, batches = _trace(nv, row, col, 23, n_upd=6, n_q=16, mean_gap=0.0)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        res = e.serve(reqs, slots=0, realtime=False)
    qi = [i for i, r in enumerate(reqs) if r["kind"] == "query"][:8]
    for i in qi:
        r, c = reqs[i], res[i]
        with sgs.Engine(group_size=1) as a:
            a.load_csr(nv, row, col, w)
            for b in batches[:c["version"]]:
                a.apply_batch(*b)
            q = a.add_query(r["algo"], r["source"])
            v = q.value()
        if r["algo"] == sgs.PR:
            assert np.max(np.abs(v - r["value_out"])) <= 1e-6
        else:
            assert np.array_equal(v, r["value_out"])


def test_failed_update_does_not_stop_the_loop():
    nv, row, col = O.rmat_csr(11, 16, 8)
    w = O.weights(nv, row, col, 3, 0)
    reqs, batches = _trace(nv, row, col, 31, n_upd=5, n_q=10, mean_gap=0.0, bad_update=2)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, w)
        res = e.serve(reqs, realtime=False)
    st = [c["status"] for c, r in zip(res, reqs) if r["kind"] == "update"]
    assert st[2] < 0
    assert all(s == 0 for k, s in enumerate(st) if k != 2)
    ok = [k != 2 for k in range(len(batches))]
    snaps = _snapshots(nv, row, col, w, batches, ok)
    _check_all(reqs, res, nv, snaps, 0)


def test_serve_rejects_malformed_requests():
    nv, row, col = O.rmat_csr(8, 8, 1)
    with sgs.Engine() as e:
        e.load_csr(nv, row, col, O.weights(nv, row, col, 1, 0))
        with pytest.raises(sgs.SgsError):
            e.serve([{"kind": "query", "algo": 0, "arrival_s": -1.0}])
        assert e.serve([]) == []


def test_queries_join_a_running_flight():
    """Continuous batching: queries that arrive while others are on the GPU
    start at the next round boundary and finish on their own -- some query
    starts while another is still running -- and results stay exact."""
    nv, row, col = O.rmat_csr(14, 16, 6)
    w = O.weights(nv, row, col, 3, 0)
    rng = np.random.default_rng(4)
    reqs = []
    t = 0.0
    for k in range(40):
        t += rng.exponential(0.0005)
        a = [sgs.BFS, sgs.SSSP][k % 2]
        reqs.append({"kind": "query", "algo": a, "source": int(rng.integers(0, nv)), "arrival_s": t,
                     "value_out": np.empty(nv, np.uint32), "parent_out": np.empty(nv, np.uint32)})
    with sgs.Engine(group_size=64) as e:
        e.load_csr(nv, row, col, w)
        res = e.serve(reqs, slots=16, realtime=True)
    overlap = False
    for i, a in enumerate(res):
        for b in res[i + 1:]:
            if a["start_s"] < b["start_s"] < a["done_s"] or b["start_s"] < a["start_s"] < b["done_s"]:
                overlap = True
    assert overlap
    assert max(c["batch"] for c in res) <= 16
    m = Mirror(nv, row, col, w)
    for r, c in zip(reqs, res):
        assert c["status"] == 0 and c["version"] == 0
        check_query(Res(r["algo"], r["source"], r["value_out"], r["parent_out"]), m, sgs.W_EXPLICIT)


def test_updates_do_not_wait_for_a_pagerank_job():
    """An update that arrives while a PageRank computation runs is applied at
    once: the snapshot amends the running computation, which continues on
    the new graph; its result equals the PageRank of the snapshot its
    completion reports, and the BFS behind the update sees it."""
    nv, row, col = O.rmat_csr(14, 16, 2)
    w = O.weights(nv, row, col, 3, 0)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 99, 3000, 3000)
    iw = O.weights_pairs(3, i_s, i_d)
    reqs = [{"kind": "query", "algo": sgs.PR, "source": 0, "arrival_s": 0.0,
             "value_out": np.empty(nv, np.float64)},
            {"kind": "update", "arrival_s": 0.0001, "ins_src": i_s, "ins_dst": i_d, "ins_w": iw,
             "del_src": d_s, "del_dst": d_d},
            {"kind": "query", "algo": sgs.BFS, "source": 0, "arrival_s": 0.0002,
             "value_out": np.empty(nv, np.uint32), "parent_out": np.empty(nv, np.uint32)}]
    with sgs.Engine(pr_warm=0) as e:
        e.load_csr(nv, row, col, w)
        res = e.serve(reqs, realtime=False)
    pr, upd, bfs = res
    assert all(c["status"] == 0 for c in res)
    assert upd["version"] == 1 and upd["done_s"] < pr["done_s"]  # did not wait for the PageRank
    assert pr["version"] == 1 and bfs["version"] == 1
    r2, c2, w2 = O.apply(nv, row, col, w, i_s, i_d, iw, d_s, d_d)
    assert np.max(np.abs(reqs[0]["value_out"] - O.pagerank(nv, r2, c2))) <= 1e-6
    check_query(Res(sgs.BFS, 0, reqs[2]["value_out"], reqs[2]["parent_out"]), Mirror(nv, r2, c2, w2),
                sgs.W_EXPLICIT)


@pytest.mark.parametrize("gs", [4, 64])
def test_update_preempts_the_flight(gs):
    """An update that reaches the head while BFS/SSSP/CC queries are in
    flight is applied at the next round boundary, not after them: the
    queries in flight restart from their sources on the new snapshot and
    give exactly its results (the same as alone on it).  A query restarted
    once holds the next update back until it completes (serve_restarts = 1),
    so no query starves.  Three slots: the fourth query joins when the first
    finishes, and the update behind it then stops queries that have run
    rounds already."""
    nv, row, col = O.rmat_csr(13, 16, 9)
    w = O.weights(nv, row, col, 3, 0)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 41, 4000, 4000)
    iw = O.weights_pairs(3, i_s, i_d)
    h = len(i_s) // 2
    b1 = (i_s[:h], i_d[:h], iw[:h], d_s[:h], d_d[:h])
    b2 = (i_s[h:], i_d[h:], iw[h:], d_s[h:], d_d[h:])
    rng = np.random.default_rng(5)
    reqs = []
    for a in (sgs.BFS, sgs.CC, sgs.SSSP, sgs.BFS):
        reqs.append({"kind": "query", "algo": a, "source": int(rng.integers(0, nv)), "arrival_s": 0.0,
                     "value_out": np.empty(nv, np.uint32), "parent_out": np.empty(nv, np.uint32)})
    for b in (b1, b2):
        reqs.append({"kind": "update", "arrival_s": 0.0, "ins_src": b[0], "ins_dst": b[1], "ins_w": b[2],
                     "del_src": b[3], "del_dst": b[4]})
    with sgs.Engine(group_size=gs, serve_restarts=1) as e:
        e.load_csr(nv, row, col, w)
        res = e.serve(reqs, slots=3, realtime=False)
    qs, (u1, u2) = res[:4], res[4:]
    assert all(c["status"] == 0 for c in res)
    assert u1["version"] == 1 and u2["version"] == 2
    restarted = [c for c in qs if c["restarts"]]
    assert restarted, "no query was preempted"
    # the first update did not wait for the flight to drain; the second did
    assert u1["done_s"] < max(c["done_s"] for c in restarted)
    assert u2["start_s"] >= max(c["done_s"] for c in restarted)
    snaps = _snapshots(nv, row, col, w, [b1, b2], [True, True])
    for r, c in zip(reqs[:4], qs):
        assert c["restarts"] in (0, 1) and c["version"] == c["restarts"]
        rv, cv, wv = snaps[c["version"]]
        check_query(Res(r["algo"], r["source"], r["value_out"], r["parent_out"]), Mirror(nv, rv, cv, wv),
                    sgs.W_EXPLICIT)
        with sgs.Engine(group_size=1) as a:  # the same query alone on that snapshot
            a.load_csr(nv, row, col, w)
            if c["version"]:
                a.apply_batch(*b1)
            assert np.array_equal(a.add_query(r["algo"], r["source"]).value(), r["value_out"])


def test_pagerank_query_joins_the_running_job():
    """A PageRank query that reaches the head while a PageRank job runs joins
    it instead of waiting for it (and holding back the requests behind it):
    both complete together with the PageRank of the snapshot they report,
    which holds every update that arrived before either."""
    nv, row, col = O.rmat_csr(13, 16, 4)
    w = O.weights(nv, row, col, 3, 0)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 77, 2000, 2000)
    iw = O.weights_pairs(3, i_s, i_d)
    reqs = [{"kind": "query", "algo": sgs.PR, "source": 0, "arrival_s": 0.0,
             "value_out": np.empty(nv, np.float64)},
            {"kind": "update", "arrival_s": 0.0, "ins_src": i_s, "ins_dst": i_d, "ins_w": iw,
             "del_src": d_s, "del_dst": d_d},
            {"kind": "query", "algo": sgs.PR, "source": 0, "arrival_s": 0.0,
             "value_out": np.empty(nv, np.float64)},
            {"kind": "query", "algo": sgs.BFS, "source": 3, "arrival_s": 0.0,
             "value_out": np.empty(nv, np.uint32), "parent_out": np.empty(nv, np.uint32)}]
    with sgs.Engine(pr_warm=0) as e:
        e.load_csr(nv, row, col, w)
        res = e.serve(reqs, realtime=False)
    p1, upd, p2, bfs = res
    assert all(c["status"] == 0 for c in res)
    assert p1["batch"] == 2 and p2["batch"] == 2 and p1["done_s"] == p2["done_s"]
    assert p1["version"] == 1 and p2["version"] == 1 and upd["version"] == 1
    assert bfs["done_s"] < p2["done_s"]  # the BFS behind the second PR did not wait for the job
    r2, c2, w2 = O.apply(nv, row, col, w, i_s, i_d, iw, d_s, d_d)
    x = O.pagerank(nv, r2, c2)
    for k in (0, 2):
        assert np.max(np.abs(reqs[k]["value_out"] - x)) <= 1e-6
    check_query(Res(sgs.BFS, 3, reqs[3]["value_out"], reqs[3]["parent_out"]), Mirror(nv, r2, c2, w2),
                sgs.W_EXPLICIT)
