"""Parity at the sizes of the benchmark configurations, through the C ABI.

* Incremental PageRank exactly as the first configuration states it: R-MAT
  scale 16 (edge factor 16, seed 1, a/b/c/d = 0.57/0.19/0.19/0.05, duplicates
  and self-loops removed), damping 0.85, two snapshots of 10,000 new-edge
  inserts and 10,000 deletes of existing edges, 512 segments, no edge cache
  (samples/hybrid_pr/hybrid_pr.cu:154-200 drives the same sequence).  Ranks
  within L-infinity 1e-6 of the FP64 power iteration after every snapshot,
  with pull and push sweeps.
* The headline snapshot stream at R-MAT scale 20: three snapshots of 1M
  updates (500k inserts, 500k deletes), explicit weights uniform in [1,64],
  SSSP and BFS from vertex 0 and CC (samples/hybrid_sssp/hybrid_sssp.cu:
  204-296 drives the same sequence), bit-exact against the oracle after
  every snapshot -- with the reference's re-push repair, with the pull
  repair, and with most blocks in the pinned-host tier behind the edge cache.
* Batched lanes at scale 20: a 64-lane group of BFS and SSSP sources drawn
  from the largest weakly connected component, two snapshots of 100k
  updates, a sample of lanes bit-exact against the oracle.
* A served trace at scale 16: Poisson arrivals of update batches (sizes
  log-uniform in [100, 10k], half inserts, half deletes) and BFS / SSSP / CC /
  PageRank queries; every query equals the oracle on the snapshot of its
  version.
"""
import numpy as np
import pytest

import oracle as O
import sgs
from test_gpu_parity import Mirror, check_query

pytestmark = pytest.mark.gpu

PR_TOL = 1e-6


def _rmat(scale, seed=1):
    return O.rmat_csr(scale, 16, seed)


@pytest.mark.parametrize("pull", [1, 0])
def test_config1_pagerank_scale16_two_snapshots(pull):
    nv, row, col = _rmat(16, 1)
    assert nv == 65536 and 900_000 < len(col) < 1_100_000  # ~1.05M draws, fewer after dedupe
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 1000003, 20000, 20000)
    with sgs.Engine(segments=512, cache_gb=0.0, weight_mode=sgs.W_UNIT, pull=pull) as e:
        e.load_rmat(16, 16, 1)
        r0, c0, _ = e.export()
        assert np.array_equal(r0, row)
        q = e.add_query(sgs.PR)
        assert np.max(np.abs(q.value() - O.pagerank(nv, row, col))) <= PR_TOL
        m = Mirror(nv, row, col, None)
        for k in range(2):
            sl = slice(k * 10000, (k + 1) * 10000)
            e.apply_batch(i_s[sl], i_d[sl], None, d_s[sl], d_d[sl])
            m.apply(i_s[sl], i_d[sl], None, d_s[sl], d_d[sl])
            st = e.engine_stats()
            assert st["last_inserted"] == 10000 and st["last_deleted"] == 10000
            err = float(np.max(np.abs(q.value() - O.pagerank(nv, m.row, m.col))))
            assert err <= PR_TOL, (k, err)
            assert q.stats()["converged"] == 1


@pytest.mark.parametrize("repair,budget_gb,cache_gb", [(0, 4.0, 0.0), (1, 4.0, 0.0), (0, 0.04, 0.016)])
def test_headline_stream_scale20(repair, budget_gb, cache_gb):
    nv, row, col = _rmat(20, 1)
    w = O.weights(nv, row, col, 1, 0)
    half = 500_000
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 1000003, 3 * half, 3 * half)
    iw = O.weights_pairs(1, i_s, i_d)
    with sgs.Engine(hbm_budget_gb=budget_gb, cache_gb=cache_gb, repair=repair) as e:
        e.load_rmat(20, 16, 1, wseed=1)
        st = e.engine_stats()
        if budget_gb < 1:
            assert st["arena_bytes_host"] > st["arena_bytes_hbm"]  # most blocks host-resident
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 0), e.add_query(sgs.CC, 0)]
        m = Mirror(nv, row, col, w)
        for k in range(3):
            sl = slice(k * half, (k + 1) * half)
            e.apply_batch(i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
            m.apply(i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
                assert q.stats()["converged"] == 1
        assert e.engine_stats()["ne"] == len(m.col)


def _wcc_sources(nv, row, col, n, seed):
    import scipy.sparse as sp
    import scipy.sparse.csgraph as cg

    A = sp.csr_matrix((np.ones(len(col), np.int8), col.astype(np.int64), row.astype(np.int64)),
                      shape=(nv, nv))
    _, lab = cg.connected_components(A, directed=True, connection="weak")
    big = int(np.argmax(np.bincount(lab)))
    cand = np.nonzero(lab == big)[0]
    return np.random.default_rng(seed).choice(cand, n, replace=False).astype(np.uint32)


def test_batched_lanes_scale20():
    nv, row, col = _rmat(20, 1)
    w = O.weights(nv, row, col, 1, 0)
    src = _wcc_sources(nv, row, col, 64, 5)
    specs = [(sgs.BFS if k % 2 == 0 else sgs.SSSP, int(s)) for k, s in enumerate(src)]
    half = 50_000
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 77, 2 * half, 2 * half)
    iw = O.weights_pairs(1, i_s, i_d)
    sample = [0, 1, 2, 3, 30, 31, 62, 63]
    with sgs.Engine(group_size=64) as e:
        e.load_rmat(20, 16, 1, wseed=1)
        qs = e.add_queries(specs)
        m = Mirror(nv, row, col, w)
        for k in sample:
            check_query(qs[k], m, sgs.W_EXPLICIT)
        for k in range(2):
            sl = slice(k * half, (k + 1) * half)
            e.apply_batch(i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
            m.apply(i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
            for j in sample:
                check_query(qs[j], m, sgs.W_EXPLICIT)
                assert qs[j].stats()["converged"] == 1


class _Res:
    def __init__(self, algo, source, value, parent):
        self.algo, self.source, self._v, self._p = algo, source, value, parent

    def value(self):
        return self._v

    def parent(self):
        return self._p

    def stats(self):
        return {"converged": 1}


def test_served_trace_scale16():
    nv, row, col = _rmat(16, 1)
    w = O.weights(nv, row, col, 1, 0)
    rng = np.random.default_rng(11)
    n_upd, n_q = 8, 24
    sizes = np.exp(rng.uniform(np.log(100), np.log(10_000), n_upd)).astype(int)
    tot = int(sizes.sum())
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, 12345, tot, tot)
    iw = O.weights_pairs(1, i_s, i_d)
    kinds = ["update"] * n_upd + ["query"] * n_q
    rng.shuffle(kinds)
    t = np.cumsum(rng.exponential(0.003, len(kinds)))
    reqs, batches, off, u = [], [], 0, 0
    algos = [sgs.BFS, sgs.SSSP, sgs.CC, sgs.PR]
    for k, kind in enumerate(kinds):
        if kind == "update":
            sl = slice(off, off + int(sizes[u]))
            off += int(sizes[u])
            u += 1
            b = (i_s[sl], i_d[sl], iw[sl], d_s[sl], d_d[sl])
            batches.append(b)
            reqs.append({"kind": "update", "arrival_s": float(t[k]), "ins_src": b[0], "ins_dst": b[1],
                         "ins_w": b[2], "del_src": b[3], "del_dst": b[4]})
        else:
            a = algos[k % 4]
            reqs.append({"kind": "query", "algo": a, "source": int(rng.integers(0, nv)),
                         "arrival_s": float(t[k]),
                         "value_out": np.empty(nv, np.float64 if a == sgs.PR else np.uint32),
                         "parent_out": np.empty(nv, np.uint32)})
    with sgs.Engine(group_size=64) as e:
        e.load_rmat(16, 16, 1, wseed=1)
        res = e.serve(reqs, slots=16, realtime=True)
    m = Mirror(nv, row, col, w)
    snaps = [(m.row, m.col, m.w)]
    for b in batches:
        m.apply(*b)
        snaps.append((m.row, m.col, m.w))
    n_upd_seen = 0
    for i in np.argsort([r["arrival_s"] for r in reqs], kind="stable"):
        r, c = reqs[i], res[i]
        assert c["status"] == 0
        if r["kind"] == "update":
            n_upd_seen += 1
            continue
        # at least the updates that arrived before it; a BFS/SSSP/CC query
        # moves to a later snapshot only when an update restarted it
        assert n_upd_seen <= c["version"] <= len(batches)
        if r["algo"] != sgs.PR:
            assert (c["version"] > n_upd_seen) == (c["restarts"] > 0)
        rr, cc, ww = snaps[c["version"]]
        check_query(_Res(r["algo"], r["source"], r["value_out"], r["parent_out"]),
                    Mirror(nv, rr, cc, ww), sgs.W_EXPLICIT)
