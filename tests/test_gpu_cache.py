"""Device edge cache of the host tier (cache_gb carved out of hbm_budget_gb):
hotness-window admission per snapshot, line copies on a side stream, the
snapshot's writes made to both copies (write-through).

The cache must never change a result: every query stays bit-exact with the
CPU oracle (PageRank within 1e-6) through snapshots that delete, insert,
relocate and repack blocks while lines of them are cached.  The counters show
that the cache is used: after an admission, reads of the host tier are served
from HBM."""
import numpy as np
import pytest

import oracle as O
import sgs
from test_gpu_parity import Mirror, check_graph, check_query

pytestmark = pytest.mark.gpu


def _graph(scale, ef, seed, wseed):
    nv, row, col = O.rmat_csr(scale, ef, seed)
    w = O.weights(nv, row, col, wseed, 0)
    return nv, row, col, w


def _batch(nv, row, col, seed, ni, nd, wseed):
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, seed, ni, nd)
    iw = np.array([O.weight_of(wseed, u, v) for u, v in zip(i_s, i_d)], np.uint32)
    return i_s, i_d, iw, d_s, d_d


@pytest.mark.parametrize("gs", [4, 64])
def test_cached_snapshots_stay_exact(gs):
    nv, row, col, w = _graph(13, 16, 4, 6)
    gb = len(col) * 8 / 1e9
    # 15 % of the graph in static HBM segments, 15 % as cache lines
    with sgs.Engine(hbm_budget_gb=0.3 * gb, cache_gb=0.15 * gb, segments=64, group_size=gs) as e:
        e.load_csr(nv, row, col, w)
        st = e.engine_stats()
        assert st["cache_lines"] > 0 and st["arena_bytes_host"] > 0
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 3), e.add_query(sgs.CC),
              e.add_query(sgs.PR)]
        for q in qs:
            check_query(q, m, sgs.W_EXPLICIT)
        e.cache_refresh()
        st = e.engine_stats()
        assert st["cache_admissions"] == 1 and st["cache_resident"] > 0
        for k in range(4):
            b = _batch(m.nv, m.row, m.col, 20 + k, 1500, 1500, 6)
            e.apply_batch(*b)
            m.apply(*b)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        check_graph(e, m)
        st = e.engine_stats()
        assert st["cache_admissions"] == 5
        assert st["cache_hit_slots"] > 0
        assert st["cache_miss_slots"] > 0  # the cache holds only part of the host tier


def test_cache_larger_than_host_tier_serves_every_read():
    """With room for every line read in the window, a query run after the
    admission reads no host-tier slot over the link."""
    nv, row, col, w = _graph(12, 16, 7, 3)
    gb = len(col) * 8 / 1e9
    with sgs.Engine(hbm_budget_gb=1.6 * gb, cache_gb=1.5 * gb, segments=32) as e:
        e.load_csr(nv, row, col, w)
        st = e.engine_stats()
        assert st["arena_bytes_host"] > 0
        m = Mirror(nv, row, col, w)
        q0 = e.add_query(sgs.SSSP, 0)
        e.cache_refresh()
        a = e.engine_stats()
        q1 = e.add_query(sgs.SSSP, 0)
        b = e.engine_stats()
        assert b["cache_hit_slots"] - a["cache_hit_slots"] > 0
        assert b["cache_miss_slots"] == a["cache_miss_slots"]
        for q in (q0, q1):
            check_query(q, m, sgs.W_EXPLICIT)
        # a snapshot writes tombstones and appends into cached lines (written
        # through to both copies) and relocates blocks to new lines
        for k in range(2):
            bt = _batch(m.nv, m.row, m.col, 3 + k, 800, 800, 3)
            e.apply_batch(*bt)
            m.apply(*bt)
            for q in (q0, q1):
                check_query(q, m, sgs.W_EXPLICIT)
        check_graph(e, m)
        st = e.engine_stats()
        assert st["cache_admissions"] == 3 and st["last_relocated"] > 0


def test_cache_through_relocation_and_repack():
    """No slack and no headroom: inserts relocate blocks and the arenas are
    repacked (every cached line dropped) while the cache is on."""
    nv, row, col, w = _graph(11, 8, 8, 5)
    gb = len(col) * 8 / 1e9
    with sgs.Engine(slack_div=0, arena_headroom=0.0, hbm_budget_gb=0.5 * gb, cache_gb=0.25 * gb,
                    segments=16) as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.PR)]
        e.cache_refresh()
        for k in range(3):
            b = _batch(m.nv, m.row, m.col, 40 + k, 3000, 200, 5)
            e.apply_batch(*b)
            m.apply(*b)
            check_graph(e, m)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        st = e.engine_stats()
        assert st["repacks"] >= 1 and st["cache_admissions"] == 4


def test_cache_needs_a_budget():
    nv, row, col, w = _graph(10, 8, 1, 1)
    with sgs.Engine(cache_gb=0.01) as e:  # no HBM budget: everything in HBM, no cache
        e.load_csr(nv, row, col, w)
        q = e.add_query(sgs.BFS, 0)
        e.cache_refresh()
        st = e.engine_stats()
        assert st["cache_lines"] == 0 and st["arena_bytes_host"] == 0
        check_query(q, Mirror(nv, row, col, w), sgs.W_EXPLICIT)


@pytest.mark.parametrize("repair", [0, 1])
@pytest.mark.parametrize("policy", [1, 2])
def test_explicit_host_policy(policy, repair):
    """-hybrid 1/2: the repair reads an HBM copy of the host tier made by the
    copy engine (every snapshot, or only for dense repairs); results exact.
    With the pull repair (repair=1) the push rounds after its pull round read
    the copy too."""
    nv, row, col, w = _graph(13, 16, 4, 6)
    gb = len(col) * 8 / 1e9
    with sgs.Engine(hbm_budget_gb=0.2 * gb, segments=64, host_policy=policy, repair=repair) as e:
        e.load_csr(nv, row, col, w)
        m = Mirror(nv, row, col, w)
        qs = [e.add_query(sgs.SSSP, 0), e.add_query(sgs.BFS, 3), e.add_query(sgs.CC)]
        for k in range(3):
            b = _batch(m.nv, m.row, m.col, 90 + k, 1500, 1500 if k != 1 else 0, 6)
            e.apply_batch(*b)
            m.apply(*b)
            for q in qs:
                check_query(q, m, sgs.W_EXPLICIT)
        check_graph(e, m)
        st = e.engine_stats()
        assert st["arena_bytes_host"] > 0
        if policy == 1:
            assert st["host_stagings"] == 3 and st["last_stage_bytes"] > 0
        elif repair == 0:
            assert 1 <= st["host_stagings"] <= 3
        else:  # the pull repair's first frontier is never dense
            assert st["host_stagings"] <= 3
