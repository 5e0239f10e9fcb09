"""User algorithms written as AppBase functors (include/sgs_app.cuh), run on
the engine's snapshot path (sgs_apply_batch calls their deletion and repair
phases through sgs_app_attach's hooks).

The sample functors (c-gpustreamgraph_b200/apps/sample_apps.cu) must give:
BFS depths, SSSP distances, CC labels and widest-path widths bit-exact
against the CPU oracle, and PageRank within L-infinity 1e-6 of the FP64
power iteration, at the start and after every snapshot (deletes and
inserts, insert-only, delete-only, out-of-HBM tier); the monotone ones also
equal the engine's built-in queries on the same engine, and BFS/SSSP parents
form valid tight trees.  A functor written in the reference samples' style
(override, sepgraph::api::AppBase, utils::pair, sepgraph::engine::Engine)
runs the samples' driver sequence on the README example files.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
import sgs
from test_gpu_parity import Mirror

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIX = os.path.join(REPO, "tests", "golden", "readme")
BFS, SSSP, CC, PR, WIDEST = 0, 1, 2, 3, 4


def _lib():
    sgs.lib()  # the engine library first (the samples link it)
    L = C.CDLL(os.path.join(REPO, "c-gpustreamgraph_b200", "lib", "libsgs_apps.so"))
    L.sgs_sample_app_create.argtypes = [C.c_void_p, C.c_int, C.c_uint32, C.c_double, C.c_double,
                                        C.POINTER(C.c_void_p)]
    L.sgs_sample_app_start.argtypes = [C.c_void_p]
    L.sgs_sample_app_values.argtypes = [C.c_void_p, C.c_void_p]
    L.sgs_sample_app_parents.argtypes = [C.c_void_p, C.c_void_p]
    L.sgs_sample_app_stats.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_uint32), C.POINTER(C.c_double)]
    L.sgs_sample_app_destroy.argtypes = [C.c_void_p]
    L.sgs_sample_refstyle_sssp.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_uint32, C.c_uint32,
                                           C.c_void_p, C.c_uint32]
    return L


class App:
    def __init__(self, L, eng, kind, source=0, err=1e-12, alpha=0.85):
        self.L, self.kind, self.source, self.nv = L, kind, source, eng.nv
        h = C.c_void_p()
        rc = L.sgs_sample_app_create(eng.h, kind, source, err, alpha, C.byref(h))
        assert rc == 0, sgs.lib().sgs_last_error()
        self.h = h

    def start(self):
        assert self.L.sgs_sample_app_start(self.h) == 0, sgs.lib().sgs_last_error()

    def value(self):
        out = np.empty(self.nv, np.float64 if self.kind == PR else np.uint32)
        assert self.L.sgs_sample_app_values(self.h, out.ctypes.data) == 0
        return out

    def parent(self):
        out = np.empty(self.nv, np.uint32)
        assert self.L.sgs_sample_app_parents(self.h, out.ctypes.data) == 0
        return out

    def stats(self):
        e, r, n, ms = C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_double()
        assert self.L.sgs_sample_app_stats(self.h, C.byref(e), C.byref(r), C.byref(n), C.byref(ms)) == 0
        return {"edges": e.value, "resets": r.value, "rounds": n.value, "ms": ms.value}

    def close(self):
        if self.h:
            self.L.sgs_sample_app_destroy(self.h)
            self.h = None


def _check(app, m):
    nv, row, col, w = m.nv, m.row, m.col, m.w
    got = app.value()
    if app.kind == PR:
        assert np.max(np.abs(got - O.pagerank(nv, row, col))) <= 1e-6
    elif app.kind == CC:
        assert np.array_equal(got, O.cc(nv, row, col))
    elif app.kind == WIDEST:
        assert np.array_equal(got, O.widest(nv, row, col, w, app.source))
    else:
        ww = w if app.kind == SSSP else None
        d, _ = (O.sssp(nv, row, col, ww, app.source) if app.kind == SSSP else O.bfs(nv, row, col, app.source))
        assert np.array_equal(got, d)
        assert O.check_tree(nv, row, col, ww, app.source, got, app.parent()) == 0


def _stream(nv, row, col, seed, sizes):
    tot_i, tot_d = sum(s[0] for s in sizes), sum(s[1] for s in sizes)
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, seed, tot_i, tot_d)
    iw = O.weights_pairs(1, i_s, i_d)
    out, oi, od = [], 0, 0
    for ni, nd in sizes:
        out.append((i_s[oi:oi + ni], i_d[oi:oi + ni], iw[oi:oi + ni], d_s[od:od + nd], d_d[od:od + nd]))
        oi += ni
        od += nd
    return out


@pytest.mark.parametrize("budget", [0.0, 0.3])
def test_functor_apps_through_snapshots(budget):
    L = _lib()
    nv, row, col = O.rmat_csr(14, 16, 3)
    w = O.weights(nv, row, col, 1, 0)
    kw = {}
    if budget:
        gb = len(col) * 8 / 1e9
        kw = {"hbm_budget_gb": budget * gb, "cache_gb": 0.1 * gb, "segments": 64}
    batches = _stream(nv, row, col, 21, [(3000, 3000), (2000, 0), (0, 2500)])
    with sgs.Engine(**kw) as e:
        e.load_rmat(14, 16, 3, wseed=1)
        if budget:
            assert e.engine_stats()["arena_bytes_host"] > 0
        apps = [App(L, e, BFS, 0), App(L, e, SSSP, 0), App(L, e, CC), App(L, e, WIDEST, 0), App(L, e, PR)]
        built_in = {BFS: e.add_query(sgs.BFS, 0), SSSP: e.add_query(sgs.SSSP, 0), CC: e.add_query(sgs.CC, 0)}
        for a in apps:
            a.start()
            assert a.stats()["rounds"] >= 1
        m = Mirror(nv, row, col, w)
        for a in apps:
            _check(a, m)
        for k, b in enumerate(batches):
            e.apply_batch(*b)
            m.apply(*b)
            for a in apps:
                _check(a, m)
                if a.kind in built_in:
                    assert np.array_equal(a.value(), built_in[a.kind].value()), (k, a.kind)
            st = apps[1].stats()
            assert st["edges"] > 0
            if len(b[3]):
                # some vertex of the SSSP tree lost its parent edge
                assert st["resets"] > 0
        for a in apps:
            a.close()
        # detached: later snapshots do not touch them
        e.apply_batch(*_stream(m.nv, m.row, m.col, 5, [(100, 100)])[0])


def test_functor_apps_widest_with_synth_weights_and_many_sources():
    """Several widest-path sources over the reference's synthesized weights
    ((u+v)%128+1), through snapshots."""
    L = _lib()
    nv, row, col = O.rmat_csr(13, 16, 8)
    wsyn = O.weights(nv, row, col, 0, 1)
    batches = _stream(nv, row, col, 9, [(1500, 1500), (1500, 1500)])
    with sgs.Engine(weight_mode=sgs.W_SYNTH) as e:
        e.load_csr(nv, row, col, None)
        srcs = [0, 5, 77, 4000]
        apps = [App(L, e, WIDEST, s) for s in srcs]
        for a in apps:
            a.start()
        r, c = row, col
        for a in apps:
            assert np.array_equal(a.value(), O.widest(nv, r, c, wsyn, a.source))
        for b in batches:
            e.apply_batch(b[0], b[1], None, b[3], b[4])
            r, c, _ = O.apply(nv, r, c, None, b[0], b[1], None, b[3], b[4])
            ws = O.weights(nv, r, c, 0, 1)
            for a in apps:
                assert np.array_equal(a.value(), O.widest(nv, r, c, ws, a.source))
        for a in apps:
            a.close()


def test_reference_style_functor_runs_the_sample_driver():
    """A functor written like samples/hybrid_sssp (override, AppBase from
    sepgraph::api, utils::pair) driven through sepgraph::engine::Engine's
    LoadGraph / InitGraph / Start / get_update_file / del_edge + add_edge /
    GatherValue on the README example (synthesized weights): distances after
    the two snapshots are those worked by hand."""
    L = _lib()
    out = np.zeros(5, np.uint32)
    rc = L.sgs_sample_refstyle_sssp(os.path.join(FIX, "input.txt").encode(),
                                    os.path.join(FIX, "stream_size.txt").encode(),
                                    os.path.join(FIX, "update.txt").encode(), 0, 2, out.ctypes.data, 5)
    assert rc == 0, sgs.lib().sgs_last_error()
    assert out.tolist() == [0, O.INF, O.INF, 4, 5]
