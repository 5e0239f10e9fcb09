"""Python binding of the B200 streaming-graph engine (``include/sgs.h``).

Thin ctypes layer over ``lib/libsgs.so``; every call goes through the C ABI.
There is no fallback: importing works without a GPU (so CPU tests can check
that the library loads and exports its symbols), but every compute call
needs the CUDA library and a B200, and raises if either is missing.

Two spellings are offered:

* :class:`Engine` -- the C ABI in Python form (load / add_query /
  apply_batch / gather);
* :class:`Ppr` -- differentiable weighted personalized PageRank on a
  prepared graph (``sgs_ppr_*``; the torch op is in :mod:`sgs.autograd`);
* :class:`HybridEngine` -- the call sequence of the reference's sample
  drivers (``samples/hybrid_sssp/hybrid_sssp.cu:204-296``,
  ``samples/hybrid_pr/hybrid_pr.cu:154-200``): ``LoadGraph``, ``InitGraph``,
  ``Start``, per snapshot ``del_edge`` + ``add_edge`` (or ``Cancelation`` +
  ``Compensate`` for PageRank), then ``GatherValue`` / ``GatherParent`` /
  ``GatherBuffer``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libsgs.so")

BFS, SSSP, CC, PR = 0, 1, 2, 3
ALGOS = {"bfs": BFS, "sssp": SSSP, "cc": CC, "pr": PR}
MEM_HOST, MEM_DEVICE = 0, 1
W_EXPLICIT, W_SYNTH, W_UNIT = 0, 1, 2
FIELD_VALUE, FIELD_PARENT, FIELD_BUFFER = 0, 1, 2
INF = 0xFFFFFFFF

OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory",
          -4: "bad state", -5: "not converged"}

EXPORTS = [
    "sgs_version", "sgs_last_error", "sgs_config_default", "sgs_create",
    "sgs_destroy", "sgs_load_csr", "sgs_load_edge_list", "sgs_load_rmat",
    "sgs_query_add", "sgs_query_add_many", "sgs_query_remove", "sgs_apply_batch", "sgs_gather",
    "sgs_get_query_stats", "sgs_get_engine_stats", "sgs_graph_export",
    "sgs_synchronize", "sgs_kernel_timing", "sgs_get_kernel_stats",
    "sgs_query_summary", "sgs_gen_update_stream", "sgs_hash_weights",
    "sgs_read_edge_list", "sgs_read_stream_sizes", "sgs_read_update_file", "sgs_free",
    "sgs_ppr_create_csr", "sgs_ppr_create", "sgs_ppr_destroy", "sgs_ppr_info",
    "sgs_ppr_export", "sgs_ppr_forward", "sgs_ppr_backward", "sgs_ppr_timing",
    "sgs_ppr_get_stats", "sgs_serve", "sgs_autotune", "sgs_cache_refresh",
    "sgs_stage_batch", "sgs_apply_staged", "sgs_query_summaries",
]

K_GROUP, K_GROUP_INVAL, K_PR_PUSH, K_WIDE, K_WIDE_INVAL, K_PR_PULL, K_GROUP_SWEEP = range(7)
KERNEL_KINDS = {"group_relax": K_GROUP, "group_invalidate": K_GROUP_INVAL, "pr_push": K_PR_PUSH,
                "wide_relax": K_WIDE, "wide_invalidate": K_WIDE_INVAL, "pr_pull": K_PR_PULL,
                "group_sweep": K_GROUP_SWEEP}


class SgsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("device", C.c_int),
        ("segments", C.c_uint32),
        ("n_stream", C.c_uint32),
        ("block_size", C.c_uint32),
        ("cache_gb", C.c_double),
        ("hbm_budget_gb", C.c_double),
        ("weight_mode", C.c_int),
        ("max_rounds", C.c_uint32),
        ("pr_alpha", C.c_double),
        ("pr_tol", C.c_double),
        ("slack_div", C.c_uint32),
        ("arena_headroom", C.c_double),
        ("group_size", C.c_uint32),
        ("persistent", C.c_uint32),
        ("pull", C.c_uint32),
        ("host_policy", C.c_uint32),
        ("pr_warm", C.c_uint32),
        ("repair", C.c_uint32),
        ("serve_restarts", C.c_uint32),
    ]


class QueryStats(C.Structure):
    _fields_ = [
        ("edges_traversed", C.c_uint64),
        ("edges_total", C.c_uint64),
        ("invalidated", C.c_uint64),
        ("rounds", C.c_uint32),
        ("converged", C.c_uint32),
        ("ms", C.c_double),
        ("pr_residual_l1", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EngineStats(C.Structure):
    _fields_ = [
        ("nv", C.c_uint64),
        ("ne", C.c_uint64),
        ("slots", C.c_uint64),
        ("arena_bytes_hbm", C.c_uint64),
        ("arena_bytes_host", C.c_uint64),
        ("hbm_resident_vertices", C.c_uint64),
        ("last_inserted", C.c_uint64),
        ("last_deleted", C.c_uint64),
        ("last_relocated", C.c_uint64),
        ("repacks", C.c_uint64),
        ("last_apply_ms", C.c_double),
        ("last_batch_ms", C.c_double),
        ("kernel_launches", C.c_uint64),
        ("last_batch_edges", C.c_uint64),
        ("cache_lines", C.c_uint64),
        ("cache_resident", C.c_uint64),
        ("cache_admissions", C.c_uint64),
        ("last_admitted", C.c_uint64),
        ("last_evicted", C.c_uint64),
        ("cache_hit_slots", C.c_uint64),
        ("cache_miss_slots", C.c_uint64),
        ("in_store_bytes", C.c_uint64),
        ("in_store_builds", C.c_uint64),
        ("bfs_bottom_up_rounds", C.c_uint64),
        ("host_stagings", C.c_uint64),
        ("last_stage_bytes", C.c_uint64),
        ("pr_warm_starts", C.c_uint64),
        ("reclaimed_slots", C.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class KernelStats(C.Structure):
    _fields_ = [
        ("launches", C.c_uint64),
        ("slots", C.c_uint64),
        ("entries", C.c_uint64),
        ("bytes_alg", C.c_double),
        ("ms", C.c_double),
        ("max_slots", C.c_uint64),
        ("max_entries", C.c_uint64),
        ("max_bytes_alg", C.c_double),
        ("max_ms", C.c_double),
        ("host_slots", C.c_uint64),
        ("max_host_slots", C.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


REQ_QUERY, REQ_UPDATE = 0, 1


class Request(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("algo", C.c_int), ("source", C.c_uint32), ("reserved", C.c_uint32),
        ("arrival_s", C.c_double), ("value_out", C.c_void_p), ("parent_out", C.c_void_p),
        ("ins_src", C.c_void_p), ("ins_dst", C.c_void_p), ("ins_w", C.c_void_p),
        ("del_src", C.c_void_p), ("del_dst", C.c_void_p),
        ("n_ins", C.c_uint64), ("n_del", C.c_uint64),
    ]


class Completion(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("batch", C.c_uint32), ("version", C.c_uint64),
        ("start_s", C.c_double), ("done_s", C.c_double),
        ("summary", C.c_uint64 * 4), ("edges", C.c_uint64),
        ("restarts", C.c_uint32), ("reserved", C.c_uint32),
    ]


class Tune(C.Structure):
    _fields_ = [("ctas_per_sm", C.c_uint32), ("persistent", C.c_uint32), ("best_ms", C.c_double),
                ("tried", C.c_uint32)]


class PprStats(C.Structure):
    _fields_ = [
        ("iters", C.c_int32),
        ("pieces_in", C.c_uint32),
        ("pieces_out", C.c_uint32),
        ("reserved", C.c_uint32),
        ("ms", C.c_double),
        ("steps_ms", C.c_double),
        ("bytes_alg_step", C.c_double),
        ("kernel_launches", C.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_lib = None


def lib():
    """Loads lib/libsgs.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {PKG}`")
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, i32, dbl = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double
    L.sgs_version.restype = C.c_char_p
    L.sgs_last_error.restype = C.c_char_p
    L.sgs_config_default.argtypes = [C.POINTER(Config)]
    L.sgs_config_default.restype = None
    L.sgs_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.sgs_destroy.argtypes = [vp]
    L.sgs_load_csr.argtypes = [vp, u32, vp, vp, vp, i32]
    L.sgs_load_edge_list.argtypes = [vp, u32, u64, vp, vp, vp, i32]
    L.sgs_load_rmat.argtypes = [vp, u32, u32, u64, dbl, dbl, dbl, u64]
    L.sgs_query_add.argtypes = [vp, i32, u32, C.POINTER(i32)]
    L.sgs_query_add_many.argtypes = [vp, u32, vp, vp, vp]
    L.sgs_query_remove.argtypes = [vp, i32]
    L.sgs_apply_batch.argtypes = [vp, vp, vp, vp, u64, vp, vp, u64, i32]
    L.sgs_gather.argtypes = [vp, i32, i32, vp, i32]
    L.sgs_get_query_stats.argtypes = [vp, i32, C.POINTER(QueryStats)]
    L.sgs_get_engine_stats.argtypes = [vp, C.POINTER(EngineStats)]
    L.sgs_graph_export.argtypes = [vp, vp, vp, vp, i32]
    L.sgs_synchronize.argtypes = [vp]
    L.sgs_kernel_timing.argtypes = [vp, i32]
    L.sgs_get_kernel_stats.argtypes = [vp, i32, C.POINTER(KernelStats)]
    L.sgs_query_summary.argtypes = [vp, i32, vp]
    L.sgs_gen_update_stream.argtypes = [u32, vp, vp, u64, u64, u64, vp, vp, vp, vp]
    L.sgs_hash_weights.argtypes = [u64, u64, vp, vp, vp]
    L.sgs_hash_weights.restype = None
    pp = C.POINTER(C.c_void_p)
    L.sgs_read_edge_list.argtypes = [C.c_char_p, C.POINTER(u32), C.POINTER(u64), pp, pp, pp]
    L.sgs_read_stream_sizes.argtypes = [C.c_char_p, C.POINTER(u32), pp, pp]
    L.sgs_read_update_file.argtypes = [C.c_char_p, C.POINTER(u64), pp, pp, pp, C.POINTER(u64),
                                       pp, pp, pp]
    L.sgs_free.argtypes = [vp]
    L.sgs_free.restype = None
    L.sgs_ppr_create_csr.argtypes = [i32, u32, vp, vp, i32, C.POINTER(vp)]
    L.sgs_ppr_create.argtypes = [vp, C.POINTER(vp)]
    L.sgs_ppr_destroy.argtypes = [vp]
    L.sgs_ppr_info.argtypes = [vp, C.POINTER(u32), C.POINTER(u64)]
    L.sgs_ppr_export.argtypes = [vp, vp, vp, i32]
    L.sgs_ppr_forward.argtypes = [vp, vp, vp, u32, dbl, dbl, u32, vp, C.POINTER(i32), i32]
    L.sgs_ppr_backward.argtypes = [vp, vp, vp, vp, u32, dbl, dbl, u32, vp, vp, C.POINTER(i32), i32]
    L.sgs_ppr_timing.argtypes = [vp, i32]
    L.sgs_serve.argtypes = [vp, C.POINTER(Request), u32, u32, i32, C.POINTER(Completion)]
    L.sgs_autotune.argtypes = [vp, C.POINTER(Tune)]
    L.sgs_cache_refresh.argtypes = [vp]
    L.sgs_stage_batch.argtypes = [vp, vp, vp, vp, u64, vp, vp, u64, i32]
    L.sgs_apply_staged.argtypes = [vp]
    L.sgs_query_summaries.argtypes = [vp, u32, vp, vp]
    L.sgs_ppr_get_stats.argtypes = [vp, C.POINTER(PprStats)]
    for name in EXPORTS:
        if name not in ("sgs_version", "sgs_last_error", "sgs_config_default",
                        "sgs_hash_weights", "sgs_free"):
            getattr(L, name).restype = i32
    _lib = L
    return L


def _check(rc):
    if rc != OK:
        raise SgsError(rc, lib().sgs_last_error().decode())


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):  # device pointer
        return C.c_void_p(a)
    return C.c_void_p(a.ctypes.data)


def _u32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint32)


def default_config(**overrides) -> Config:
    c = Config()
    lib().sgs_config_default(C.byref(c))
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise TypeError(f"unknown config field {k}")
        setattr(c, k, v)
    return c


def gen_update_stream(nv, row, col, seed, n_ins, n_del):
    """Deterministic synthetic update stream w.r.t. a CSR with sorted rows:
    (ins_src, ins_dst, del_src, del_dst)."""
    row = np.ascontiguousarray(row, np.uint64)
    col = np.ascontiguousarray(col, np.uint32)
    out = [np.empty(max(n, 1), np.uint32) for n in (n_ins, n_ins, n_del, n_del)]
    _check(lib().sgs_gen_update_stream(nv, _ptr(row), _ptr(col), seed, n_ins, n_del,
                                       *[_ptr(a) for a in out]))
    return out[0][:n_ins], out[1][:n_ins], out[2][:n_del], out[3][:n_del]


def _take(ptr, n, dtype):
    """Copies n elements out of a library-allocated array and frees it."""
    if not ptr:
        return None
    ct = C.c_uint32 if dtype == np.uint32 else C.c_uint64
    out = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(max(n, 1),))[:n].copy()
    lib().sgs_free(ptr)
    return out.astype(dtype, copy=False)


def read_edge_list(path):
    """market_big edge list: (nv, src, dst, w or None), edges in file order."""
    nv, ne = C.c_uint32(), C.c_uint64()
    s, d, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(lib().sgs_read_edge_list(str(path).encode(), C.byref(nv), C.byref(ne), C.byref(s),
                                    C.byref(d), C.byref(w)))
    n = ne.value
    return nv.value, _take(s.value, n, np.uint32), _take(d.value, n, np.uint32), \
        _take(w.value, n, np.uint32)


def read_stream_sizes(path):
    """Stream-size file: (adds[k], dels[k]) per snapshot."""
    n = C.c_uint32()
    a, d = C.c_void_p(), C.c_void_p()
    _check(lib().sgs_read_stream_sizes(str(path).encode(), C.byref(n), C.byref(a), C.byref(d)))
    return _take(a.value, n.value, np.uint64), _take(d.value, n.value, np.uint64)


def read_update_file(path):
    """Update file: dict of add_u/add_v/add_w and del_u/del_v/del_w arrays."""
    na, nd = C.c_uint64(), C.c_uint64()
    ptrs = [C.c_void_p() for _ in range(6)]
    _check(lib().sgs_read_update_file(str(path).encode(), C.byref(na), C.byref(ptrs[0]),
                                      C.byref(ptrs[1]), C.byref(ptrs[2]), C.byref(nd),
                                      C.byref(ptrs[3]), C.byref(ptrs[4]), C.byref(ptrs[5])))
    names = ["add_u", "add_v", "add_w", "del_u", "del_v", "del_w"]
    counts = [na.value] * 3 + [nd.value] * 3
    return {k: _take(p.value, n, np.uint32) for k, p, n in zip(names, ptrs, counts)}


def hash_weights(wseed, src, dst):
    src, dst = _u32(src), _u32(dst)
    w = np.empty(max(len(src), 1), np.uint32)
    lib().sgs_hash_weights(wseed, len(src), _ptr(src), _ptr(dst), _ptr(w))
    return w[: len(src)]


class Query:
    def __init__(self, engine, qid, algo, source):
        self.engine, self.qid, self.algo, self.source = engine, qid, algo, source

    def value(self):
        return self.engine.gather(self.qid, FIELD_VALUE)

    def parent(self):
        return self.engine.gather(self.qid, FIELD_PARENT)

    def buffer(self):
        return self.engine.gather(self.qid, FIELD_BUFFER)

    def stats(self):
        return self.engine.query_stats(self.qid)

    def summary(self):
        return self.engine.summary(self.qid)


class Engine:
    """One dynamic graph plus registered queries on one GPU."""

    def __init__(self, config: Config | None = None, **overrides):
        self.cfg = config if config is not None else default_config(**overrides)
        h = C.c_void_p()
        _check(lib().sgs_create(C.byref(self.cfg), C.byref(h)))
        self.h = h
        self.nv = 0
        self._queries = {}

    def close(self):
        if getattr(self, "h", None):
            lib().sgs_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- load
    def load_csr(self, nv, row, col, w=None):
        row = np.ascontiguousarray(row, dtype=np.uint64)
        col, w = _u32(col), _u32(w)
        _check(lib().sgs_load_csr(self.h, nv, _ptr(row), _ptr(col), _ptr(w), MEM_HOST))
        self.nv = nv
        self._queries.clear()

    def load_edge_list(self, src, dst, w=None, nv=0):
        src, dst, w = _u32(src), _u32(dst), _u32(w)
        _check(lib().sgs_load_edge_list(self.h, nv, len(src), _ptr(src), _ptr(dst), _ptr(w), MEM_HOST))
        self.nv = int(self.engine_stats()["nv"])
        self._queries.clear()

    def load_rmat(self, scale, edge_factor=16, seed=1, a=0.57, b=0.19, c=0.19, wseed=1):
        _check(lib().sgs_load_rmat(self.h, scale, edge_factor, seed, a, b, c, wseed))
        self.nv = 1 << scale
        self._queries.clear()

    # -- queries
    def add_query(self, algo, source=0) -> Query:
        if isinstance(algo, str):
            algo = ALGOS[algo]
        qid = C.c_int()
        _check(lib().sgs_query_add(self.h, algo, source, C.byref(qid)))
        q = Query(self, qid.value, algo, source)
        self._queries[qid.value] = q
        return q

    def add_queries(self, specs):
        """Registers many queries at once: specs = [(algo, source), ...].  The
        BFS/SSSP/CC ones share group lanes and converge together."""
        specs = [(ALGOS[a] if isinstance(a, str) else int(a), int(src)) for a, src in specs]
        n = len(specs)
        algos = np.array([a for a, _ in specs], np.int32)
        srcs = np.array([x for _, x in specs], np.uint32)
        ids = np.zeros(max(n, 1), np.int32)
        _check(lib().sgs_query_add_many(self.h, n, _ptr(algos), _ptr(srcs), _ptr(ids)))
        out = []
        for i, (a, src) in enumerate(specs):
            q = Query(self, int(ids[i]), a, src)
            self._queries[q.qid] = q
            out.append(q)
        return out

    def serve(self, requests, slots=0, realtime=True):
        """Runs sgs_serve over a trace.  requests: dicts with kind "query"
        (algo, source, arrival_s, optional value_out / parent_out numpy
        buffers) or "update" (ins_src, ins_dst, ins_w, del_src, del_dst,
        arrival_s).  Returns one dict per request."""
        n = len(requests)
        arr = (Request * max(n, 1))()
        keep = []
        for i, r in enumerate(requests):
            q = arr[i]
            q.arrival_s = float(r.get("arrival_s", 0.0))
            if r["kind"] == "query":
                q.kind = REQ_QUERY
                a = r["algo"]
                q.algo = ALGOS[a] if isinstance(a, str) else int(a)
                q.source = int(r.get("source", 0))
                for f in ("value_out", "parent_out"):
                    b = r.get(f)
                    if b is not None:
                        keep.append(b)
                        setattr(q, f, b.ctypes.data)
            else:
                q.kind = REQ_UPDATE
                for f in ("ins_src", "ins_dst", "ins_w", "del_src", "del_dst"):
                    b = r.get(f)
                    if b is not None:
                        b = _u32(b)
                        keep.append(b)
                        setattr(q, f, b.ctypes.data)
                q.n_ins = len(r.get("ins_src", ()))
                q.n_del = len(r.get("del_src", ()))
        out = (Completion * max(n, 1))()
        _check(lib().sgs_serve(self.h, arr, n, slots, int(realtime), out))
        res = []
        for i in range(n):
            c = out[i]
            res.append({"status": c.status, "batch": c.batch, "version": c.version,
                        "start_s": c.start_s, "done_s": c.done_s,
                        # closed loop (not realtime): every request counts as
                        # arrived at the start
                        "latency_s": c.done_s - (arr[i].arrival_s if realtime else 0.0),
                        "summary": list(c.summary), "edges": c.edges, "restarts": c.restarts})
        return res

    def autotune(self):
        """sgs_autotune: picks the relaxation map's CTAs per SM and the launch
        mode by timing a probe on the loaded graph; returns the choice."""
        t = Tune()
        _check(lib().sgs_autotune(self.h, C.byref(t)))
        return {"ctas_per_sm": t.ctas_per_sm, "persistent": t.persistent, "best_ms": t.best_ms,
                "tried": t.tried}

    def remove_query(self, q):
        _check(lib().sgs_query_remove(self.h, q.qid if isinstance(q, Query) else q))

    def stage_batch_ptr(self, isp, idp, iwp, ni, dsp, ddp, nd, mem):
        """Copies a batch into a staging slot on the copy stream and returns
        at once (raw pointers, pinned host or device); apply_staged applies it."""
        _check(lib().sgs_stage_batch(self.h, _ptr(isp), _ptr(idp), _ptr(iwp), ni,
                                     _ptr(dsp), _ptr(ddp), nd, mem))

    def apply_staged(self):
        _check(lib().sgs_apply_staged(self.h))

    def apply_batch_ptr(self, isp, idp, iwp, ni, dsp, ddp, nd, mem):
        """Raw-pointer form (host pinned or device memory, as ints)."""
        _check(lib().sgs_apply_batch(self.h, _ptr(isp), _ptr(idp), _ptr(iwp), ni,
                                     _ptr(dsp), _ptr(ddp), nd, mem))

    def apply_batch(self, ins_src=(), ins_dst=(), ins_w=None, del_src=(), del_dst=(), mem=MEM_HOST):
        if mem == MEM_DEVICE:
            # device pointers (ints) with explicit counts: (ptr, n) tuples
            (isp, ni), (idp, _), (dsp, nd), (ddp, _) = ins_src, ins_dst, del_src, del_dst
            iwp = ins_w[0] if ins_w is not None else None
            _check(lib().sgs_apply_batch(self.h, _ptr(isp), _ptr(idp), _ptr(iwp), ni,
                                         _ptr(dsp), _ptr(ddp), nd, MEM_DEVICE))
            return
        isrc, idst, iw = _u32(ins_src), _u32(ins_dst), _u32(ins_w)
        dsrc, ddst = _u32(del_src), _u32(del_dst)
        _check(lib().sgs_apply_batch(self.h, _ptr(isrc), _ptr(idst), _ptr(iw), len(isrc),
                                     _ptr(dsrc), _ptr(ddst), len(dsrc), MEM_HOST))

    def gather(self, qid, field=FIELD_VALUE):
        q = self._queries.get(qid)
        pr = q is not None and q.algo == PR
        out = np.empty(self.nv, np.float64 if pr else np.uint32)
        _check(lib().sgs_gather(self.h, qid, field, _ptr(out), MEM_HOST))
        return out

    def query_stats(self, qid):
        s = QueryStats()
        _check(lib().sgs_get_query_stats(self.h, qid, C.byref(s)))
        return s.as_dict()

    def summary(self, qid):
        out = np.zeros(4, np.uint64)
        _check(lib().sgs_query_summary(self.h, qid, _ptr(out)))
        return out

    def summaries(self, queries):
        """[n, 4] summaries of several queries (Query objects or ids), one read-back."""
        ids = np.array([q.qid if isinstance(q, Query) else q for q in queries], np.int32)
        out = np.zeros((len(ids), 4), np.uint64)
        _check(lib().sgs_query_summaries(self.h, len(ids), _ptr(ids), _ptr(out)))
        return out

    def engine_stats(self):
        s = EngineStats()
        _check(lib().sgs_get_engine_stats(self.h, C.byref(s)))
        return s.as_dict()

    def export(self, weights=False):
        st = self.engine_stats()
        nv, ne = int(st["nv"]), int(st["ne"])
        row = np.empty(nv + 1, np.uint64)
        col = np.empty(max(ne, 1), np.uint32)
        w = np.empty(max(ne, 1), np.uint32) if weights else None
        _check(lib().sgs_graph_export(self.h, _ptr(row), _ptr(col), _ptr(w), MEM_HOST))
        return row, col[:ne], (None if w is None else w[:ne])

    def synchronize(self):
        _check(lib().sgs_synchronize(self.h))

    def cache_refresh(self):
        """Edge-cache admission now, from the current hotness window; returns
        when the admitted lines are visible (no-op without a cache)."""
        _check(lib().sgs_cache_refresh(self.h))

    def kernel_timing(self, enable=True):
        _check(lib().sgs_kernel_timing(self.h, int(enable)))

    def kernel_stats(self):
        out = {}
        for name, k in KERNEL_KINDS.items():
            s = KernelStats()
            _check(lib().sgs_get_kernel_stats(self.h, k, C.byref(s)))
            out[name] = s.as_dict()
        return out


class HybridEngine:
    """The reference sample drivers' call sequence over :class:`Engine`.

    ``algo`` is one of "pr", "sssp", "bfs", "cc" (the HybridPageRank /
    HybridSSSP / HybridBFS / HybridCC drivers).  Snapshots come from the
    reference's update-file format (see :mod:`sgs.io`).
    """

    def __init__(self, algo, **cfg):
        self.algo = ALGOS[algo] if isinstance(algo, str) else algo
        self.engine = Engine(**cfg)
        self.q = None
        self._source = 0
        self._pending = None

    # Engine::LoadGraph
    def LoadGraph(self, src=None, dst=None, w=None, nv=0, csr=None):
        if csr is not None:
            self.engine.load_csr(*csr)
        else:
            self.engine.load_edge_list(src, dst, w, nv)

    # Engine::InitGraph(args...): the source node (SSSP/BFS), error (PR)
    def InitGraph(self, arg=0):
        if self.algo in (SSSP, BFS):
            self._source = int(arg)

    # Engine::Start: static convergence
    def Start(self):
        self.q = self.engine.add_query(self.algo, self._source)
        return self.q.stats()

    # SSSP/BFS/CC snapshot: del_edge(...) then add_edge(...)
    def del_edge(self, del_src, del_dst):
        self._pending = (np.asarray(del_src, np.uint32), np.asarray(del_dst, np.uint32))

    def add_edge(self, ins_src, ins_dst, ins_w=None):
        d = self._pending or (np.empty(0, np.uint32), np.empty(0, np.uint32))
        self._pending = None
        self.engine.apply_batch(ins_src, ins_dst, ins_w, d[0], d[1])
        return self.q.stats()

    # PR snapshot: Cancelation(...) then Compensate(...)
    Cancelation = del_edge
    Compensate = add_edge

    def GatherValue(self):
        return self.q.value()

    def GatherParent(self):
        return self.q.parent()

    def GatherBuffer(self):
        return self.q.buffer()

    def GetNodeNum(self):
        return self.engine.nv


class Ppr:
    """A graph prepared for differentiable weighted personalized PageRank
    (``sgs_ppr_*``): FP64 forward X = (1-alpha) T + alpha P^T X and its
    adjoint.  Edge weights are given per edge in the CSR order of the
    prepared graph (:meth:`export`).

    Arrays may be numpy (host) or CUDA torch tensors (device, float64,
    contiguous); results come back in the same form as ``T`` / ``X``.
    ``tol`` is the L1 change of one Jacobi step summed over all nv*K entries
    below which the iteration stops (default 1e-13 * nv * K).
    """

    def __init__(self, nv=None, row=None, col=None, engine: Engine | None = None, device=0):
        h = C.c_void_p()
        if engine is not None:
            _check(lib().sgs_ppr_create(engine.h, C.byref(h)))
        else:
            row = np.ascontiguousarray(row, np.uint64)
            col = np.ascontiguousarray(col, np.uint32)
            _check(lib().sgs_ppr_create_csr(device, nv, _ptr(row), _ptr(col), MEM_HOST, C.byref(h)))
        self.h = h
        n, m = C.c_uint32(), C.c_uint64()
        _check(lib().sgs_ppr_info(self.h, C.byref(n), C.byref(m)))
        self.nv, self.ne = n.value, m.value
        self.last_iters = 0

    def close(self):
        if self.h:
            lib().sgs_ppr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def export(self):
        row = np.empty(self.nv + 1, np.uint64)
        col = np.empty(max(self.ne, 1), np.uint32)
        _check(lib().sgs_ppr_export(self.h, _ptr(row), _ptr(col), MEM_HOST))
        return row, col[: self.ne]

    def timing(self, enable=True):
        """Per-step CUDA events (steps_ms in :meth:`stats`)."""
        _check(lib().sgs_ppr_timing(self.h, int(enable)))

    def stats(self):
        st = PprStats()
        _check(lib().sgs_ppr_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def _tol(self, tol, K):
        return 1e-13 * self.nv * K if tol is None else float(tol)

    @staticmethod
    def _is_torch(a):
        return type(a).__module__.startswith("torch")

    @staticmethod
    def _dev_args(*arrs):
        import torch

        for a in arrs:
            if a is None:
                continue
            if not (a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()):
                raise ValueError("device arrays must be contiguous float64 CUDA tensors")
        # the library runs on its own stream: make the caller's work visible
        torch.cuda.current_stream().synchronize()

    def forward(self, w, T, alpha=0.85, tol=None, max_iter=100000):
        it = C.c_int()
        if self._is_torch(T):
            import torch

            T2 = T.reshape(self.nv, -1)
            K = T2.shape[1]
            X = torch.empty_like(T2)
            self._dev_args(w, T2, X)
            _check(lib().sgs_ppr_forward(self.h, w.data_ptr(), T2.data_ptr(), K, alpha,
                                         self._tol(tol, K), max_iter, X.data_ptr(), C.byref(it),
                                         MEM_DEVICE))
        else:
            w = np.ascontiguousarray(w, np.float64)
            T2 = np.ascontiguousarray(np.asarray(T, np.float64).reshape(self.nv, -1))
            K = T2.shape[1]
            X = np.empty_like(T2)
            _check(lib().sgs_ppr_forward(self.h, _ptr(w), _ptr(T2), K, alpha, self._tol(tol, K),
                                         max_iter, _ptr(X), C.byref(it), MEM_HOST))
        self.last_iters = it.value
        return X

    def backward(self, w, X, G, alpha=0.85, tol=None, max_iter=100000, want_w=True, want_T=True):
        """(dL/dw, dL/dT) for the upstream gradient G = dL/dX."""
        it = C.c_int()
        if self._is_torch(X):
            import torch

            K = X.shape[1]
            G = G.reshape(self.nv, K).contiguous()
            gw = torch.empty(max(self.ne, 1), dtype=torch.float64, device=X.device) if want_w else None
            gT = torch.empty_like(X) if want_T else None
            self._dev_args(w, X, G, gw, gT)
            _check(lib().sgs_ppr_backward(self.h, w.data_ptr(), X.data_ptr(), G.data_ptr(), K,
                                          alpha, self._tol(tol, K), max_iter,
                                          gw.data_ptr() if gw is not None else None,
                                          gT.data_ptr() if gT is not None else None,
                                          C.byref(it), MEM_DEVICE))
        else:
            w = np.ascontiguousarray(w, np.float64)
            X = np.ascontiguousarray(X, np.float64)
            K = X.shape[1]
            G = np.ascontiguousarray(np.asarray(G, np.float64).reshape(self.nv, K))
            gw = np.empty(max(self.ne, 1)) if want_w else None
            gT = np.empty_like(X) if want_T else None
            _check(lib().sgs_ppr_backward(self.h, _ptr(w), _ptr(X), _ptr(G), K, alpha,
                                          self._tol(tol, K), max_iter, _ptr(gw), _ptr(gT),
                                          C.byref(it), MEM_HOST))
        gw = gw[: self.ne] if gw is not None else None
        self.last_iters = it.value
        return gw, gT
