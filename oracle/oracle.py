"""CPU oracle bindings (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker or the timed CPU path.  The
product library (``c-gpustreamgraph_b200``) never imports it.

Two native libraries are wrapped:

* ``liboracle.so`` -- the plain-C restatement in ``sgs_oracle.c`` (built by
  ``make`` in this folder);
* ``_ref/libsgsref.so`` -- the reference's own host oracles and host PMA
  (``SSSPHostNaive``, ``BFSHost``, ``PageRankHost``, ``host::PMAGraph``),
  compiled from the reference sources by ``make ref`` where the reference tree
  is available.  Optional: functions raise if it was not built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
INF = 0xFFFFFFFF

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_vp = C.c_void_p

_lib = None
_ref = None


def build(ref: bool = False) -> None:
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])


def _opt(p):
    return None if p is None else p


def lib():
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    u32, u64, i32, dbl = C.c_uint32, C.c_uint64, C.c_int, C.c_double
    sig = {
        "sgso_mix64": (u64, [u64]),
        "sgso_rmat_raw": (None, [u32, u64, u64, u64, u64, u64, _u32p, _u32p]),
        "sgso_rmat_csr_par": (u64, [u32, u32, u64, u64, u64, u64, _u64p, _u32p]),
        "sgso_build_csr": (u64, [u32, u64, _u32p, _u32p, i32, i32, _u64p, _u32p]),
        "sgso_csr_file_order": (None, [u32, u64, _u32p, _u32p, _vp, _u64p, _u32p, _vp]),
        "sgso_weight_of": (u32, [u64, u32, u32]),
        "sgso_weights_pairs": (None, [u64, u64, _u32p, _u32p, _u32p]),
        "sgso_weights": (None, [u32, _u64p, _u32p, u64, i32, _u32p]),
        "sgso_gen_updates": (i32, [u32, _u64p, _u32p, u64, u64, u64, _u32p, _u32p, _u32p, _u32p]),
        "sgso_apply": (u64, [u32, _u64p, _u32p, _vp, u64, _u32p, _u32p, _vp, u64,
                             _u32p, _u32p, _u64p, _u32p, _vp, u64]),
        "sgso_apply_refexact": (u64, [u32, _u64p, _u32p, u64, _u32p, _u32p, u64, _u32p, _u32p,
                                      _u64p, _u32p, u64]),
        "sgso_bfs": (u64, [u32, _u64p, _u32p, u32, _u32p, _vp]),
        "sgso_sssp": (u64, [u32, _u64p, _u32p, _vp, u32, _u32p, _vp]),
        "sgso_cc": (u64, [u32, _u64p, _u32p, _u32p]),
        "sgso_widest": (u64, [u32, _u64p, _u32p, _vp, u32, _u32p]),
        "sgso_pagerank": (i32, [u32, _u64p, _u32p, dbl, dbl, i32, _f64p]),
        "sgso_sssp_fifo_budget": (u64, [u32, _u64p, _u32p, _vp, u32, _u32p, u64]),
        "sgso_bfs_fifo_budget": (u64, [u32, _u64p, _u32p, u32, _u32p, u64]),
        "sgso_pr_host_float": (u64, [u32, _u64p, _u32p, dbl, dbl, _f32p]),
        "sgso_check_tree": (u64, [u32, _u64p, _u32p, _vp, u32, _u32p, _u32p]),
        "sgso_check_cc_parent": (u64, [u32, _u64p, _u32p, _u32p, _u32p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ref_lib():
    """The reference's own host code (oracle/_ref), or None if not built."""
    global _ref
    if _ref is not None:
        return _ref
    path = os.path.join(HERE, "_ref", "libsgsref.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    u32, u64, dbl = C.c_uint32, C.c_uint64, C.c_double
    L.ref_sssp_host.argtypes = [u32, _u64p, _u32p, u32, _u32p]
    L.ref_bfs_host.argtypes = [u32, _u64p, _u32p, u32, _u32p]
    L.ref_pr_host.argtypes = [u32, _u64p, _u32p, dbl, _f32p]
    L.ref_graph_create.restype = _vp
    L.ref_graph_create.argtypes = [u32, _u64p, _u32p]
    L.ref_graph_destroy.argtypes = [_vp]
    L.ref_graph_bfs.argtypes = [_vp, u32, _u32p]
    L.ref_graph_sssp.argtypes = [_vp, u32, _u32p]
    L.ref_pma_create.restype = _vp
    L.ref_pma_create.argtypes = [u32, _u64p, _u32p]
    L.ref_pma_insert.argtypes = [_vp, u32, u32]
    L.ref_pma_del.argtypes = [_vp, u32, u32]
    L.ref_pma_apply.argtypes = [_vp, u64, _u32p, _u32p, u64, _u32p, _u32p]
    L.ref_pma_export.restype = u64
    L.ref_pma_export.argtypes = [_vp, _u64p, _u32p, u64]
    L.ref_pma_destroy.argtypes = [_vp]
    _ref = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- generators
def rmat_thresholds(a=0.57, b=0.19, c=0.19):
    """Integer thresholds floor(p * 2^53) for the cumulative quadrant
    probabilities; shared with the device generator."""
    s = float(1 << 53)
    return int(a * s), int((a + b) * s), int((a + b + c) * s)


def rmat_csr(scale, edge_factor=16, seed=1, a=0.57, b=0.19, c=0.19):
    """Directed R-MAT, self-loops and duplicates removed, rows sorted."""
    nv = 1 << scale
    ne = nv * edge_factor
    tA, tAB, tABC = rmat_thresholds(a, b, c)
    src = np.empty(ne, np.uint32)
    dst = np.empty(ne, np.uint32)
    L = lib()
    L.sgso_rmat_raw(scale, ne, seed, tA, tAB, tABC, src, dst)
    row = np.empty(nv + 1, np.uint64)
    col = np.empty(ne, np.uint32)
    m = L.sgso_build_csr(nv, ne, src, dst, 1, 1, row, col)
    return nv, row, col[:m].copy()


def rmat_csr_par(scale, edge_factor=16, seed=1, a=0.57, b=0.19, c=0.19):
    """rmat_csr built with OpenMP threads (same graph)."""
    nv = 1 << scale
    tA, tAB, tABC = rmat_thresholds(a, b, c)
    row = np.empty(nv + 1, np.uint64)
    col = np.empty(nv * edge_factor, np.uint32)
    m = lib().sgso_rmat_csr_par(scale, edge_factor, seed, tA, tAB, tABC, row, col)
    return nv, row, col[:m]


def csr_from_edges(nv, src, dst, dedupe=True, drop_self=True):
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    row = np.empty(nv + 1, np.uint64)
    col = np.empty(max(len(src), 1), np.uint32)
    m = lib().sgso_build_csr(nv, len(src), src, dst, int(dedupe), int(drop_self), row, col)
    return row, col[:m].copy()


def csr_file_order(nv, src, dst, w=None):
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    row = np.empty(nv + 1, np.uint64)
    col = np.empty(max(len(src), 1), np.uint32)
    wout = None
    if w is not None:
        w = np.ascontiguousarray(w, np.uint32)
        wout = np.empty(max(len(src), 1), np.uint32)
    lib().sgso_csr_file_order(nv, len(src), src, dst, _ptr(w), row, col, _ptr(wout))
    m = len(src)
    return row, col[:m].copy(), (None if wout is None else wout[:m].copy())


def weights(nv, row, col, wseed=1, mode=0):
    """mode 0: uniform [1,64] from seed; 1: reference synth (u+v)%128+1; 2: unit."""
    w = np.empty(max(len(col), 1), np.uint32)
    lib().sgso_weights(nv, row, col, wseed, mode, w)
    return w[: len(col)].copy()


def weight_of(wseed, u, v):
    return lib().sgso_weight_of(wseed, u, v)


def weights_pairs(wseed, u, v):
    """weight_of for every pair of two equal-length id arrays."""
    u = np.ascontiguousarray(u, np.uint32)
    v = np.ascontiguousarray(v, np.uint32)
    w = np.empty(max(len(u), 1), np.uint32)
    lib().sgso_weights_pairs(wseed, len(u), u, v, w)
    return w[: len(u)].copy()


def gen_updates(nv, row, col, seed, n_ins, n_del):
    ins_s = np.empty(max(n_ins, 1), np.uint32)
    ins_d = np.empty(max(n_ins, 1), np.uint32)
    del_s = np.empty(max(n_del, 1), np.uint32)
    del_d = np.empty(max(n_del, 1), np.uint32)
    rc = lib().sgso_gen_updates(nv, row, col, seed, n_ins, n_del, ins_s, ins_d, del_s, del_d)
    if rc != 0:
        raise ValueError("update generation failed (graph too small or too dense)")
    return ins_s[:n_ins].copy(), ins_d[:n_ins].copy(), del_s[:n_del].copy(), del_d[:n_del].copy()


# ---------------------------------------------------------------- snapshot apply
def apply(nv, row, col, w, ins_s, ins_d, ins_w, del_s, del_d):
    ins_s = np.ascontiguousarray(ins_s, np.uint32)
    ins_d = np.ascontiguousarray(ins_d, np.uint32)
    del_s = np.ascontiguousarray(del_s, np.uint32)
    del_d = np.ascontiguousarray(del_d, np.uint32)
    if ins_w is not None:
        ins_w = np.ascontiguousarray(ins_w, np.uint32)
    cap = len(col) + len(ins_s) + 1
    row_o = np.empty(nv + 1, np.uint64)
    col_o = np.empty(cap, np.uint32)
    w_o = np.empty(cap, np.uint32) if w is not None else None
    m = lib().sgso_apply(nv, row, col, _ptr(w), len(ins_s), ins_s, ins_d, _ptr(ins_w),
                         len(del_s), del_s, del_d, row_o, col_o, _ptr(w_o), cap)
    assert m != 2**64 - 1
    return row_o, col_o[:m].copy(), (None if w_o is None else w_o[:m].copy())


def apply_refexact(nv, row, col, ins_s, ins_d, del_s, del_d):
    """Snapshot apply reproducing the reference PMA exactly (see
    sgso_apply_refexact); only for pinning the oracle."""
    ins_s = np.ascontiguousarray(ins_s, np.uint32)
    ins_d = np.ascontiguousarray(ins_d, np.uint32)
    del_s = np.ascontiguousarray(del_s, np.uint32)
    del_d = np.ascontiguousarray(del_d, np.uint32)
    cap = len(col) + len(ins_s) + 1
    row_o = np.empty(nv + 1, np.uint64)
    col_o = np.empty(cap, np.uint32)
    m = lib().sgso_apply_refexact(nv, row, col, len(ins_s), ins_s, ins_d, len(del_s),
                                  del_s, del_d, row_o, col_o, cap)
    assert m != 2**64 - 1
    return row_o, col_o[:m].copy()


# ---------------------------------------------------------------- ground truth
def bfs(nv, row, col, source):
    d = np.empty(nv, np.uint32)
    p = np.empty(nv, np.uint32)
    lib().sgso_bfs(nv, row, col, source, d, _ptr(p))
    return d, p


def sssp(nv, row, col, w, source):
    d = np.empty(nv, np.uint32)
    p = np.empty(nv, np.uint32)
    lib().sgso_sssp(nv, row, col, _ptr(w), source, d, _ptr(p))
    return d, p


def widest(nv, row, col, w, source):
    """Widest-path widths from source (2^32-1 at the source, 0 unreachable)."""
    out = np.empty(max(nv, 1), np.uint32)
    wa = None if w is None else np.ascontiguousarray(w, np.uint32)
    lib().sgso_widest(nv, row, col, _ptr(wa), source, out)
    return out[:nv]


def cc(nv, row, col):
    lab = np.empty(nv, np.uint32)
    lib().sgso_cc(nv, row, col, lab)
    return lab


def pagerank(nv, row, col, alpha=0.85, tol=1e-14, max_iter=10000):
    x = np.empty(max(nv, 1), np.float64)
    lib().sgso_pagerank(nv, row, col, alpha, tol, max_iter, x)
    return x[:nv]


def sssp_fifo(nv, row, col, w, source, max_edges=2**64 - 1):
    d = np.empty(nv, np.uint32)
    e = lib().sgso_sssp_fifo_budget(nv, row, col, _ptr(w), source, d, max_edges)
    return d, e


def bfs_fifo(nv, row, col, source, max_edges=2**64 - 1):
    d = np.empty(nv, np.uint32)
    e = lib().sgso_bfs_fifo_budget(nv, row, col, source, d, max_edges)
    return d, e


def pr_host_float(nv, row, col, alpha=0.85, err=1e-6):
    r = np.empty(max(nv, 1), np.float32)
    lib().sgso_pr_host_float(nv, row, col, alpha, err, r)
    return r[:nv]


def check_tree(nv, row, col, w, source, value, parent):
    return lib().sgso_check_tree(nv, row, col, _ptr(w), source,
                                 np.ascontiguousarray(value, np.uint32),
                                 np.ascontiguousarray(parent, np.uint32))


def check_cc_parent(nv, row, col, label, parent):
    return lib().sgso_check_cc_parent(nv, row, col,
                                      np.ascontiguousarray(label, np.uint32),
                                      np.ascontiguousarray(parent, np.uint32))


# ---------------------------------------------------------------- reference code
class RefPMA:
    """The reference's host::PMAGraph, driven through its own insert/del_edge."""

    def __init__(self, nv, row, col):
        R = ref_lib()
        if R is None:
            raise RuntimeError("oracle/_ref not built (make -C oracle ref)")
        self.R, self.nv = R, nv
        self.row = np.ascontiguousarray(row, np.uint64)
        self.col = np.ascontiguousarray(col, np.uint32)
        self.h = R.ref_pma_create(nv, self.row, self.col)
        self.cap = len(col) + 16

    def insert(self, u, v):
        self.R.ref_pma_insert(self.h, int(u), int(v))
        self.cap += 1

    def delete(self, u, v):
        self.R.ref_pma_del(self.h, int(u), int(v))

    def apply(self, ins_u, ins_v, del_u, del_v):
        """One snapshot in one call: every insert, then every delete."""
        iu, iv = np.ascontiguousarray(ins_u, np.uint32), np.ascontiguousarray(ins_v, np.uint32)
        du, dv = np.ascontiguousarray(del_u, np.uint32), np.ascontiguousarray(del_v, np.uint32)
        self.R.ref_pma_apply(self.h, len(iu), iu, iv, len(du), du, dv)
        self.cap += len(iu)

    def export(self):
        row = np.empty(self.nv + 1, np.uint64)
        col = np.empty(self.cap, np.uint32)
        m = self.R.ref_pma_export(self.h, row, col, self.cap)
        assert m != 2**64 - 1
        return row, col[:m].copy()

    def close(self):
        if self.h:
            self.R.ref_pma_destroy(self.h)
            self.h = None


def ref_sssp_host(nv, row, col, source):
    d = np.empty(nv, np.uint32)
    ref_lib().ref_sssp_host(nv, row, col, source, d)
    return d


def ref_bfs_host(nv, row, col, source):
    d = np.empty(nv, np.uint32)
    ref_lib().ref_bfs_host(nv, row, col, source, d)
    return d


def ref_pr_host(nv, row, col, err=1e-6):
    r = np.empty(max(nv, 1), np.float32)
    ref_lib().ref_pr_host(nv, row, col, err, r)
    return r[:nv]


class RefGraph:
    """A CSR bound once into the reference's groute host::CSRGraph, for timed
    calls of its BFSHost / SSSPHostNaive (ctypes releases the GIL, so calls
    from several Python threads run concurrently)."""

    def __init__(self, nv, row, col):
        R = ref_lib()
        if R is None:
            raise RuntimeError("oracle/_ref not built (make -C oracle ref)")
        self.R, self.nv = R, nv
        self.h = R.ref_graph_create(nv, np.ascontiguousarray(row, np.uint64),
                                    np.ascontiguousarray(col, np.uint32))

    def bfs(self, source, out):
        self.R.ref_graph_bfs(self.h, int(source), out)

    def sssp(self, source, out):
        self.R.ref_graph_sssp(self.h, int(source), out)

    def close(self):
        if self.h:
            self.R.ref_graph_destroy(self.h)
            self.h = None
