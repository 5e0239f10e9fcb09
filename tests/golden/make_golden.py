"""Generates the golden fixtures in this folder from the REFERENCE's own code.

Run here, where the reference tree is available:

    make -C oracle ref          # builds oracle/_ref/libsgsref.so from the
                                # reference sources (SSSPHostNaive, BFSHost,
                                # PageRankHost, host::PMAGraph)
    python tests/golden/make_golden.py

Each fixture is an .npz with the inputs (a small graph and, for the PMA case,
an update batch) and the outputs of the reference's code on them.  The CPU
oracle is pinned against these files by tests/test_oracle.py, which also runs
where the reference tree is absent.

Graphs are small seeded R-MAT graphs from the oracle's generator (the
generator itself is pinned separately against the device generator) and the
5-vertex example of the reference README (README.md:68-96).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import oracle as O  # noqa: E402

# README.md:68-75 (graph), :78-89 (updates), :93-96 (stream sizes "2 3" x2)
README_EDGES = [(0, 1), (0, 2), (1, 2), (1, 3), (2, 4), (3, 4)]
README_ADDS = [(0, 3), (0, 4), (1, 4), (2, 3)]
README_DELS = [(0, 1), (0, 2), (1, 2), (1, 3), (2, 4), (3, 4)]
README_SIZES = [(2, 3), (2, 3)]


def graph_cases():
    src = np.array([e[0] for e in README_EDGES], np.uint32)
    dst = np.array([e[1] for e in README_EDGES], np.uint32)
    row, col, _ = O.csr_file_order(5, src, dst)
    yield "readme", 5, row, col
    for scale, seed in [(8, 1), (10, 2), (12, 3)]:
        nv, row, col = O.rmat_csr(scale, 16, seed)
        yield f"rmat{scale}_s{seed}", nv, row, col


def main():
    R = O.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libsgsref.so not built: run `make -C oracle ref`")
    for name, nv, row, col in graph_cases():
        out = dict(nv=np.uint32(nv), row=row, col=col)
        for s in sorted({0, nv // 3, nv - 1}):
            out[f"sssp_{s}"] = O.ref_sssp_host(nv, row, col, s)
            out[f"bfs_{s}"] = O.ref_bfs_host(nv, row, col, s)
        out["pr"] = O.ref_pr_host(nv, row, col, 1e-6)
        np.savez_compressed(os.path.join(HERE, f"ref_algos_{name}.npz"), **out)
        print("wrote", name)
    # PMA snapshots: reference insert/del_edge applied per snapshot
    cases = []
    src = np.array([e[0] for e in README_EDGES], np.uint32)
    dst = np.array([e[1] for e in README_EDGES], np.uint32)
    row, col, _ = O.csr_file_order(5, src, dst)
    adds = np.array(README_ADDS, np.uint32)
    dels = np.array(README_DELS, np.uint32)
    batches, ia, idl = [], 0, 0
    for na, nd in README_SIZES:
        batches.append((adds[ia:ia + na], dels[idl:idl + nd]))
        ia += na
        idl += nd
    cases.append(("readme", 5, row, col, batches))
    rng = np.random.default_rng(7)
    for scale, seed in [(8, 4), (10, 5)]:
        nv, row, col = O.rmat_csr(scale, 16, seed)
        bl = []
        for k in range(3):
            i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, seed * 1000003 + k, 64, 64)
            # messy extras: duplicate inserts, insert+delete of one edge,
            # delete of a non-edge, self loop insert
            extra_i = np.array([[i_s[0], i_d[0]], [3, 3], [int(col[0]) % nv, 1]], np.uint32)
            extra_d = np.array([[i_s[1], i_d[1]], [nv - 1, nv - 2]], np.uint32)
            ins = np.concatenate([np.stack([i_s, i_d], 1), extra_i, np.stack([i_s[1:2], i_d[1:2]], 1)])
            de = np.concatenate([np.stack([d_s, d_d], 1), extra_d])
            rng.shuffle(ins)
            bl.append((ins.astype(np.uint32), de.astype(np.uint32)))
        cases.append((f"rmat{scale}_s{seed}", nv, row, col, bl))
    for name, nv, row, col, bl in cases:
        pma = O.RefPMA(nv, row, col)
        out = dict(nv=np.uint32(nv), row=row, col=col, nsnap=np.uint32(len(bl)))
        for k, (ins, de) in enumerate(bl):
            for u, v in ins:
                pma.insert(u, v)
            for u, v in de:
                pma.delete(u, v)
            r, c = pma.export()
            out[f"ins_{k}"] = ins
            out[f"del_{k}"] = de
            out[f"row_{k}"] = r
            out[f"col_{k}"] = c
        pma.close()
        np.savez_compressed(os.path.join(HERE, f"ref_pma_{name}.npz"), **out)
        print("wrote pma", name)


if __name__ == "__main__":
    main()
