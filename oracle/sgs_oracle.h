/*
 * sgs_oracle.h -- CPU oracle for the incremental streaming-graph engine.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, the smoke check and bench.py's CPU-baseline
 * leg use it, and only as the checker / the timed CPU reference path.
 *
 * It restates, in plain C, the semantics of the reference
 * (Yongze-zzz/C-GpuStreamGraph) for the hot path:
 *   - graph input: edge list read in file order and bucketed per source
 *     (src/utils/parser.cpp:296-406, ReadGraphMarket_bigdata);
 *   - snapshot update semantics of the PMA dynamic graph: inserts are appended
 *     to the source's list without a duplicate check, then deletes remove the
 *     matching (src,dst) entries (framework.cuh:1001-1023 add_edge_pr then
 *     del_edge_pr; include/groute/graphs/csr_graph.cuh:658-811 insert/del_edge);
 *   - from-scratch ground truth per snapshot for BFS depth, SSSP distance,
 *     directed min-label CC and PageRank (samples/hybrid_{bfs,sssp,cc,pr});
 *   - the reference's serial host oracles, restated for CPU timing
 *     (samples/hybrid_sssp/hybrid_sssp_host.cu:35-63 SSSPHostNaive,
 *      samples/hybrid_bfs/hybrid_bfs_host.cpp:33-60 BFSHost,
 *      samples/hybrid_pr/hybrid_pr_host.cu:43-124 PageRankHost).
 * Plus the synthetic-input generators (R-MAT, seeded weights, update streams)
 * whose integer arithmetic is shared bit-for-bit with the device generator.
 */
#ifndef SGS_ORACLE_H
#define SGS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGSO_INF 0xFFFFFFFFu

/* ---- hashing / generators ------------------------------------------- */
uint64_t sgso_mix64(uint64_t x);
/* R-MAT edge k of the stream: thresholds are floor(p * 2^53) of the cumulative
 * quadrant probabilities a, a+b, a+b+c. */
void sgso_rmat_edge(uint32_t scale, uint64_t seed, uint64_t k, uint64_t tA,
                    uint64_t tAB, uint64_t tABC, uint32_t *u, uint32_t *v);
void sgso_rmat_raw(uint32_t scale, uint64_t ne, uint64_t seed, uint64_t tA,
                   uint64_t tAB, uint64_t tABC, uint32_t *src, uint32_t *dst);
/* Sort edges by (src,dst), optionally drop self loops and duplicates, and
 * write a CSR.  Returns the number of edges written. */
uint64_t sgso_build_csr(uint32_t nv, uint64_t ne, const uint32_t *src,
                        const uint32_t *dst, int dedupe, int drop_self,
                        uint64_t *row, uint32_t *col);
/* Same graph as sgso_rmat_raw + sgso_build_csr(dedupe, drop_self), built
 * with OpenMP threads (for scale 20+ inputs of the CPU baselines).  col must
 * hold edge_factor << scale entries.  Returns the edge count. */
uint64_t sgso_rmat_csr_par(uint32_t scale, uint32_t edge_factor, uint64_t seed,
                           uint64_t tA, uint64_t tAB, uint64_t tABC,
                           uint64_t *row, uint32_t *col);
/* CSR in input (file) order: counting sort by source, stable. */
void sgso_csr_file_order(uint32_t nv, uint64_t ne, const uint32_t *src,
                         const uint32_t *dst, const uint32_t *w, uint64_t *row,
                         uint32_t *col, uint32_t *wout);
uint32_t sgso_weight_of(uint64_t wseed, uint32_t u, uint32_t v);
void sgso_weights_pairs(uint64_t wseed, uint64_t n, const uint32_t *u,
                        const uint32_t *v, uint32_t *w);
uint32_t sgso_weight_synth(uint32_t u, uint32_t v);
void sgso_weights(uint32_t nv, const uint64_t *row, const uint32_t *col,
                  uint64_t wseed, int mode, uint32_t *w);
/* Update stream: n_del distinct existing edges sampled uniformly (by edge
 * index) and n_ins distinct non-edges (u != v) sampled uniformly over vertex
 * pairs, both from the initial graph (rows sorted).  Returns 0 or -1. */
int sgso_gen_updates(uint32_t nv, const uint64_t *row, const uint32_t *col,
                     uint64_t seed, uint64_t n_ins, uint64_t n_del,
                     uint32_t *ins_src, uint32_t *ins_dst, uint32_t *del_src,
                     uint32_t *del_dst);

/* ---- snapshot apply (reference PMA semantics on an edge multiset) ---- */
/* New graph = (old ++ inserts) minus every (src,dst) that appears in the
 * delete list.  Per-vertex order: surviving old entries, then inserts in batch
 * order.  row_out has nv+1 entries; col_out/w_out must hold cap_out entries.
 * Returns the new edge count, or UINT64_MAX if cap_out is too small. */
uint64_t sgso_apply(uint32_t nv, const uint64_t *row, const uint32_t *col,
                    const uint32_t *w, uint64_t n_ins, const uint32_t *ins_src,
                    const uint32_t *ins_dst, const uint32_t *ins_w,
                    uint64_t n_del, const uint32_t *del_src,
                    const uint32_t *del_dst, uint64_t *row_out,
                    uint32_t *col_out, uint32_t *w_out, uint64_t cap_out);

/* Same, but reproducing the reference's del_edge exactly, including its
 * index slip: after removing a match it does not re-examine the slot it just
 * shifted into, so in a run of k adjacent copies one call removes ceil(k/2)
 * (csr_graph.cuh:795-805).  Deletes are applied one call per listed delete,
 * in batch order.  Used only to pin the oracle against the reference. */
uint64_t sgso_apply_refexact(uint32_t nv, const uint64_t *row,
                             const uint32_t *col, uint64_t n_ins,
                             const uint32_t *ins_src, const uint32_t *ins_dst,
                             uint64_t n_del, const uint32_t *del_src,
                             const uint32_t *del_dst, uint64_t *row_out,
                             uint32_t *col_out, uint64_t cap_out);

/* ---- ground truth (from scratch) ------------------------------------- */
/* depth / dist: SGSO_INF when unreached.  parent: the smallest-id tight
 * predecessor (dist[p] + w(p,v) == dist[v]); SGSO_INF for the source and
 * unreached vertices.  Path lengths >= 2^32-1 count as unreachable. */
uint64_t sgso_bfs(uint32_t nv, const uint64_t *row, const uint32_t *col,
                  uint32_t source, uint32_t *depth, uint32_t *parent);
uint64_t sgso_sssp(uint32_t nv, const uint64_t *row, const uint32_t *col,
                   const uint32_t *w, uint32_t source, uint32_t *dist,
                   uint32_t *parent);
/* label(v) = min id over all vertices that reach v along out-edges
 * (v reaches itself). */
/* widest (maximum-bottleneck) path from source; 0 = unreachable */
uint64_t sgso_widest(uint32_t nv, const uint64_t *row, const uint32_t *col,
                     const uint32_t *w, uint32_t source, uint32_t *width);
uint64_t sgso_cc(uint32_t nv, const uint64_t *row, const uint32_t *col,
                 uint32_t *label);
/* FP64 power iteration of x = (1-alpha) + alpha * A^T D^-1 x (dangling mass
 * dropped).  Stops when the L1 change < tol.  Returns iterations. */
int sgso_pagerank(uint32_t nv, const uint64_t *row, const uint32_t *col,
                  double alpha, double tol, int max_iter, double *x);

/* ---- restated reference host oracles (timed CPU path) ---------------- */
/* FIFO Bellman-Ford of SSSPHostNaive, with the weight array given
 * (w == NULL: the reference's synthesized (u+v)%128).  Returns relaxed
 * edges (traversed edge count). */
uint64_t sgso_sssp_fifo(uint32_t nv, const uint64_t *row, const uint32_t *col,
                        const uint32_t *w, uint32_t source, uint32_t *dist);
uint64_t sgso_bfs_fifo(uint32_t nv, const uint64_t *row, const uint32_t *col,
                       uint32_t source, uint32_t *depth);
/* FIFO residual-push PageRank in float (PageRankHost). */
uint64_t sgso_pr_host_float(uint32_t nv, const uint64_t *row,
                            const uint32_t *col, double alpha, double err,
                            float *ranks);
/* Edge-budgeted variants for bounded CPU timing: stop after max_edges edge
 * relaxations; return edges actually relaxed. */
uint64_t sgso_sssp_fifo_budget(uint32_t nv, const uint64_t *row,
                               const uint32_t *col, const uint32_t *w,
                               uint32_t source, uint32_t *dist,
                               uint64_t max_edges);
uint64_t sgso_bfs_fifo_budget(uint32_t nv, const uint64_t *row,
                              const uint32_t *col, uint32_t source,
                              uint32_t *depth, uint64_t max_edges);

/* ---- checks ----------------------------------------------------------- */
/* Verifies a (value,parent) pair against a graph for SSSP/BFS (w==NULL means
 * unit weights): every edge satisfies value[v] <= value[u]+w, and every
 * reached non-source vertex has parent p with an edge p->v that is tight.
 * Returns the number of violations. */
uint64_t sgso_check_tree(uint32_t nv, const uint64_t *row, const uint32_t *col,
                         const uint32_t *w, uint32_t source,
                         const uint32_t *value, const uint32_t *parent);
/* CC parents: label[parent[v]] == label[v], edge parent[v]->v exists, roots
 * (label[v]==v) have parent SGSO_INF, and parent chains are acyclic. */
uint64_t sgso_check_cc_parent(uint32_t nv, const uint64_t *row,
                              const uint32_t *col, const uint32_t *label,
                              const uint32_t *parent);

#ifdef __cplusplus
}
#endif
#endif
