/*
 * ref_wrap.cu -- C entry points over the reference's OWN host code, compiled
 * from its sources where they lie (see oracle/Makefile, target _ref).
 *
 * TEST INFRASTRUCTURE ONLY: used to pin the CPU oracle (sgs_oracle.c) and as
 * the "reference" CPU baseline.  The product library never links it.
 *
 * Wrapped reference code (paths relative to the reference project):
 *   samples/hybrid_sssp/hybrid_sssp_host.cu:35-63   SSSPHostNaive
 *   samples/hybrid_bfs/hybrid_bfs_host.cpp:33-60    BFSHost
 *   samples/hybrid_pr/hybrid_pr_host.cu:43-124      PageRankHost
 *   include/groute/graphs/csr_graph.cuh:384-811     host::PMAGraph
 *                                                    Bind / insert / del_edge
 * Each reference source is compiled as its own object (they define different
 * IDENTITY_ELEMENT macros); this file only declares what it calls.
 */
#include <cstdint>
#include <cstring>
#include <vector>
#include <groute/graphs/csr_graph.cuh>

typedef uint32_t ref_dist_t;
std::vector<ref_dist_t> SSSPHostNaive(const groute::graphs::host::CSRGraph &g,
                                      index_t source_node);
std::vector<uint32_t> BFSHost(const groute::graphs::host::CSRGraph &g,
                              index_t source_node);
std::vector<float> PageRankHost(const groute::graphs::host::CSRGraph &g);

/* Flags the wrapped sources declare but do not define. */
double FLAGS_error = 0.000001;
bool FLAGS_verbose = false;

static void fill_csr(groute::graphs::host::CSRGraph &g, uint32_t nv,
                     const uint64_t *row, const uint32_t *col) {
  for (uint32_t v = 0; v <= nv; ++v) g.row_start[v] = row[v];
  for (uint64_t e = 0; e < row[nv]; ++e) g.edge_dst[e] = col[e];
}

extern "C" {

void ref_sssp_host(uint32_t nv, const uint64_t *row, const uint32_t *col,
                   uint32_t source, uint32_t *out) {
  groute::graphs::host::CSRGraph g(nv, row[nv]);
  fill_csr(g, nv, row, col);
  std::vector<ref_dist_t> d = SSSPHostNaive(g, source);
  std::memcpy(out, d.data(), sizeof(uint32_t) * nv);
}

void ref_bfs_host(uint32_t nv, const uint64_t *row, const uint32_t *col,
                  uint32_t source, uint32_t *out) {
  groute::graphs::host::CSRGraph g(nv, row[nv]);
  fill_csr(g, nv, row, col);
  std::vector<uint32_t> d = BFSHost(g, source);
  std::memcpy(out, d.data(), sizeof(uint32_t) * nv);
}

void ref_pr_host(uint32_t nv, const uint64_t *row, const uint32_t *col,
                 double err, float *out) {
  groute::graphs::host::CSRGraph g(nv, row[nv]);
  fill_csr(g, nv, row, col);
  FLAGS_error = err;
  std::vector<float> r = PageRankHost(g);
  std::memcpy(out, r.data(), sizeof(float) * nv);
}

/* A graph built once and reused by many timed oracle calls. */
void *ref_graph_create(uint32_t nv, const uint64_t *row, const uint32_t *col) {
  auto *g = new groute::graphs::host::CSRGraph(nv, row[nv]);
  fill_csr(*g, nv, row, col);
  return g;
}
void ref_graph_destroy(void *h) { delete (groute::graphs::host::CSRGraph *)h; }
void ref_graph_bfs(void *h, uint32_t source, uint32_t *out) {
  auto &g = *(groute::graphs::host::CSRGraph *)h;
  std::vector<uint32_t> d = BFSHost(g, source);
  std::memcpy(out, d.data(), sizeof(uint32_t) * g.nnodes);
}
void ref_graph_sssp(void *h, uint32_t source, uint32_t *out) {
  auto &g = *(groute::graphs::host::CSRGraph *)h;
  std::vector<ref_dist_t> d = SSSPHostNaive(g, source);
  std::memcpy(out, d.data(), sizeof(uint32_t) * g.nnodes);
}

/* The PMA is bound the way traversal.h:165-170 does (row/col of the input
 * graph, no weights), then updated with the reference's own insert/del_edge. */
struct ref_pma {
  std::vector<uint64_t> row;
  std::vector<uint32_t> col;
  groute::graphs::host::PMAGraph pma;
};

void *ref_pma_create(uint32_t nv, const uint64_t *row, const uint32_t *col) {
  ref_pma *p = new ref_pma();
  p->row.assign(row, row + nv + 1);
  p->col.assign(col, col + row[nv]);
  p->pma.Bind(nv, row[nv], p->row.data(), p->col.data(), nullptr, nullptr);
  return p;
}

void ref_pma_insert(void *h, uint32_t u, uint32_t v) {
  ref_pma *p = (ref_pma *)h;
  p->pma.insert(u, v, (u + v) % 128 + 1);
}

void ref_pma_del(void *h, uint32_t u, uint32_t v) {
  ref_pma *p = (ref_pma *)h;
  p->pma.del_edge(u, v, (u + v) % 128 + 1);
}

/* One snapshot through the reference's host PMA, in the reference's order
 * within a snapshot (framework.cuh:1011-1012): every insert, then every
 * delete, each through its own insert / del_edge call. */
void ref_pma_apply(void *h, uint64_t ni, const uint32_t *iu, const uint32_t *iv,
                   uint64_t nd, const uint32_t *du, const uint32_t *dv) {
  ref_pma *p = (ref_pma *)h;
  for (uint64_t i = 0; i < ni; ++i) p->pma.insert(iu[i], iv[i], (iu[i] + iv[i]) % 128 + 1);
  for (uint64_t i = 0; i < nd; ++i) p->pma.del_edge(du[i], dv[i], (du[i] + dv[i]) % 128 + 1);
}

/* Writes each vertex's live list edges_[index, index+degree) as a CSR.
 * Returns the edge count, or UINT64_MAX when cap is too small. */
uint64_t ref_pma_export(void *h, uint64_t *row_out, uint32_t *col_out,
                        uint64_t cap) {
  ref_pma *p = (ref_pma *)h;
  auto &g = p->pma;
  uint64_t m = 0;
  for (uint32_t v = 0; v < g.nnodes; ++v) {
    row_out[v] = m;
    uint64_t b = g.sync_vertices_[v].index;
    uint32_t d = g.sync_vertices_[v].degree;
    if (m + d > cap) return UINT64_MAX;
    for (uint32_t i = 0; i < d; ++i) col_out[m++] = g.edges_[b + i];
  }
  row_out[g.nnodes] = m;
  return m;
}

void ref_pma_destroy(void *h) { delete (ref_pma *)h; }

} /* extern "C" */
