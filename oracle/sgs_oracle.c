/*
 * sgs_oracle.c -- CPU oracle (test infrastructure only; see sgs_oracle.h).
 *
 * Plain C, single-threaded.  Every function cites the reference behaviour it
 * restates.  The generator arithmetic (splitmix64 finalizer, 53-bit R-MAT
 * thresholds, multiply-high range reduction) is integer-only so that the
 * device generator in the product library reproduces it bit for bit.
 */
#include "sgs_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define GAMMA 0x9E3779B97F4A7C15ull

/* splitmix64 output function (Steele, Lea, Flood 2014; constants as published
 * by Vigna in splitmix64.c). */
static inline uint64_t fin64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t sgso_mix64(uint64_t x) { return fin64(x + GAMMA); }
/* i-th output of a splitmix64 stream whose state starts at key. */
static inline uint64_t stream_at(uint64_t key, uint64_t i) {
  return fin64(key + (i + 1) * GAMMA);
}
static inline uint64_t mulhi64(uint64_t a, uint64_t b) {
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
}

/* ---------------------------------------------------------------------- */
/* R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): each of `scale` levels
 * picks a quadrant with probabilities a,b,c,d; bit MSB first.  The reference
 * ships a GAP-style generator (include/framework/generator.h:82-116) that is
 * never compiled; this restates the published definition without the id
 * permutation. */
void sgso_rmat_edge(uint32_t scale, uint64_t seed, uint64_t k, uint64_t tA,
                    uint64_t tAB, uint64_t tABC, uint32_t *u, uint32_t *v) {
  uint64_t key = sgso_mix64(seed ^ 0x524D4154ull /* "RMAT" */);
  uint32_t uu = 0, vv = 0;
  for (uint32_t l = 0; l < scale; ++l) {
    uint64_t r = stream_at(key, k * 64u + l) >> 11;
    uint32_t bu, bv;
    if (r < tA) { bu = 0; bv = 0; }
    else if (r < tAB) { bu = 0; bv = 1; }
    else if (r < tABC) { bu = 1; bv = 0; }
    else { bu = 1; bv = 1; }
    uu = (uu << 1) | bu;
    vv = (vv << 1) | bv;
  }
  *u = uu;
  *v = vv;
}

void sgso_rmat_raw(uint32_t scale, uint64_t ne, uint64_t seed, uint64_t tA,
                   uint64_t tAB, uint64_t tABC, uint32_t *src, uint32_t *dst) {
  for (uint64_t k = 0; k < ne; ++k)
    sgso_rmat_edge(scale, seed, k, tA, tAB, tABC, &src[k], &dst[k]);
}

/* LSD radix sort of 64-bit keys, 16-bit digits. */
static void radix_sort_u64(uint64_t *a, uint64_t n) {
  if (n < 2) return;
  uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
  uint64_t *cnt = (uint64_t *)malloc(65536 * sizeof(uint64_t));
  uint64_t *from = a, *to = tmp;
  for (int pass = 0; pass < 4; ++pass) {
    int sh = pass * 16;
    memset(cnt, 0, 65536 * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) cnt[(from[i] >> sh) & 0xFFFF]++;
    uint64_t s = 0;
    for (int d = 0; d < 65536; ++d) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
    for (uint64_t i = 0; i < n; ++i) to[cnt[(from[i] >> sh) & 0xFFFF]++] = from[i];
    uint64_t *t = from; from = to; to = t;
  }
  /* 4 passes: result is back in a */
  free(tmp);
  free(cnt);
}

uint64_t sgso_build_csr(uint32_t nv, uint64_t ne, const uint32_t *src,
                        const uint32_t *dst, int dedupe, int drop_self,
                        uint64_t *row, uint32_t *col) {
  uint64_t *keys = (uint64_t *)malloc((ne ? ne : 1) * sizeof(uint64_t));
  uint64_t m = 0;
  for (uint64_t i = 0; i < ne; ++i) {
    if (drop_self && src[i] == dst[i]) continue;
    keys[m++] = ((uint64_t)src[i] << 32) | dst[i];
  }
  radix_sort_u64(keys, m);
  uint64_t k = 0;
  for (uint64_t i = 0; i < m; ++i) {
    if (dedupe && i > 0 && keys[i] == keys[i - 1]) continue;
    keys[k++] = keys[i];
  }
  memset(row, 0, ((uint64_t)nv + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < k; ++i) row[(keys[i] >> 32) + 1]++;
  for (uint32_t v = 0; v < nv; ++v) row[v + 1] += row[v];
  for (uint64_t i = 0; i < k; ++i) col[i] = (uint32_t)keys[i];
  free(keys);
  return k;
}

static int cmp_u32(const void *a, const void *b) {
  uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : x > y;
}
static void sort_u32(uint32_t *a, uint64_t n) {
  if (n < 32) {
    for (uint64_t i = 1; i < n; ++i) {
      uint32_t x = a[i];
      uint64_t j = i;
      while (j > 0 && a[j - 1] > x) { a[j] = a[j - 1]; --j; }
      a[j] = x;
    }
  } else {
    qsort(a, n, sizeof(uint32_t), cmp_u32);
  }
}

/* Minimal parallel-for over [0,n) with pthreads, static contiguous blocks. */
typedef struct {
  void (*fn)(void *, uint64_t, uint64_t);
  void *arg;
  uint64_t lo, hi;
} pf_task;
static void *pf_run(void *p) {
  pf_task *t = (pf_task *)p;
  t->fn(t->arg, t->lo, t->hi);
  return NULL;
}
static void parallel_for(uint64_t n, void (*fn)(void *, uint64_t, uint64_t), void *arg) {
  long nt = sysconf(_SC_NPROCESSORS_ONLN);
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  pthread_t th[64];
  pf_task tk[64];
  for (long i = 0; i < nt; ++i) {
    tk[i].fn = fn;
    tk[i].arg = arg;
    tk[i].lo = n * i / nt;
    tk[i].hi = n * (i + 1) / nt;
    pthread_create(&th[i], NULL, pf_run, &tk[i]);
  }
  for (long i = 0; i < nt; ++i) pthread_join(th[i], NULL);
}

typedef struct {
  uint32_t scale;
  uint64_t seed, tA, tAB, tABC;
  uint64_t *cnt, *fill;
  uint32_t *col;
} rmat_par;

static void rmat_count(void *p, uint64_t lo, uint64_t hi) {
  rmat_par *a = (rmat_par *)p;
  for (uint64_t k = lo; k < hi; ++k) {
    uint32_t u, v;
    sgso_rmat_edge(a->scale, a->seed, k, a->tA, a->tAB, a->tABC, &u, &v);
    if (u != v) __atomic_fetch_add(&a->cnt[u + 1], 1, __ATOMIC_RELAXED);
  }
}
static void rmat_scatter(void *p, uint64_t lo, uint64_t hi) {
  rmat_par *a = (rmat_par *)p;
  for (uint64_t k = lo; k < hi; ++k) {
    uint32_t u, v;
    sgso_rmat_edge(a->scale, a->seed, k, a->tA, a->tAB, a->tABC, &u, &v);
    if (u != v) a->col[__atomic_fetch_add(&a->fill[u], 1, __ATOMIC_RELAXED)] = v;
  }
}
static void rmat_rows(void *p, uint64_t lo, uint64_t hi) {
  rmat_par *a = (rmat_par *)p;
  for (uint64_t u = lo; u < hi; ++u) {
    uint32_t *x = a->col + a->cnt[u];
    uint64_t n = a->cnt[u + 1] - a->cnt[u], m = 0;
    sort_u32(x, n);
    for (uint64_t i = 0; i < n; ++i)
      if (i == 0 || x[i] != x[i - 1]) x[m++] = x[i];
    a->fill[u] = m;
  }
}

uint64_t sgso_rmat_csr_par(uint32_t scale, uint32_t edge_factor, uint64_t seed,
                           uint64_t tA, uint64_t tAB, uint64_t tABC,
                           uint64_t *row, uint32_t *col) {
  const uint64_t nv = 1ull << scale, ne = nv * edge_factor;
  rmat_par a;
  a.scale = scale; a.seed = seed; a.tA = tA; a.tAB = tAB; a.tABC = tABC;
  a.cnt = (uint64_t *)calloc(nv + 1, sizeof(uint64_t));
  a.fill = (uint64_t *)malloc(nv * sizeof(uint64_t));
  a.col = col;
  parallel_for(ne, rmat_count, &a);      /* out-degrees, self loops dropped */
  for (uint64_t v = 0; v < nv; ++v) a.cnt[v + 1] += a.cnt[v];
  memcpy(a.fill, a.cnt, nv * sizeof(uint64_t));
  parallel_for(ne, rmat_scatter, &a);    /* destinations into buckets */
  parallel_for(nv, rmat_rows, &a);       /* sort + unique each bucket */
  row[0] = 0;
  for (uint64_t u = 0; u < nv; ++u) row[u + 1] = row[u] + a.fill[u];
  /* compact left to right: a row's target never passes its source */
  for (uint64_t u = 0; u < nv; ++u)
    if (row[u] != a.cnt[u]) memmove(col + row[u], col + a.cnt[u], a.fill[u] * sizeof(uint32_t));
  uint64_t m = row[nv];
  free(a.cnt);
  free(a.fill);
  return m;
}

/* parser.cpp:296-406: two passes over the file; per-source lists keep file
 * order; no dedupe, no self-loop removal. */
void sgso_csr_file_order(uint32_t nv, uint64_t ne, const uint32_t *src,
                         const uint32_t *dst, const uint32_t *w, uint64_t *row,
                         uint32_t *col, uint32_t *wout) {
  memset(row, 0, ((uint64_t)nv + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < ne; ++i) row[src[i] + 1]++;
  for (uint32_t v = 0; v < nv; ++v) row[v + 1] += row[v];
  uint64_t *fill = (uint64_t *)malloc(((uint64_t)nv + 1) * sizeof(uint64_t));
  memcpy(fill, row, ((uint64_t)nv + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < ne; ++i) {
    uint64_t p = fill[src[i]]++;
    col[p] = dst[i];
    if (w && wout) wout[p] = w[i];
  }
  free(fill);
}

uint32_t sgso_weight_of(uint64_t wseed, uint32_t u, uint32_t v) {
  uint64_t key = sgso_mix64(wseed ^ 0x57454947ull /* "WEIG" */);
  uint64_t h = fin64(key ^ (((uint64_t)u << 32) | v));
  return 1u + (uint32_t)(h >> 58); /* uniform in [1,64] */
}

/* The same seeded weight for each pair (u[i], v[i]) of an edge list (the
 * weights of an update batch's inserts). */
void sgso_weights_pairs(uint64_t wseed, uint64_t n, const uint32_t *u,
                        const uint32_t *v, uint32_t *w) {
  for (uint64_t i = 0; i < n; ++i) w[i] = sgso_weight_of(wseed, u[i], v[i]);
}

/* push_functor.h:306 -- the reference synthesizes (src+dst)%128+1 per edge. */
uint32_t sgso_weight_synth(uint32_t u, uint32_t v) { return (u + v) % 128u + 1u; }

void sgso_weights(uint32_t nv, const uint64_t *row, const uint32_t *col,
                  uint64_t wseed, int mode, uint32_t *w) {
  for (uint32_t u = 0; u < nv; ++u)
    for (uint64_t e = row[u]; e < row[u + 1]; ++e)
      w[e] = mode == 1 ? sgso_weight_synth(u, col[e])
             : mode == 2 ? 1u
                         : sgso_weight_of(wseed, u, col[e]);
}

static int has_edge_sorted(const uint64_t *row, const uint32_t *col, uint32_t u,
                           uint32_t v) {
  uint64_t lo = row[u], hi = row[u + 1];
  while (lo < hi) {
    uint64_t mid = lo + (hi - lo) / 2;
    if (col[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo < row[u + 1] && col[lo] == v;
}

int sgso_gen_updates(uint32_t nv, const uint64_t *row, const uint32_t *col,
                     uint64_t seed, uint64_t n_ins, uint64_t n_del,
                     uint32_t *ins_src, uint32_t *ins_dst, uint32_t *del_src,
                     uint32_t *del_dst) {
  uint64_t ne = row[nv];
  if (n_del > ne) return -1;
  /* deletes: distinct edge indices, uniform */
  if (n_del) {
    uint64_t *bits = (uint64_t *)calloc(ne / 64 + 1, sizeof(uint64_t));
    uint64_t key = sgso_mix64(seed ^ 0x44454C45ull /* "DELE" */);
    uint64_t got = 0, i = 0;
    while (got < n_del) {
      uint64_t idx = mulhi64(stream_at(key, i++), ne);
      if (bits[idx >> 6] >> (idx & 63) & 1) continue;
      bits[idx >> 6] |= 1ull << (idx & 63);
      uint32_t lo = 0, hi = nv; /* last u with row[u] <= idx */
      while (hi - lo > 1) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (row[mid] <= idx) lo = mid;
        else hi = mid;
      }
      del_src[got] = lo;
      del_dst[got] = col[idx];
      ++got;
    }
    free(bits);
  }
  if (n_ins) {
    if (nv < 2) return -1;
    uint64_t tsz = 1;
    while (tsz < 2 * n_ins + 16) tsz <<= 1;
    uint64_t *tab = (uint64_t *)malloc(tsz * sizeof(uint64_t));
    memset(tab, 0xFF, tsz * sizeof(uint64_t));
    uint64_t key = sgso_mix64(seed ^ 0x494E5345ull /* "INSE" */);
    uint64_t got = 0, i = 0, limit = 64 * n_ins + 1000000;
    while (got < n_ins) {
      if (i > limit) { free(tab); return -1; }
      uint64_t h = stream_at(key, i++);
      uint32_t u = (uint32_t)(((h >> 32) * (uint64_t)nv) >> 32);
      uint32_t v = (uint32_t)(((h & 0xFFFFFFFFull) * (uint64_t)nv) >> 32);
      if (u == v) continue;
      if (has_edge_sorted(row, col, u, v)) continue;
      uint64_t k = ((uint64_t)u << 32) | v;
      uint64_t s = sgso_mix64(k) & (tsz - 1);
      int dup = 0;
      while (tab[s] != ~0ull) {
        if (tab[s] == k) { dup = 1; break; }
        s = (s + 1) & (tsz - 1);
      }
      if (dup) continue;
      tab[s] = k;
      ins_src[got] = u;
      ins_dst[got] = v;
      ++got;
    }
    free(tab);
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : x > y;
}
static int in_sorted(const uint64_t *a, uint64_t n, uint64_t k) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t mid = lo + (hi - lo) / 2;
    if (a[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  return lo < n && a[lo] == k;
}

/* framework.cuh:1001-1023 applies a snapshot as: every insert via
 * PMAGraph::insert (csr_graph.cuh:658-786, appended at index+degree, no
 * duplicate check), then every delete via PMAGraph::del_edge
 * (csr_graph.cuh:789-811, removes matching entries of src's list). */
uint64_t sgso_apply(uint32_t nv, const uint64_t *row, const uint32_t *col,
                    const uint32_t *w, uint64_t n_ins, const uint32_t *ins_src,
                    const uint32_t *ins_dst, const uint32_t *ins_w,
                    uint64_t n_del, const uint32_t *del_src,
                    const uint32_t *del_dst, uint64_t *row_out,
                    uint32_t *col_out, uint32_t *w_out, uint64_t cap_out) {
  uint64_t *dk = (uint64_t *)malloc((n_del ? n_del : 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < n_del; ++i)
    dk[i] = ((uint64_t)del_src[i] << 32) | del_dst[i];
  qsort(dk, n_del, sizeof(uint64_t), cmp_u64);
  /* inserts bucketed by source, batch order kept */
  uint64_t *ib = (uint64_t *)calloc((uint64_t)nv + 1, sizeof(uint64_t));
  for (uint64_t i = 0; i < n_ins; ++i) ib[ins_src[i] + 1]++;
  for (uint32_t v = 0; v < nv; ++v) ib[v + 1] += ib[v];
  uint64_t *ifill = (uint64_t *)malloc(((uint64_t)nv + 1) * sizeof(uint64_t));
  memcpy(ifill, ib, ((uint64_t)nv + 1) * sizeof(uint64_t));
  uint64_t *iord = (uint64_t *)malloc((n_ins ? n_ins : 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < n_ins; ++i) iord[ifill[ins_src[i]]++] = i;
  /* sources that have deletes: only their lists need the per-edge lookup */
  uint8_t *hasdel = (uint8_t *)calloc((uint64_t)nv + 1, 1);
  for (uint64_t i = 0; i < n_del; ++i) hasdel[del_src[i]] = 1;
  uint64_t m = 0;
  int overflow = 0;
  for (uint32_t u = 0; u < nv; ++u) {
    row_out[u] = m;
    if (!hasdel[u]) {
      uint64_t d = row[u + 1] - row[u];
      if (m + d > cap_out) { overflow = 1; break; }
      memcpy(col_out + m, col + row[u], d * sizeof(uint32_t));
      if (w_out) {
        if (w) memcpy(w_out + m, w + row[u], d * sizeof(uint32_t));
        else for (uint64_t i = 0; i < d; ++i) w_out[m + i] = 1u;
      }
      m += d;
    } else
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      uint64_t k = ((uint64_t)u << 32) | col[e];
      if (n_del && in_sorted(dk, n_del, k)) continue;
      if (m >= cap_out) { overflow = 1; break; }
      col_out[m] = col[e];
      if (w_out) w_out[m] = w ? w[e] : 1u;
      ++m;
    }
    for (uint64_t j = ib[u]; j < ib[u + 1]; ++j) {
      uint64_t i = iord[j];
      uint64_t k = ((uint64_t)u << 32) | ins_dst[i];
      if (n_del && in_sorted(dk, n_del, k)) continue;
      if (m >= cap_out) { overflow = 1; break; }
      col_out[m] = ins_dst[i];
      if (w_out) w_out[m] = ins_w ? ins_w[i] : 1u;
      ++m;
    }
    if (overflow) break;
  }
  row_out[nv] = m;
  free(hasdel);
  free(dk);
  free(ib);
  free(ifill);
  free(iord);
  return overflow ? UINT64_MAX : m;
}

uint64_t sgso_apply_refexact(uint32_t nv, const uint64_t *row,
                             const uint32_t *col, uint64_t n_ins,
                             const uint32_t *ins_src, const uint32_t *ins_dst,
                             uint64_t n_del, const uint32_t *del_src,
                             const uint32_t *del_dst, uint64_t *row_out,
                             uint32_t *col_out, uint64_t cap_out) {
  /* per-vertex arrays with room for every insert */
  uint64_t *cnt = (uint64_t *)calloc((uint64_t)nv + 1, sizeof(uint64_t));
  for (uint64_t i = 0; i < n_ins; ++i) cnt[ins_src[i]]++;
  uint64_t *base = (uint64_t *)malloc(((uint64_t)nv + 1) * sizeof(uint64_t));
  uint32_t *deg = (uint32_t *)malloc(((uint64_t)nv + 1) * sizeof(uint32_t));
  uint64_t tot = 0;
  for (uint32_t v = 0; v < nv; ++v) {
    base[v] = tot;
    deg[v] = (uint32_t)(row[v + 1] - row[v]);
    tot += deg[v] + cnt[v];
  }
  uint32_t *buf = (uint32_t *)malloc((tot ? tot : 1) * sizeof(uint32_t));
  for (uint32_t v = 0; v < nv; ++v)
    for (uint64_t e = row[v]; e < row[v + 1]; ++e) buf[base[v] + (e - row[v])] = col[e];
  /* PMAGraph::insert appends at index+degree (csr_graph.cuh:665) */
  for (uint64_t i = 0; i < n_ins; ++i) {
    uint32_t u = ins_src[i];
    buf[base[u] + deg[u]++] = ins_dst[i];
  }
  /* PMAGraph::del_edge (csr_graph.cuh:789-811), literally */
  for (uint64_t k = 0; k < n_del; ++k) {
    uint32_t u = del_src[k], v = del_dst[k];
    uint32_t *a = buf + base[u];
    uint64_t right = deg[u];
    for (uint64_t i = 0; i < right; ++i) {
      if (a[i] == v) {
        for (uint64_t j = i + 1; j < right; ++j) a[j - 1] = a[j];
        deg[u] -= 1;
        a[right - 1] = 0xFFFFFFFFu;
      }
    }
  }
  uint64_t m = 0;
  int overflow = 0;
  for (uint32_t v = 0; v < nv && !overflow; ++v) {
    row_out[v] = m;
    for (uint32_t i = 0; i < deg[v]; ++i) {
      if (m >= cap_out) { overflow = 1; break; }
      col_out[m++] = buf[base[v] + i];
    }
  }
  row_out[nv] = m;
  free(cnt); free(base); free(deg); free(buf);
  return overflow ? UINT64_MAX : m;
}

/* ---------------------------------------------------------------------- */
static void tight_parents(uint32_t nv, const uint64_t *row, const uint32_t *col,
                          const uint32_t *w, const uint32_t *val,
                          uint32_t *parent) {
  for (uint32_t v = 0; v < nv; ++v) parent[v] = SGSO_INF;
  for (uint32_t u = 0; u < nv; ++u) {
    if (val[u] == SGSO_INF) continue;
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      uint32_t v = col[e];
      uint64_t nd = (uint64_t)val[u] + (w ? w[e] : 1u);
      if (nd == val[v] && u < parent[v]) parent[v] = u;
    }
  }
}

/* hybrid_bfs_host.cpp:33-60 (BFSHost) computes depths by FIFO BFS. */
uint64_t sgso_bfs(uint32_t nv, const uint64_t *row, const uint32_t *col,
                  uint32_t source, uint32_t *depth, uint32_t *parent) {
  for (uint32_t v = 0; v < nv; ++v) depth[v] = SGSO_INF;
  uint64_t edges = 0;
  if (source < nv) {
    uint32_t *q = (uint32_t *)malloc((uint64_t)nv * sizeof(uint32_t));
    uint64_t h = 0, t = 0;
    depth[source] = 0;
    q[t++] = source;
    while (h < t) {
      uint32_t u = q[h++];
      for (uint64_t e = row[u]; e < row[u + 1]; ++e, ++edges) {
        uint32_t v = col[e];
        if (depth[v] == SGSO_INF) { depth[v] = depth[u] + 1; q[t++] = v; }
      }
    }
    free(q);
  }
  if (parent) tight_parents(nv, row, col, NULL, depth, parent);
  return edges;
}

/* binary min-heap of (dist<<32 | vertex) */
typedef struct { uint64_t *a; uint64_t n, cap; } heap_t;
static void hpush(heap_t *h, uint64_t x) {
  if (h->n == h->cap) {
    h->cap = h->cap ? 2 * h->cap : 1024;
    h->a = (uint64_t *)realloc(h->a, h->cap * sizeof(uint64_t));
  }
  uint64_t i = h->n++;
  while (i > 0) {
    uint64_t p = (i - 1) / 2;
    if (h->a[p] <= x) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i] = x;
}
static uint64_t hpop(heap_t *h) {
  uint64_t top = h->a[0], x = h->a[--h->n];
  uint64_t i = 0;
  for (;;) {
    uint64_t c = 2 * i + 1;
    if (c >= h->n) break;
    if (c + 1 < h->n && h->a[c + 1] < h->a[c]) ++c;
    if (x <= h->a[c]) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n) h->a[i] = x;
  return top;
}

/* Ground truth for hybrid_sssp (hybrid_sssp.cu:97-118 relaxes
 * buffer[dst] = min(buffer[dst], buffer[src] + w)); Dijkstra with 64-bit
 * path sums, dist >= 2^32-1 treated as unreachable. */
uint64_t sgso_sssp(uint32_t nv, const uint64_t *row, const uint32_t *col,
                   const uint32_t *w, uint32_t source, uint32_t *dist,
                   uint32_t *parent) {
  for (uint32_t v = 0; v < nv; ++v) dist[v] = SGSO_INF;
  uint64_t edges = 0;
  if (source < nv) {
    heap_t h = {0, 0, 0};
    dist[source] = 0;
    hpush(&h, (uint64_t)source);
    while (h.n) {
      uint64_t x = hpop(&h);
      uint32_t u = (uint32_t)x, d = (uint32_t)(x >> 32);
      if (d != dist[u]) continue;
      for (uint64_t e = row[u]; e < row[u + 1]; ++e, ++edges) {
        uint32_t v = col[e];
        uint64_t nd = (uint64_t)d + (w ? w[e] : 1u);
        if (nd < dist[v]) {
          dist[v] = (uint32_t)nd;
          hpush(&h, (nd << 32) | v);
        }
      }
    }
    free(h.a);
  }
  if (parent) tight_parents(nv, row, col, w, dist, parent);
  return edges;
}

/* Widest (maximum-bottleneck) path, a user algorithm of the functor
 * surface with no counterpart among the reference's samples: width[s] =
 * 2^32-1, width[v] = max over paths s -> v of the smallest weight on the
 * path, 0 when unreachable.  Dijkstra on the max-min semiring: the heap pops
 * the widest tentative vertex first (key = ~width). */
uint64_t sgso_widest(uint32_t nv, const uint64_t *row, const uint32_t *col,
                     const uint32_t *w, uint32_t source, uint32_t *width) {
  for (uint32_t v = 0; v < nv; ++v) width[v] = 0;
  uint64_t edges = 0;
  if (source >= nv) return 0;
  heap_t h = {0, 0, 0};
  width[source] = SGSO_INF;
  hpush(&h, ((uint64_t)(uint32_t)~SGSO_INF << 32) | source);
  while (h.n) {
    uint64_t x = hpop(&h);
    uint32_t u = (uint32_t)x, b = ~(uint32_t)(x >> 32);
    if (b != width[u]) continue;
    for (uint64_t e = row[u]; e < row[u + 1]; ++e, ++edges) {
      uint32_t v = col[e];
      uint32_t we = w ? w[e] : 1u;
      uint32_t nb = b < we ? b : we;
      if (nb > width[v]) {
        width[v] = nb;
        hpush(&h, ((uint64_t)(uint32_t)~nb << 32) | v);
      }
    }
  }
  free(h.a);
  return edges;
}

/* hybrid_cc.cu:96-110 pushes atomicMin(buffer[dst], buffer[src]) along
 * out-edges from buffer[v] = v (hybrid_cc.cu:46-49): the fixed point is the
 * smallest id that reaches v.  Computed by searching from ids in increasing
 * order, each search stopping at already-labelled vertices. */
uint64_t sgso_cc(uint32_t nv, const uint64_t *row, const uint32_t *col,
                 uint32_t *label) {
  for (uint32_t v = 0; v < nv; ++v) label[v] = SGSO_INF;
  uint32_t *q = (uint32_t *)malloc(((uint64_t)nv + 1) * sizeof(uint32_t));
  uint64_t edges = 0;
  for (uint32_t r = 0; r < nv; ++r) {
    if (label[r] != SGSO_INF) continue;
    uint64_t h = 0, t = 0;
    label[r] = r;
    q[t++] = r;
    while (h < t) {
      uint32_t u = q[h++];
      for (uint64_t e = row[u]; e < row[u + 1]; ++e, ++edges) {
        uint32_t v = col[e];
        if (label[v] == SGSO_INF) { label[v] = r; q[t++] = v; }
      }
    }
  }
  free(q);
  return edges;
}

/* Fixed point of hybrid_pr.cu:43-122: value starts at 0, buffer at 1-alpha,
 * each combine moves buffer into value and pushes alpha*buffer/outdeg, so
 * x = (1-alpha) + alpha * sum_{u->v} x_u / outdeg(u); vertices without
 * out-edges push nothing.  Jacobi iteration in FP64. */
int sgso_pagerank(uint32_t nv, const uint64_t *row, const uint32_t *col,
                  double alpha, double tol, int max_iter, double *x) {
  double *y = (double *)malloc(((uint64_t)nv + 1) * sizeof(double));
  for (uint32_t v = 0; v < nv; ++v) x[v] = 1.0 - alpha;
  int it = 0;
  for (; it < max_iter; ++it) {
    for (uint32_t v = 0; v < nv; ++v) y[v] = 0.0;
    for (uint32_t u = 0; u < nv; ++u) {
      uint64_t d = row[u + 1] - row[u];
      if (!d) continue;
      double c = x[u] / (double)d;
      for (uint64_t e = row[u]; e < row[u + 1]; ++e) y[col[e]] += c;
    }
    double diff = 0.0;
    for (uint32_t v = 0; v < nv; ++v) {
      double nx = (1.0 - alpha) + alpha * y[v];
      double dd = nx - x[v];
      diff += dd < 0 ? -dd : dd;
      x[v] = nx;
    }
    if (diff < tol) { ++it; break; }
  }
  free(y);
  return it;
}

/* ---------------------------------------------------------------------- */
/* hybrid_sssp_host.cu:35-63: FIFO queue, a vertex is re-queued whenever its
 * distance drops.  w == NULL uses that file's synthesized (u+v)%128. */
uint64_t sgso_sssp_fifo_budget(uint32_t nv, const uint64_t *row,
                               const uint32_t *col, const uint32_t *w,
                               uint32_t source, uint32_t *dist,
                               uint64_t max_edges) {
  for (uint32_t v = 0; v < nv; ++v) dist[v] = SGSO_INF;
  if (source >= nv) return 0;
  uint64_t qcap = (uint64_t)nv + 16, h = 0, t = 0, n = 0;
  uint32_t *q = (uint32_t *)malloc(qcap * sizeof(uint32_t));
  uint64_t edges = 0;
  dist[source] = 0;
  q[t] = source; t = (t + 1) % qcap; n = 1;
  while (n) {
    uint32_t u = q[h]; h = (h + 1) % qcap; --n;
    uint32_t d = dist[u];
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      uint32_t v = col[e];
      uint32_t wt = w ? w[e] : (u + v) % 128u;
      ++edges;
      if (dist[v] > d + wt) {
        dist[v] = d + wt;
        if (n == qcap) { /* grow ring */
          uint64_t nc = qcap * 2;
          uint32_t *nq = (uint32_t *)malloc(nc * sizeof(uint32_t));
          for (uint64_t i = 0; i < n; ++i) nq[i] = q[(h + i) % qcap];
          free(q); q = nq; h = 0; t = n; qcap = nc;
        }
        q[t] = v; t = (t + 1) % qcap; ++n;
      }
    }
    if (edges >= max_edges) break;
  }
  free(q);
  return edges;
}
uint64_t sgso_sssp_fifo(uint32_t nv, const uint64_t *row, const uint32_t *col,
                        const uint32_t *w, uint32_t source, uint32_t *dist) {
  return sgso_sssp_fifo_budget(nv, row, col, w, source, dist, UINT64_MAX);
}

/* hybrid_bfs_host.cpp:33-60 */
uint64_t sgso_bfs_fifo_budget(uint32_t nv, const uint64_t *row,
                              const uint32_t *col, uint32_t source,
                              uint32_t *depth, uint64_t max_edges) {
  for (uint32_t v = 0; v < nv; ++v) depth[v] = SGSO_INF;
  if (source >= nv) return 0;
  uint32_t *q = (uint32_t *)malloc((uint64_t)nv * sizeof(uint32_t));
  uint64_t h = 0, t = 0, edges = 0;
  depth[source] = 0;
  q[t++] = source;
  while (h < t) {
    uint32_t u = q[h++];
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      uint32_t v = col[e];
      ++edges;
      if (depth[v] == SGSO_INF) { depth[v] = depth[u] + 1; q[t++] = v; }
    }
    if (edges >= max_edges) break;
  }
  free(q);
  return edges;
}
uint64_t sgso_bfs_fifo(uint32_t nv, const uint64_t *row, const uint32_t *col,
                       uint32_t source, uint32_t *depth) {
  return sgso_bfs_fifo_budget(nv, row, col, source, depth, UINT64_MAX);
}

/* hybrid_pr_host.cu:43-124 (PageRankHost), float ranks and residuals. */
uint64_t sgso_pr_host_float(uint32_t nv, const uint64_t *row,
                            const uint32_t *col, double alpha, double err,
                            float *ranks) {
  float *res = (float *)calloc((uint64_t)nv + 1, sizeof(float));
  for (uint32_t v = 0; v < nv; ++v) ranks[v] = (float)(1.0 - alpha);
  for (uint32_t u = 0; u < nv; ++u) {
    uint32_t d = (uint32_t)(row[u + 1] - row[u]);
    if (!d) continue;
    float upd = (float)(((1.0 - alpha) * alpha) / d);
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) res[col[e]] += upd;
  }
  uint64_t qcap = (uint64_t)nv + 16, h = 0, t = 0, n = 0, edges = 0;
  uint32_t *q = (uint32_t *)malloc(qcap * sizeof(uint32_t));
  for (uint32_t v = 0; v < nv; ++v) { q[t++] = v; ++n; }
  t %= qcap;
  while (n) {
    uint32_t u = q[h]; h = (h + 1) % qcap; --n;
    float r = res[u];
    ranks[u] += r;
    res[u] = 0;
    uint32_t d = (uint32_t)(row[u + 1] - row[u]);
    if (!d) continue;
    float upd = (float)(r * alpha / d);
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      uint32_t v = col[e];
      float prev = res[v];
      res[v] += upd;
      ++edges;
      if ((double)(prev + upd) > err && (double)prev < err) {
        if (n == qcap) {
          uint64_t nc = qcap * 2;
          uint32_t *nq = (uint32_t *)malloc(nc * sizeof(uint32_t));
          for (uint64_t i = 0; i < n; ++i) nq[i] = q[(h + i) % qcap];
          free(q); q = nq; h = 0; t = n; qcap = nc;
        }
        q[t] = v; t = (t + 1) % qcap; ++n;
      }
    }
  }
  free(q);
  free(res);
  return edges;
}

/* ---------------------------------------------------------------------- */
static int find_edge(const uint64_t *row, const uint32_t *col,
                     const uint32_t *w, uint32_t p, uint32_t v, uint64_t need,
                     int need_tight) {
  for (uint64_t e = row[p]; e < row[p + 1]; ++e) {
    if (col[e] != v) continue;
    if (!need_tight) return 1;
    if ((uint64_t)(w ? w[e] : 1u) == need) return 1;
  }
  return 0;
}

uint64_t sgso_check_tree(uint32_t nv, const uint64_t *row, const uint32_t *col,
                         const uint32_t *w, uint32_t source,
                         const uint32_t *value, const uint32_t *parent) {
  uint64_t bad = 0;
  for (uint32_t u = 0; u < nv; ++u) {
    if (value[u] == SGSO_INF) continue;
    for (uint64_t e = row[u]; e < row[u + 1]; ++e) {
      uint64_t nd = (uint64_t)value[u] + (w ? w[e] : 1u);
      if (nd < value[col[e]]) ++bad;
    }
  }
  for (uint32_t v = 0; v < nv; ++v) {
    if (v == source) {
      if (value[v] != 0 || parent[v] != SGSO_INF) ++bad;
      continue;
    }
    if (value[v] == SGSO_INF) {
      if (parent[v] != SGSO_INF) ++bad;
      continue;
    }
    uint32_t p = parent[v];
    if (p >= nv || value[p] == SGSO_INF || value[p] > value[v]) { ++bad; continue; }
    if (!find_edge(row, col, w, p, v, (uint64_t)value[v] - value[p], 1)) ++bad;
  }
  return bad;
}

uint64_t sgso_check_cc_parent(uint32_t nv, const uint64_t *row,
                              const uint32_t *col, const uint32_t *label,
                              const uint32_t *parent) {
  uint64_t bad = 0;
  for (uint32_t v = 0; v < nv; ++v) {
    if (label[v] == v) {
      if (parent[v] != SGSO_INF) ++bad;
      continue;
    }
    uint32_t p = parent[v];
    if (p >= nv || label[p] != label[v]) { ++bad; continue; }
    if (!find_edge(row, col, NULL, p, v, 0, 0)) ++bad;
  }
  if (bad) return bad;
  /* acyclic: 0 = unknown, 1 = on stack, 2 = reaches a root */
  uint8_t *st = (uint8_t *)calloc((uint64_t)nv + 1, 1);
  uint32_t *path = (uint32_t *)malloc(((uint64_t)nv + 1) * sizeof(uint32_t));
  for (uint32_t v = 0; v < nv; ++v) {
    uint64_t n = 0;
    uint32_t x = v;
    while (x != SGSO_INF && st[x] == 0) {
      st[x] = 1;
      path[n++] = x;
      x = parent[x];
    }
    if (x != SGSO_INF && st[x] == 1) ++bad; /* cycle */
    for (uint64_t i = 0; i < n; ++i) st[path[i]] = 2;
  }
  free(st);
  free(path);
  return bad;
}
