// sgs_kernels.cuh -- sm_100a kernels of the streaming-graph engine.
//
// Reference behaviour each kernel re-implements (paths relative to the
// reference project):
//   seg_map (sgs_segmap.cuh) and the group ops (sgs_group.cuh)
//                         <- kernel::SyncPushDDBDelta / RelaxCTADB /
//                            CTAWorkSchedulerNew / PushFunctorDB
//                            (variants/driver.cuh:1893-1935,
//                             variants/sync_push_dd.cuh:170-268,
//                             groute/device/cta_scheduler_hybrid.cuh:59-245,
//                             variants/push_functor.h:252-321), the deletion
//                            phase reset_del_edges + SyncPushDDB_del
//                            (driver.cuh:398-430, :1985-2031) and the
//                            all-vertices re-push SyncPushDDBAll (:1727-1761)
//   frontier_append       <- RebuildWorklist* + dev::Queue::append
//                            (driver.cuh:654-909, groute/device/queue.cuh:84-88)
//   PR absorb/push/amend  <- hybrid_pr.cu:66-122 CombineValueBuffer /
//                            CombineValueBufferAmend / AccumulateBuffer and
//                            SyncPushDDBAmend (driver.cuh:1770-1804)
//   batch-apply kernels   <- host::PMAGraph::insert / del_edge
//                            (groute/graphs/csr_graph.cuh:658-811), done on
//                            the device as sort + tombstone + append/relocate
#pragma once
#include <cub/block/block_reduce.cuh>

#include "sgs_device.cuh"
#include "sgs_segmap.cuh"

namespace sgs {

// ---------------------------------------------------------------------------
// Ops
// ---------------------------------------------------------------------------
// PageRank push of a per-source scalar (absorbed residual or +-alpha*x/deg).
struct PrPay {
  uint64_t off;
  double c;
};
struct PrPushOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = true;
  using Payload = PrPay;
  GraphView g;
  const double *pv;   // per-vertex push value (alpha * r / outdeg)
  double *r;
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const {
    PrPay p;
    p.off = g.off[v];
    p.c = pv[v];
    return p;
  }
  __device__ __forceinline__ void touch(uint32_t v, const Payload &p) const { hot_bump(g, v, p.off); }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &p, uint32_t j,
                                            bool &, uint32_t &, uint32_t &) const {
    const uint32_t dst = *adj_at(g, p.off, j);
    if (dst == SGS_TOMB) return 0;
    if (p.c != 0.0) atomicAdd(&r[dst], p.c);
    return 1;
  }
  __device__ __forceinline__ uint32_t visit4(uint32_t, const Payload &p, uint32_t j0, uint32_t len,
                                             bool (&)[4], uint32_t (&)[4], uint32_t (&)[4]) const {
    const uint4 ids = ld_quad(adj_at(g, p.off, j0));
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t dst = quad_at(ids, k);
      if (j0 + k >= len || dst == SGS_TOMB) continue;
      ++c;
      if (p.c != 0.0) atomicAdd(&r[dst], p.c);
    }
    return c;
  }
};
// Cancel (sign=-1, old graph) / compensate (sign=+1, new graph) of
// hybrid_pr.cu:88-106, restricted to sources whose out-edges changed.
struct PrAmendOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = false;
  using Payload = PrPay;
  GraphView g;
  const double *x;
  double *r;
  double scale;  // sign * alpha
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const {
    PrPay p;
    p.off = g.off[v];
    const uint32_t l = g.live[v];
    p.c = l ? scale * x[v] / (double)l : 0.0;
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &p, uint32_t j,
                                            bool &, uint32_t &, uint32_t &) const {
    const uint32_t dst = *adj_at(g, p.off, j);
    if (dst == SGS_TOMB) return 0;
    if (p.c != 0.0) atomicAdd(&r[dst], p.c);
    return 1;
  }
};

// Tombstone every slot of u whose destination is in u's sorted delete group
// (PMAGraph::del_edge removes every matching entry).  Four slots per thread,
// each looked up by binary search in the group (a few L1-resident lines); the
// block is read with a plain (coherent) load because this kernel writes it.
struct GroupPay {
  uint64_t off;
  uint32_t gs, ge;
};
struct TombOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = true;
  using Payload = GroupPay;
  GraphView g;
  const uint64_t *keys;   // sorted delete keys (src<<32|dst)
  const uint32_t *gstart; // per entry
  uint32_t nkeys;
  __device__ __forceinline__ Payload load(uint32_t slot, uint32_t v) const {
    GroupPay p;
    p.off = g.off[v];
    p.gs = gstart[slot];
    // end of the group: first key with a larger source.  Galloping from
    // the group start: most sources have one or two deletes, so the first
    // probe usually ends it; a hub's long group takes log2(size) probes.
    const uint64_t lim = ((uint64_t)v + 1) << 32;
    uint32_t lo = p.gs + 1, step = 1, hi = p.gs + 1;  // keys[gs] < lim
    while (hi < nkeys && keys[hi] < lim) {
      lo = hi + 1;
      step <<= 1;
      hi = p.gs + step;
    }
    uint32_t r = hi < nkeys ? hi : nkeys;
    uint32_t l = lo;
    while (l < r) {
      const uint32_t m = (l + r) >> 1;
      if (keys[m] < lim) l = m + 1;
      else r = m;
    }
    p.ge = l;
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &, uint32_t, bool &, uint32_t &,
                                            uint32_t &) const {
    return 0;
  }
  __device__ __forceinline__ uint32_t visit4(uint32_t u, const Payload &p, uint32_t j0, uint32_t len,
                                             bool (&)[4], uint32_t (&)[4], uint32_t (&)[4]) const {
    uint32_t *a = adj_wptr(g, p.off) + j0;
    uint32_t *ca = cache_slot_w(g, g.adj_c, p.off, j0);  // cached copy: read from it, write both
    const uint4 q = *reinterpret_cast<const uint4 *>(ca ? ca : a);
    uint64_t key[4];
    bool ok[4];
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t dst = quad_at(q, k);
      ok[k] = j0 + k < len && dst != SGS_TOMB;
      key[k] = ((uint64_t)u << 32) | dst;
      any |= ok[k];
    }
    if (!any) return 0;
    // the four lower bounds in lockstep (branchless, the same trip count for
    // all: it depends only on the group's length), so their dependent loads
    // overlap instead of running one search after the other
    uint32_t lo[4] = {p.gs, p.gs, p.gs, p.gs};
    uint32_t n = p.ge - p.gs;  // >= 1: the entry has deletes
    while (n > 1) {
      const uint32_t half = n >> 1;
#pragma unroll
      for (int k = 0; k < 4; ++k) lo[k] = __ldg(&keys[lo[k] + half]) < key[k] ? lo[k] + half : lo[k];
      n -= half;
    }
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!ok[k]) continue;
      const uint64_t kk = __ldg(&keys[lo[k]]);
      const uint32_t at = kk < key[k] ? lo[k] + 1 : lo[k];
      if (at < p.ge && (at == lo[k] ? kk : __ldg(&keys[at])) == key[k]) {
        a[k] = SGS_TOMB;
        if (ca) ca[k] = SGS_TOMB;
        ++c;
      }
    }
    if (c) atomicSub(&g.live[u], c);
    return c;
  }
};

// Copy of a whole block (slots as they are, tombstones included) from an old
// location to the vertex's current block; used by relocation and repacking.
struct CopyPay {
  uint64_t from;
  uint64_t to;
};
struct CopyBlockOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = false;
  using Payload = CopyPay;
  GraphView g;
  const uint64_t *from_off;  // per vertex: old offset (tier bit included)
  const uint64_t *to_off;    // per vertex: new offset
  uint32_t *src_adj_d, *src_wgt_d, *src_adj_h, *src_wgt_h;  // source arenas
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const {
    CopyPay p;
    p.from = from_off[v];
    p.to = to_off[v];
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &p, uint32_t j,
                                            bool &, uint32_t &, uint32_t &) const {
    const uint64_t fo = p.from & OFF_MASK;
    const bool fh = (p.from & HOST_BIT) != 0;
    const uint32_t a = (fh ? src_adj_h : src_adj_d)[fo + j];
    adj_wptr(g, p.to)[j] = a;
    if (g.wmode == W_EXPLICIT) wgt_wptr(g, p.to)[j] = (fh ? src_wgt_h : src_wgt_d)[fo + j];
    return 0;
  }
};

// Copy an input CSR (device arrays) into the arena blocks.
struct LoadCsrOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = false;
  using Payload = CopyPay;
  GraphView g;
  const uint64_t *row;
  const uint32_t *col;
  const uint32_t *w;   // null unless weights are explicit
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const {
    CopyPay p;
    p.from = row[v];
    p.to = g.off[v];
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &p, uint32_t j,
                                            bool &, uint32_t &, uint32_t &) const {
    adj_wptr(g, p.to)[j] = col[p.from + j];
    if (w) wgt_wptr(g, p.to)[j] = w[p.from + j];
    return 0;
  }
};

// Export blocks (live edges only) into a CSR whose row offsets are given.  A
// block without tombstones keeps its order; otherwise live slots are placed
// through a per-vertex counter (order not kept).
struct ExportPay {
  uint64_t from;
  uint64_t to;
  uint32_t dense;
  uint32_t pad;
};
struct ExportOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = false;
  using Payload = ExportPay;
  GraphView g;
  const uint64_t *row_out;
  uint32_t *col_out;
  uint32_t *w_out;
  uint32_t *fill;  // per-vertex fill counter (zeroed)
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const {
    ExportPay p;
    p.from = g.off[v];
    p.to = row_out[v];
    p.dense = g.slots[v] == g.live[v];
    p.pad = 0;
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t u, const Payload &p, uint32_t j,
                                            bool &, uint32_t &, uint32_t &) const {
    const uint32_t dst = adj_ptr(g, p.from)[j];
    if (dst == SGS_TOMB) return 0;
    const uint32_t k = p.dense ? j : atomicAdd(&fill[u], 1u);
    col_out[p.to + k] = dst;
    if (w_out) w_out[p.to + k] = edge_weight(g, p.from, j, u, dst);
    return 1;
  }
};

// ---------------------------------------------------------------------------
// Frontier builders (all lanes of every warp reach frontier_append)
// ---------------------------------------------------------------------------
__global__ void k_append_one(FrontierView out, uint32_t v, uint32_t d) {
  if (threadIdx.x >= 32) return;
  frontier_append(out, threadIdx.x == 0 && d > 0, v, d);
}

// Every vertex with a non-empty block (PageRank rounds, loads, repacks).
__global__ void k_dense_frontier(GraphView g, FrontierView out) {
  constexpr int N = 8;  // consecutive vertices per thread, one block append per 2048
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * N;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x * N; b < g.nv; b += stride) {
    const uint64_t v0 = b + (uint64_t)threadIdx.x * N;
    bool want[N];
    uint32_t d[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      d[i] = v0 + i < g.nv ? g.slots[v0 + i] : 0u;
      want[i] = d[i] > 0;
    }
    frontier_append_block_n<N>(out, want, (uint32_t)v0, d);
  }
}

// PageRank: value 0, buffer (residual) 1-alpha (hybrid_pr.cu:43-52).
__global__ void k_pr_init(double *x, double *r, uint32_t nv, double r0) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    x[v] = 0.0;
    r[v] = r0;
  }
}

// Warm start from a previous solution x0 (kept in x): push values
// pv = alpha * x0 / outdeg and a zeroed residual; after one sweep
// r = sum over in-edges of pv, k_pr_warm_res turns it into the residual of x0,
// r = (1 - alpha) + alpha P^T x0 - x0, so that x0 + (I - alpha P^T)^-1 r is
// the fixed point and the rounds continue from there.
__global__ void k_pr_warm_pv(GraphView g, const double *x, double *pv, double *r, double alpha) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < g.nv; v += stride) {
    const uint32_t l = g.live[v];
    pv[v] = l ? alpha * x[v] / (double)l : 0.0;
    r[v] = 0.0;
  }
}
__global__ void k_pr_warm_res(const double *x, double *r, uint32_t nv, double base) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride)
    r[v] = base + r[v] - x[v];
}

// Absorb: value += residual, residual = 0, push value alpha*res/outdeg
// (CombineValueBuffer, hybrid_pr.cu:66-85).  Accumulates the L1 norm of the
// absorbed residual into *l1.
// Coherent: r was written earlier in the same launch by other CTAs (the
// persistent round kernel), so it is read through L2.
template <bool Coherent>
__device__ __forceinline__ void pr_absorb_body(const GraphView &g, double *x, double *r, double *pv,
                                               double alpha, double *l1) {
  double acc = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < g.nv; v += stride) {
    const double rv = Coherent ? __ldcg(r + v) : r[v];
    double p = 0.0;
    if (rv != 0.0) {
      r[v] = 0.0;
      x[v] += rv;
      acc += fabs(rv);
      const uint32_t l = g.live[v];
      if (l) p = alpha * rv / (double)l;
    }
    pv[v] = p;
  }
  typedef cub::BlockReduce<double, RELAX_THREADS> BR;
  __shared__ typename BR::TempStorage tmp;
  const double tot = BR(tmp).Sum(acc);
  if (threadIdx.x == 0 && tot != 0.0) atomicAdd(l1, tot);
}

__global__ void k_pr_absorb(GraphView g, double *x, double *r, double *pv,
                            double alpha, double *l1) {
  pr_absorb_body<false>(g, x, r, pv, alpha, l1);
}

// PageRank rounds r0, r0+1, ... (at most `limit`) of the pull form in one
// cooperative launch: absorb, grid barrier, pull sweep over the dense
// in-store frontier `fin`, grid barrier, then every thread reads the round's
// absorbed L1 (complete after the barrier) and all stop together once it is
// below `tol` -- the rounds of the launch-per-kernel loop, in the same
// order, without a launch pair per round and a host read per few rounds
// (which dominate when the graph sits in L2).  *rounds_out = rounds run.
// r and pv are written by other CTAs within the launch and read through L2.
__global__ void __launch_bounds__(RELAX_THREADS)
    k_pr_rounds(GraphView g, FrontierView fin, GraphView gi, double *x, double *r, double *pv,
                double alpha, double tol, double *l1buf, uint32_t r0, uint32_t limit,
                unsigned long long *edge_stat, uint32_t *rounds_out) {
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  uint32_t k = 0;
  while (k < limit) {
    pr_absorb_body<true>(g, x, r, pv, alpha, l1buf + r0 + k);
    __threadfence();
    grid.sync();
    pull_pr_body<true>(fin, gi, pv, r, edge_stat);
    __threadfence();
    grid.sync();
    const double l1v = __ldcg(l1buf + r0 + k);
    ++k;
    if (l1v < tol) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *rounds_out = k;
}

// ---------------------------------------------------------------------------
// Batch apply
// ---------------------------------------------------------------------------
__global__ void k_make_keys(const uint32_t *src, const uint32_t *dst, uint64_t n,
                            uint32_t nv, uint64_t *keys, const uint32_t *w,
                            int check_w, unsigned int *err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t u = src[i], v = dst[i];
    if (u >= nv || v >= nv) atomicOr(err, 1u);
    if (check_w && w && w[i] == 0) atomicOr(err, 2u);
    keys[i] = ((uint64_t)u << 32) | v;
  }
}

__device__ __forceinline__ bool sorted_has(const uint64_t *a, uint32_t n, uint64_t k) {
  uint32_t l = 0, r = n;
  while (l < r) {
    uint32_t m = (l + r) >> 1;
    if (a[m] < k) l = m + 1;
    else r = m;
  }
  return l < n && a[l] == k;
}

// flag[i] = insert i survives the batch's deletes (insert-then-delete order of
// framework.cuh:1011-1012).
__global__ void k_filter_inserts(const uint64_t *ins, uint32_t n_ins,
                                 const uint64_t *del, uint32_t n_del,
                                 unsigned char *flag) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_ins; i += stride)
    flag[i] = n_del ? !sorted_has(del, n_del, ins[i]) : 1;
}

// One entry per distinct source of a sorted key list (group heads); aux =
// group start.  With `mark`, sources already marked with `stamp` are skipped,
// which builds the union of the sources of several lists.
__global__ void k_group_heads(GraphView g, const uint64_t *keys,
                              const uint32_t *n_ptr, uint32_t n_fixed,
                              uint32_t *gstart, uint32_t *mark, uint32_t stamp,
                              FrontierView out) {
  const uint32_t n = n_ptr ? *n_ptr : n_fixed;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    bool want = false;
    uint32_t u = 0, d = 0;
    if (i < n) {
      u = (uint32_t)(keys[i] >> 32);
      const bool head = i == 0 || (uint32_t)(keys[i - 1] >> 32) != u;
      if (head) {
        d = g.slots[u];
        want = d > 0;
        if (want && mark) want = atomicExch(&mark[u], stamp) != stamp;
      }
    }
    frontier_append_block(out, want, u, d, gstart, (uint32_t)i);
  }
}

// Insert phase 1 (one thread per distinct source of the kept, sorted inserts):
// append in place when the block has room, else relocate the block to a new
// region of the same tier (capacity grows 1.5x) and queue the copy of the old
// slots.  Mirrors PMAGraph::insert's "append at index+degree" and its
// resize-on-overflow, without shifting neighbours.
struct InsertCtx {
  unsigned long long *arena_top;   // [2] per tier
  uint64_t arena_cap[2];
  unsigned int *err;
  uint64_t *wbase;                 // per vertex: write position of its inserts
  // relocation list
  uint32_t *rl_vtx;
  uint64_t *rl_from;
  uint64_t *rl_to;
  uint32_t *rl_len;
  unsigned long long *rl_count64;
};

__device__ __forceinline__ uint32_t grow_cap(uint32_t need) {
  uint64_t c = (uint64_t)need + (need >> 1) + 4;
  c = (c + 3) & ~3ull;
  return (uint32_t)min(c, (uint64_t)0xFFFFFFF0u);
}

__global__ void k_insert_plan(GraphView g, const uint64_t *keys, const uint32_t *n_ptr,
                              InsertCtx c, int dry, unsigned long long *demand) {
  const uint32_t n = *n_ptr;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    // per-lane decision; the arena/demand/relocation atomics are warp-aggregated
    bool head = false, reloc = false;
    uint32_t u = 0, k = 0, sl = 0, nc = 0;
    uint64_t o = 0;
    int tier = 0;
    if (i < n) {
      u = (uint32_t)(keys[i] >> 32);
      head = i == 0 || (uint32_t)(keys[i - 1] >> 32) != u;
    }
    if (head) {
      // group end: exponential then binary search (groups are usually tiny)
      const uint64_t lim = ((uint64_t)u + 1) << 32;
      uint32_t lo = (uint32_t)i + 1, step = 1, hi = lo;
      while (hi < n && keys[hi] < lim) {
        lo = hi + 1;
        hi = (uint32_t)min((uint64_t)hi + step, (uint64_t)n);
        step <<= 1;
      }
      while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (keys[m] < lim) lo = m + 1;
        else hi = m;
      }
      k = lo - (uint32_t)i;
      sl = g.slots[u];
      const uint32_t cp = g.cap[u];
      const uint64_t need = (uint64_t)sl + k;
      o = g.off[u];
      tier = (o & HOST_BIT) ? 1 : 0;
      if (need <= cp) {
        if (!dry) {
          c.wbase[u] = o + sl;
          g.slots[u] = (uint32_t)need;
          g.live[u] += k;
        }
      } else if (need > 0xFFFFFFF0ull) {
        atomicOr(c.err, 4u);
      } else {
        reloc = true;
        nc = grow_cap((uint32_t)need);
      }
    }
    if (dry) {
      for (int t = 0; t < 2; ++t) warp_atomic_add(&demand[t], reloc && tier == t, nc);
      continue;
    }
    unsigned long long pos[2];
    for (int t = 0; t < 2; ++t) pos[t] = warp_atomic_add(&c.arena_top[t], reloc && tier == t, nc);
    const unsigned long long q =
        warp_atomic_add((unsigned long long *)c.rl_count64, reloc && sl > 0, 1ull);
    if (reloc) {
      const unsigned long long p0 = pos[tier];
      if (p0 + nc > c.arena_cap[tier]) {
        atomicOr(c.err, 8u);
      } else {
        const uint64_t no = p0 | (tier ? HOST_BIT : 0);
        if (sl) {
          c.rl_vtx[q] = u;
          c.rl_from[q] = o;
          c.rl_to[q] = no;
          c.rl_len[q] = sl;
        }
        c.wbase[u] = no + sl;
        g.off[u] = no;
        g.cap[u] = nc;
        g.slots[u] = sl + k;
        g.live[u] += k;
      }
    }
  }
}

// Insert phase 2: one thread per kept insert writes (dst, w) at its rank
// within its source's group.
__global__ void k_insert_write(GraphView g, const uint64_t *keys, const uint32_t *w,
                               const uint32_t *n_ptr, const uint64_t *wbase) {
  const uint32_t n = *n_ptr;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t k = keys[i];
    const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
    // group start: exponential search backwards, then binary search
    const uint64_t lo_key = (uint64_t)u << 32;
    uint32_t hi = (uint32_t)i, step = 1, lo = hi;
    while (lo > 0 && keys[lo - 1] >= lo_key) {
      hi = lo - 1;
      lo = lo > step ? lo - step : 0;
      step <<= 1;
    }
    while (lo < hi) {
      const uint32_t m = (lo + hi) >> 1;
      if (keys[m] < lo_key) lo = m + 1;
      else hi = m;
    }
    const uint64_t pos = wbase[u] + (i - lo);
    const bool ew = g.wmode == W_EXPLICIT;
    store_slot(g, pos, 0, v, ew, ew ? w[i] : 0u);
  }
}

// Relocation list -> frontier of copy entries; the entry's vertex field holds
// the relocation list index.
__global__ void k_reloc_frontier(const unsigned long long *rl_count, const uint32_t *rl_len,
                                 FrontierView out) {
  const uint32_t n = (uint32_t)*rl_count;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    const uint32_t d = i < n ? rl_len[i] : 0u;
    frontier_append(out, d > 0, (uint32_t)i, d);
  }
}

// Copy op over relocation entries: vertex field = relocation list index.
// Tombstone reclamation.  The reference's del_edge shifts the rest of the
// list left on every delete (csr_graph.cuh:789-811) and its PMA rebalances
// windows by density (:813-933).  Here a snapshot's deletes only write
// tombstones, and then every block they touched whose dead slots reach a
// sixteenth of its live ones is compacted in place: one warp per block reads 32
// slots at a time, keeps the live ones (ballot + prefix) and writes them
// forward, so the block's used slots become its live count and the next
// inserts append right after them.  Each compaction costs at most 17 times
// the slots it reclaims, and no block walked by a relaxation keeps more than
// a sixteenth of dead slots.  Input: the frontier of the touched blocks (one
// entry per source); reclaimed slots are added to *reclaimed.  A block of
// COMPACT_LARGE slots or more (the hubs, which lose edges in every snapshot
// and cross the threshold together) is not walked by a warp, whose steps
// each wait for one load: its vertex goes to `big` (count in big_n) for
// k_compact_large, a CTA per block.
constexpr uint32_t COMPACT_LARGE = 1024;
__global__ void k_compact_blocks(GraphView g, FrontierView f, unsigned long long *reclaimed,
                                 uint32_t *big, uint32_t *big_n) {
  const uint32_t n = (uint32_t)(__ldcg((const unsigned long long *)f.counter) >> CNT_SHIFT);
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const bool ew = g.wmode == W_EXPLICIT;
  unsigned long long got = 0;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    const uint32_t v = __ldcg(&f.vtx[i]);
    const uint32_t sl = g.slots[v], lv = g.live[v];
    const uint32_t dead = sl - lv;
    if (dead == 0 || (uint64_t)dead * 16 < lv) continue;  // warp-uniform
    if (sl >= COMPACT_LARGE) {
      if (lane == 0) big[atomicAdd(big_n, 1u)] = v;
      continue;
    }
    const uint64_t o = g.off[v];
    const uint32_t *a = adj_wptr(g, o);
    const uint32_t *wt = ew ? wgt_wptr(g, o) : nullptr;
    uint32_t out = 0;
    for (uint32_t j = 0; j < sl; j += 32) {
      const uint32_t k = j + lane;
      const uint32_t id = k < sl ? __ldcg(a + k) : SGS_TOMB;
      const uint32_t w = (ew && k < sl) ? __ldcg(wt + k) : 0u;
      const bool keep = id != SGS_TOMB;
      const uint32_t b = __ballot_sync(0xFFFFFFFFu, keep);
      // every lane's reads of this step are done before any write; writes
      // land at or below the positions just read, never on unread slots
      __syncwarp();
      if (keep) store_slot(g, o, out + __popc(b & ((1u << lane) - 1u)), id, ew, w);
      out += __popc(b);
      __syncwarp();
    }
    if (lane == 0) {
      g.slots[v] = out;
      got += sl - out;
    }
  }
  if (lane == 0 && got) atomicAdd(reclaimed, got);
}

// In-place compaction of the large blocks listed by k_compact_blocks, one
// CTA per block, in tiles of 4 * COMPACT_THREADS slots: every thread loads a
// 16-B quad of ids (and weights), the CTA scans the live counts and writes
// the live slots forward.  A tile's writes land at or below the positions it
// read, all of which were read before the first barrier of the tile, and
// below the next tile's first slot, so the next tile is loaded before the
// current one is written (software pipeline).  Blocks start on a 4-slot
// boundary and hold a multiple of 4 slots of capacity, so a quad read past
// the used slots stays inside the block.
constexpr int COMPACT_THREADS = 512;
__global__ void __launch_bounds__(COMPACT_THREADS)
    k_compact_large(GraphView g, const uint32_t *big, const uint32_t *big_n, unsigned long long *reclaimed) {
  constexpr int NW = COMPACT_THREADS / 32;
  constexpr uint32_t TILE = 4u * COMPACT_THREADS;
  __shared__ uint32_t s_warp[NW];
  __shared__ uint32_t s_tot;
  const uint32_t n = __ldcg(big_n);
  const bool ew = g.wmode == W_EXPLICIT;
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint4 none = make_uint4(SGS_TOMB, SGS_TOMB, SGS_TOMB, SGS_TOMB);
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t v = __ldcg(&big[i]);
    const uint32_t sl = g.slots[v];
    const uint64_t o = g.off[v];
    const uint32_t *a = adj_wptr(g, o);
    const uint32_t *wt = ew ? wgt_wptr(g, o) : nullptr;
    auto load = [&](uint32_t j, uint4 &ids, uint4 &ws) {
      const uint32_t k0 = j + 4 * threadIdx.x;
      ids = none;
      ws = make_uint4(0, 0, 0, 0);
      if (k0 < sl) {
        ids = __ldcg(reinterpret_cast<const uint4 *>(a + k0));
        if (ew) ws = __ldcg(reinterpret_cast<const uint4 *>(wt + k0));
      }
    };
    uint4 ids, ws;
    load(0, ids, ws);
    uint32_t out = 0;  // CTA-uniform
    for (uint32_t j = 0; j < sl; j += TILE) {
      uint4 nids = none, nws = make_uint4(0, 0, 0, 0);
      if (j + TILE < sl) load(j + TILE, nids, nws);
      const uint32_t k0 = j + 4 * threadIdx.x;
      uint32_t keep = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (k0 + k < sl && quad_at(ids, k) != SGS_TOMB) keep |= 1u << k;
      const uint32_t c = __popc(keep);
      uint32_t x = c;  // inclusive scan over the warp
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= (uint32_t)d) x += y;
      }
      if (lane == 31) s_warp[wid] = x;
      __syncthreads();
      if (wid == 0) {
        const uint32_t t = lane < (uint32_t)NW ? s_warp[lane] : 0u;
        uint32_t u = t;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, u, d);
          if (lane >= (uint32_t)d) u += y;
        }
        if (lane < (uint32_t)NW) s_warp[lane] = u - t;
        if (lane == NW - 1) s_tot = u;
      }
      __syncthreads();
      uint32_t pos = out + s_warp[wid] + x - c;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (keep >> k & 1u) store_slot(g, o, pos++, quad_at(ids, k), ew, quad_at(ws, k));
      out += s_tot;
      __syncthreads();  // s_warp / s_tot are rewritten by the next tile
      ids = nids;
      ws = nws;
    }
    if (threadIdx.x == 0) {
      g.slots[v] = out;
      if (sl > out) atomicAdd(reclaimed, (unsigned long long)(sl - out));
    }
  }
}

struct RelocCopyOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = false;
  using Payload = CopyPay;
  GraphView g;
  const uint64_t *rl_from;
  const uint64_t *rl_to;
  __device__ __forceinline__ Payload load(uint32_t, uint32_t q) const {
    CopyPay p;
    p.from = rl_from[q];
    p.to = rl_to[q];
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &p, uint32_t j,
                                            bool &, uint32_t &, uint32_t &) const {
    const bool ew = g.wmode == W_EXPLICIT;
    store_slot(g, p.to, j, *adj_at(g, p.from, j), ew, ew ? *wgt_at(g, p.from, j) : 0u);
    return 0;
  }
};

// Per-vertex block layout for a fresh arena: capacity with slack.
__global__ void k_layout_caps(const uint32_t *deg, uint32_t nv, uint32_t slack_div,
                              uint32_t *cap) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    const uint32_t d = deg[v];
    uint64_t c = d ? (uint64_t)d + (slack_div ? d / slack_div : 0) + 2 : 0;
    c = (c + 3) & ~3ull;
    cap[v] = (uint32_t)min(c, (uint64_t)0xFFFFFFF0u);
  }
}

// Device-side validation of a caller CSR: offsets start at 0 and do not
// decrease, destinations < nv, explicit weights >= 1.
__global__ void k_validate_csr(const uint64_t *row, const uint32_t *col, const uint32_t *w,
                               uint32_t nv, uint64_t ne, unsigned int *err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0 && row[0] != 0) atomicOr(err, 4u);
  for (uint64_t v = tid; v < nv; v += stride)
    if (row[v + 1] < row[v]) atomicOr(err, 4u);
  for (uint64_t i = tid; i < ne; i += stride) {
    if (col[i] >= nv) atomicOr(err, 1u);
    if (w && w[i] == 0) atomicOr(err, 2u);
  }
}

__global__ void k_row_degrees(const uint64_t *row, uint32_t nv, uint32_t *deg) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride)
    deg[v] = (uint32_t)(row[v + 1] - row[v]);
}

// Assign tiers: vertices [0, split) in HBM, the rest in the host arena; the
// offsets come from an exclusive scan of capacities per tier.
__global__ void k_assign_off(const uint64_t *scan, uint32_t nv, uint32_t split,
                             uint64_t host_base_scan, uint64_t *off) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride)
    off[v] = v < split ? scan[v] : ((scan[v] - host_base_scan) | HOST_BIT);
}

__global__ void k_u32_to_u64(const uint32_t *a, uint32_t n, uint64_t *b) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    b[i] = a[i];
}

// ---------------------------------------------------------------------------
// Device R-MAT generator: bit-identical to the oracle's sgso_rmat_edge.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t fin64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
constexpr uint64_t GAMMA = 0x9E3779B97F4A7C15ull;

__global__ void k_rmat(uint32_t scale, uint64_t ne, uint64_t key, uint64_t tA,
                       uint64_t tAB, uint64_t tABC, int drop_self, uint64_t *keys) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < ne; k += stride) {
    uint32_t uu = 0, vv = 0;
    for (uint32_t l = 0; l < scale; ++l) {
      const uint64_t r = fin64(key + (k * 64u + l + 1) * GAMMA) >> 11;
      uint32_t bu, bv;
      if (r < tA) { bu = 0; bv = 0; }
      else if (r < tAB) { bu = 0; bv = 1; }
      else if (r < tABC) { bu = 1; bv = 0; }
      else { bu = 1; bv = 1; }
      uu = (uu << 1) | bu;
      vv = (vv << 1) | bv;
    }
    keys[k] = (drop_self && uu == vv) ? ~0ull : (((uint64_t)uu << 32) | vv);
  }
}

// Weight of edge (u,v) = 1 + top 6 bits of fin64(wkey ^ (u<<32|v)): uniform in
// [1,64]; identical to the oracle's sgso_weight_of.
__global__ void k_hash_weights(const uint64_t *keys, const uint32_t *n_ptr, uint64_t wkey,
                               uint32_t *w) {
  const uint32_t n = *n_ptr;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    w[i] = 1u + (uint32_t)(fin64(wkey ^ keys[i]) >> 58);
}

// row[v] = first index of a key with source >= v in a sorted key list.
__global__ void k_row_from_sorted(const uint64_t *keys, const uint32_t *n_ptr, uint32_t nv,
                                  uint64_t *row) {
  const uint32_t n = *n_ptr;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= nv; v += stride) {
    const uint64_t k = v << 32;
    uint32_t l = 0, r = n;
    while (l < r) {
      uint32_t m = (l + r) >> 1;
      if (keys[m] < k) l = m + 1;
      else r = m;
    }
    row[v] = l;
  }
}

__global__ void k_keys_low(const uint64_t *keys, const uint32_t *n_ptr, uint32_t *col) {
  const uint32_t n = *n_ptr;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    col[i] = (uint32_t)keys[i];
}

__global__ void k_summary_pr(const double *x, uint32_t nv, double *out) {
  double sum = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) sum += x[v];
  typedef cub::BlockReduce<double, RELAX_THREADS> BR;
  __shared__ typename BR::TempStorage tmp;
  const double s = BR(tmp).Sum(sum);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

}  // namespace sgs
