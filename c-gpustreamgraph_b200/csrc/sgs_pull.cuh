// sgs_pull.cuh -- in-edge (CSC) store and the pull kernels over it.
//
// The reference declares pull variants (include/framework/variants/
// pull_functor.h:139-164) that its engine never instantiates (its AppBase
// has no pull entry points, api.cuh:67-78).  Here the in-edges live in a
// second block store with the same layout as the out-edges (per vertex
// off/slots/live/cap, 16-B aligned blocks of source ids, tombstones for
// deletes, HBM only, no weights), built by transposing the out-store once and
// then updated by every snapshot with the same tombstone / append /
// relocation kernels, fed the batch's keys transposed.
//
// PageRank's sweep over all vertices (r[v] = sum over in-edges u->v of
// alpha * r(u) / outdeg(u)) reads it as a pull: every vertex sums its own
// in-edges, so the per-edge FP64 atomicAdd of the push form (hybrid_pr.cu:
// 109-122) becomes a gather plus one store per vertex.  BFS frontiers that
// cover much of the graph run bottom-up over it (an unreached vertex looks
// for a parent among its in-neighbours and stops at the first one found).
#pragma once
#include "sgs_group.cuh"
#include "sgs_segmap.cuh"

namespace sgs {

// In-degree of every vertex from the live slots of the out-store.
struct InCountOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = true;
  struct Payload {
    uint64_t off;
  };
  GraphView g;
  uint32_t *indeg;
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const { return Payload{g.off[v]}; }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &, uint32_t, bool &, uint32_t &,
                                            uint32_t &) const {
    return 0;
  }
  __device__ __forceinline__ uint32_t visit4(uint32_t, const Payload &p, uint32_t j0, uint32_t len,
                                             bool (&)[4], uint32_t (&)[4], uint32_t (&)[4]) const {
    const uint4 ids = ld_quad(adj_at(g, p.off, j0));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t d = quad_at(ids, k);
      if (j0 + k < len && d != SGS_TOMB) atomicAdd(&indeg[d], 1u);
    }
    return 0;
  }
};

// Fill: source u of every live out-slot (u -> d) at the next free place of
// d's in-block (per-destination cursor; order within a block is arbitrary).
struct InFillOp {
  static constexpr bool kAppends = false;
  static constexpr bool kQuad = true;
  struct Payload {
    uint64_t off;
  };
  GraphView g;
  const uint64_t *in_off;
  uint32_t *cursor;
  uint32_t *in_adj;
  uint32_t *in_wgt;  // null: ids only
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const { return Payload{g.off[v]}; }
  __device__ __forceinline__ uint32_t visit(uint32_t, const Payload &, uint32_t, bool &, uint32_t &,
                                            uint32_t &) const {
    return 0;
  }
  __device__ __forceinline__ uint32_t visit4(uint32_t u, const Payload &p, uint32_t j0, uint32_t len,
                                             bool (&)[4], uint32_t (&)[4], uint32_t (&)[4]) const {
    const uint4 ids = ld_quad(adj_at(g, p.off, j0));
    const uint4 ws = in_wgt ? ld_quad(wgt_at(g, p.off, j0)) : make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t d = quad_at(ids, k);
      if (j0 + k >= len || d == SGS_TOMB) continue;
      const uint64_t at = in_off[d] + atomicAdd(&cursor[d], 1u);
      in_adj[at] = u;
      if (in_wgt) in_wgt[at] = quad_at(ws, k);
    }
    return 0;
  }
};

// (src << 32 | dst) -> (dst << 32 | src) for the first *n_dev (or n) keys.
__global__ void k_transpose_keys(const uint64_t *in, uint32_t n, const uint32_t *n_dev, uint64_t *out) {
  const uint32_t cnt = n_dev ? *n_dev : n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const uint64_t k = in[i];
    out[i] = (k << 32) | (k >> 32);
  }
}

// PageRank pull sweep: r[v] = sum over live in-slots u of pv[u], for every
// entry of a dense frontier over the in-store (len = in-slots).  Same unit /
// chunk scheme as seg_map; a thread sums the pv of its quad, a warp reduces
// runs of lanes on the same entry (lanes walk consecutive positions, so an
// entry's lanes are contiguous), run heads add into a shared per-entry sum,
// and each entry is written once per CTA: a plain store when the CTA holds
// all of its positions, an atomicAdd (r is zero from the absorb step) when it
// is split between CTAs.  edge_stat counts the live slots read.
// Coherent: pv was written earlier in the same launch (the persistent round
// kernel k_pr_rounds), so it is read through L2 instead of the non-coherent
// read-only path.
template <bool Coherent>
__device__ __forceinline__ void pull_pr_body(const FrontierView &in, const GraphView &gi, const double *pv,
                                             double *r, unsigned long long *edge_stat) {
  constexpr int GC = CHUNK;
  __shared__ uint64_t s_eb[GC + 1];
  __shared__ uint32_t s_len[GC];
  __shared__ uint32_t s_vtx[GC];
  __shared__ uint64_t s_off[GC];
  __shared__ double s_acc[GC];
  const uint64_t packed = __ldcg((const unsigned long long *)in.counter);
  const uint32_t n = (uint32_t)(packed >> CNT_SHIFT);
  const uint64_t T = packed & EDGE_MASK;
  const uint64_t nunits = (T + UNIT - 1) / UNIT;
  const uint64_t ub = (uint64_t)blockIdx.x * nunits / gridDim.x;
  const uint64_t ue = (uint64_t)(blockIdx.x + 1) * nunits / gridDim.x;
  const int lane = threadIdx.x & 31;
  uint32_t counted = 0;
  if (n != 0 && ub < ue) {
    const uint64_t E0 = ub * UNIT;
    const uint64_t E1 = min(ue * (uint64_t)UNIT, T);
    uint32_t s = __ldcg(&in.ustart[ub]);
    for (;;) {
      __syncthreads();  // previous chunk fully written out
      {
        const uint32_t t = threadIdx.x;
        const uint32_t idx = s + t;
        const uint64_t eb = idx < n ? __ldcg((const unsigned long long *)&in.ebase[idx]) : T;
        s_eb[t] = eb;
        s_acc[t] = 0.0;
        if (t == 0) {
          const uint32_t j = s + GC;
          s_eb[GC] = j < n ? __ldcg((const unsigned long long *)&in.ebase[j]) : T;
        }
        if (idx < n && eb < E1) {
          const uint32_t v = __ldcg(&in.vtx[idx]);
          s_vtx[t] = v;
          s_len[t] = __ldcg(&in.len[idx]);
          s_off[t] = gi.off[v];
        }
      }
      __syncthreads();
      const uint64_t lo = max(E0, s_eb[0]);
      const uint64_t hi = min(E1, s_eb[GC]);
      // every thread of the CTA runs the same trip count (full warps below)
      for (uint64_t base = lo; base < hi; base += 4 * RELAX_THREADS) {
        const uint64_t e = base + 4 * threadIdx.x;
        int l = GC;  // sentinel: no entry
        double part = 0.0;
        if (e < hi) {
          int a = 0, b = GC - 1;
          while (a < b) {
            const int m = (a + b + 1) >> 1;
            if (s_eb[m] <= e) a = m;
            else b = m - 1;
          }
          l = a;
          const uint32_t j0 = (uint32_t)(e - s_eb[a]);
          const uint32_t len = s_len[a];
          if (j0 < len) {
            const uint4 ids = ld_quad(gi.adj_d + s_off[a] + j0);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const uint32_t u = quad_at(ids, k);
              if (j0 + k < len && u != SGS_TOMB) {
                part += Coherent ? __ldcg(pv + u) : __ldg(pv + u);
                ++counted;
              }
            }
          }
        }
        // segmented suffix sums over runs of equal l
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const double o = __shfl_down_sync(0xFFFFFFFFu, part, d);
          const int ol = __shfl_down_sync(0xFFFFFFFFu, l, d);
          if (lane + d < 32 && ol == l) part += o;
        }
        const int pl = __shfl_up_sync(0xFFFFFFFFu, l, 1);
        if (l < GC && (lane == 0 || pl != l) && part != 0.0) atomicAdd(&s_acc[l], part);
      }
      __syncthreads();
      {
        const uint32_t t = threadIdx.x;
        const uint32_t idx = s + t;
        if (idx < n && s_eb[t] < E1) {
          const uint64_t ee = s_eb[t] + ((s_len[t] + 3u) & ~3u);  // end of the entry's padded range
          const double x = s_acc[t];
          if (s_eb[t] >= E0 && ee <= E1) r[s_vtx[t]] = x;
          else if (x != 0.0) atomicAdd(&r[s_vtx[t]], x);
        }
      }
      if (s_eb[GC] >= E1 || s + GC >= n) break;
      s += GC;
    }
  }
  if (edge_stat) {
    const unsigned long long c = warp_sum((unsigned long long)counted);
    if (lane == 0 && c) atomicAdd(edge_stat, c);
  }
}

__global__ void __launch_bounds__(RELAX_THREADS)
    k_pull_pr(FrontierView in, GraphView gi, const double *pv, double *r,
              unsigned long long *edge_stat) {
  pull_pr_body<false>(in, gi, pv, r, edge_stat);
}

// One bottom-up BFS round of a narrow group (S lanes, all running lanes
// BFS): every vertex still unreached in some lane of `lanes` scans its
// in-edges for a parent in frontier r of that lane (m_in bit set), takes
// depth(parent) + 1 and stops once every such lane found one -- Beamer's
// bottom-up step, which reads far fewer edges than the top-down one when the
// frontier holds a large part of the graph.  A vertex is written only by its
// own thread, so no atomics.  Found vertices get their lanes in m_out and are
// appended to frontier r+1 (with their out-slots, as the top-down round
// appends them).  The kernel also clears the masks of frontier r-1 and adds
// frontier r's (lane, out-edge) pairs to lane_edges, as a top-down round
// would have counted them, so the traversed-edge figures keep the reference's
// definition.
template <int S>
__global__ void __launch_bounds__(RELAX_THREADS)
    k_bfs_pull_round(GraphView g, GraphView gi, unsigned long long *st, uint32_t *val, uint32_t lanes,
                     const uint32_t *m_in, uint32_t *m_out, FrontierView cur, const uint32_t *prev_vtx,
                     const unsigned long long *prev_cnt, uint32_t *prev_mask, FrontierView out,
                     unsigned long long *lane_edges) {
  clear_prev_masks(prev_vtx, prev_cnt, prev_mask);
  // (lane, edge) pairs of frontier r
  {
    __shared__ unsigned long long s_lane[S];
    if (threadIdx.x < S) s_lane[threadIdx.x] = 0;
    __syncthreads();
    uint32_t acc[S];
#pragma unroll
    for (int q = 0; q < S; ++q) acc[q] = 0;
    const uint32_t nc = (uint32_t)(__ldcg((const unsigned long long *)cur.counter) >> CNT_SHIFT);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
      const uint32_t v = __ldcg(&cur.vtx[i]);
      const uint32_t m = __ldcg(&m_in[v]) & lanes;
      const uint32_t l = g.live[v];
#pragma unroll
      for (int q = 0; q < S; ++q) acc[q] += (m >> q & 1u) ? l : 0u;
    }
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const unsigned long long x = warp_sum((unsigned long long)acc[q]);
      if ((threadIdx.x & 31) == 0 && x) atomicAdd(&s_lane[q], x);
    }
    __syncthreads();
    if (threadIdx.x < S && s_lane[threadIdx.x] && lane_edges) atomicAdd(&lane_edges[threadIdx.x], s_lane[threadIdx.x]);
  }
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < g.nv; b += stride) {
    const uint64_t v = b + threadIdx.x;
    bool want = false;
    uint32_t d = 0;
    if (v < g.nv) {
      uint32_t cv[S];
      load_vals<S>(val, (uint32_t)v, cv);
      uint32_t need = 0;
#pragma unroll
      for (int q = 0; q < S; ++q)
        if ((lanes >> q & 1u) && cv[q] == INF32) need |= 1u << q;
      uint32_t found = 0;
      if (need) {
        const uint64_t o = gi.off[v];
        const uint32_t n = gi.slots[v];
        for (uint32_t j = 0; j < n && need; ++j) {
          const uint32_t u = __ldg(gi.adj_d + o + j);
          if (u == SGS_TOMB) continue;
          const uint32_t m = __ldcg(&m_in[u]) & need;
          if (!m) continue;
#pragma unroll
          for (int q = 0; q < S; ++q) {
            if (!(m >> q & 1u)) continue;
            const uint32_t du = __ldcg(&val[(uint64_t)u * S + q]) + 1u;
            st[v * S + q] = ((unsigned long long)du << 32) | u;
            val[v * S + q] = du;
          }
          found |= m;
          need &= ~m;
        }
      }
      if (found) {
        d = g.slots[v];
        if (d) {
          m_out[v] = found;
          want = true;
        }
      }
    }
    frontier_append(out, want, (uint32_t)v, d);
  }
}

// Work-efficient repair, round 0 of a narrow group after an invalidation:
// instead of re-pushing from every reached vertex, every vertex the
// invalidation reset pulls over its in-edges (the in-edge store, with
// weights) and takes, per lane, the best candidate its in-neighbours give.
// Before the repair every other edge already satisfies value(u) + w >=
// value(v), so the edges into reset vertices (and the inserted edges, relaxed
// right after) hold every violated edge; later rounds push from the
// vertices that improved.  Runs in group_map with the in-edge store as the
// map's graph; a vertex is appended with its out-slots.
template <int S>
struct GroupPullOp {
  using Payload = GPay<S>;
  GraphView g;                 // the in-edge store
  const uint32_t *out_slots;   // out-store slots (append lengths)
  unsigned long long *st;
  uint32_t *val;
  const uint32_t *m_in;
  uint32_t *m_out;
  LaneAlgo algo;
  int wmode;                   // weights of the SSSP lanes (SGS_W_*)
  __device__ __forceinline__ Payload load(uint32_t v) const {
    Payload p;
    p.off = g.off[v];
    p.mask = __ldcg(&m_in[v]);
    load_vals<S>(val, v, p.val);
    return p;
  }
  struct Quad {
    uint4 ids, ws;
  };
  __device__ __forceinline__ uint32_t append_len(uint32_t v) const { return out_slots[v]; }
  template <bool H>
  __device__ __forceinline__ Quad fetch(const Payload &p, uint32_t j0) const {
    Quad q;
    q.ids = ld_quad(g.adj_d + p.off + j0);
    q.ws = wmode == W_EXPLICIT ? ld_quad(g.wgt_d + p.off + j0) : make_uint4(1, 1, 1, 1);
    return q;
  }
  __device__ __forceinline__ uint32_t visit4(uint32_t v, const Payload &p, uint32_t j0, uint32_t len,
                                             const Quad &qd, uint32_t (&dst)[4]) const {
    uint32_t best[S], bu[S];
#pragma unroll
    for (int q = 0; q < S; ++q) {
      best[q] = INF32;
      bu[q] = 0;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t u = quad_at(qd.ids, k);
      if (j0 + k >= len || u == SGS_TOMB) continue;
      uint32_t cu[S];
      load_vals<S>(val, u, cu);
#pragma unroll
      for (int q = 0; q < S; ++q) {
        if (!(p.mask >> q & 1u)) continue;
        const int a = algo.at(q);
        uint32_t cand;
        if (a == A_CC) {
          cand = cu[q];
        } else {
          if (cu[q] == INF32) continue;
          uint32_t w = 1u;
          if (a == A_SSSP)
            w = wmode == W_EXPLICIT ? quad_at(qd.ws, k) : wmode == W_SYNTH ? (u + v) % 128u + 1u : 1u;
          const uint64_t nd = (uint64_t)cu[q] + w;
          if (nd >= INF32) continue;
          cand = (uint32_t)nd;
        }
        if (cand < best[q]) {
          best[q] = cand;
          bu[q] = u;
        }
      }
    }
    uint32_t bits = 0;
#pragma unroll
    for (int q = 0; q < S; ++q) {
      if (best[q] >= p.val[q]) continue;
      const uint64_t idx = (uint64_t)v * S + q;
      if (relax_mirror_packed(&val[idx], &st[idx], best[q], bu[q])) bits |= 1u << q;
    }
    dst[0] = v;
    dst[1] = dst[2] = dst[3] = 0;
    return bits && out_slots[v] && atomicOr(&m_out[v], bits) == 0u ? 1u : 0u;
  }
};

// Frontier of the vertices set in a bitmap that have in-edges (len = their
// in-slots), with lane mask `lanes` in m_out; eight vertices per thread.
__global__ void k_bits_frontier(const uint32_t *bits, GraphView gi, uint32_t lanes, uint32_t *m_out,
                                FrontierView out) {
  constexpr int N = 8;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * N;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x * N; b < gi.nv; b += stride) {
    const uint64_t v0 = b + (uint64_t)threadIdx.x * N;
    bool want[N];
    uint32_t d[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const uint64_t v = v0 + i;
      want[i] = false;
      d[i] = 0;
      if (v < gi.nv && bit_at(bits, (uint32_t)v)) {
        d[i] = gi.slots[v];
        want[i] = d[i] > 0;
        if (want[i]) m_out[v] = lanes;
      }
    }
    frontier_append_block_n<N>(out, want, (uint32_t)v0, d);
  }
}

}  // namespace sgs
