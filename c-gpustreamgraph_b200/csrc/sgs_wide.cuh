// sgs_wide.cuh -- wide query groups: up to 64 BFS / SSSP / CC queries (any
// sources, uneven frontiers) relaxed together over one edge stream.
//
// Layout: st[v * 64 + q] u64 packed (value << 32 | parent) and the u32 value
// mirror val[v * 64 + q], so the 64 lanes of one vertex are one contiguous
// row (512 B / 256 B).  Lane masks are u64 per vertex in three rotating
// buffers, with the same protocol as the narrow groups (sgs_group.cuh): round
// r reads mask r%3, writes (r+1)%3 and clears the previous frontier's masks,
// and the thread whose atomicOr turns a mask non-zero appends the vertex.
//
// Mapping: a warp walks 32 consecutive edge slots of the frontier at a time
// (one coalesced id read), then relaxes them one by one with the warp's
// threads covering the lanes -- thread t owns lanes t and t + 32 -- so every
// destination row is read with two coalesced 128-B requests and lanes that
// are not active at the source issue no load at all.  This is the batched
// form of the single-query relaxation (hybrid_sssp.cu:97-118 min relaxation,
// hybrid_cc.cu:96-110 label propagation) and of the parent-tree reset
// (reset_del_edges / SyncPushDDB_del, driver.cuh:398-430, :1985-2031).
#pragma once
#include "sgs_device.cuh"
#include "sgs_group.cuh"
#include "sgs_segmap.cuh"

namespace sgs {

constexpr int WLANES = 64;
constexpr int WCHUNK = 256;  // entries staged per chunk by wide_map
// a window with more (edge, lane) pairs than this many per edge on average
// takes the per-edge path of wide_map, a sparser one the per-pair path
constexpr uint32_t WIDE_DENSE_LANES = 12;

// Lane algorithms of a wide group as bit masks (a lane in neither is BFS).
struct WideAlgo {
  uint64_t sssp;
  uint64_t cc;
};

__device__ __forceinline__ uint64_t ballot64(bool lo, bool hi) {
  const uint32_t a = __ballot_sync(0xFFFFFFFFu, lo);
  const uint32_t b = __ballot_sync(0xFFFFFFFFu, hi);
  return (uint64_t)a | ((uint64_t)b << 32);
}

__device__ __forceinline__ void clear_prev_masks64(const uint32_t *vtx, const unsigned long long *cnt,
                                                   unsigned long long *mask) {
  if (!cnt) return;
  const uint32_t n = (uint32_t)(__ldcg(cnt) >> CNT_SHIFT);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    mask[__ldcg(&vtx[i])] = 0ull;
}

// Relaxation of one lane: candidate from the source value, strict
// improvement through the packed word, mirror lowered after it.
template <bool Restrict = false>
struct WideRelaxOp {
  static constexpr bool kNeedsSourceValues = true;
  static constexpr bool kRestrict = Restrict;
  using Pre = uint32_t;
  unsigned long long *st;
  uint32_t *val;
  WideAlgo algo;
  // restricted rounds: per vertex, the lanes the last invalidation reset
  // there; an edge is relaxed only in those lanes of its destination
  const unsigned long long *only = nullptr;
  unsigned long long *mark = nullptr;
  // the destination's current value (loaded ahead of the decision)
  __device__ __forceinline__ Pre pre(uint32_t v, int q) const {
    return __ldcg(&val[(uint64_t)v * WLANES + q]);
  }
  // is_sssp / is_cc: this lane's algorithm; vu: the lane's value at u.
  __device__ __forceinline__ bool lane(uint32_t u, uint32_t v, uint32_t w, uint32_t vu, int q,
                                       bool is_sssp, bool is_cc) const {
    return fin(u, v, w, vu, q, is_sssp, is_cc, pre(v, q));
  }
  __device__ __forceinline__ bool fin(uint32_t u, uint32_t v, uint32_t w, uint32_t vu, int q,
                                      bool is_sssp, bool is_cc, Pre cur) const {
    uint32_t cand;
    if (is_cc) {
      cand = vu;
    } else {
      if (vu == INF32) return false;
      const uint64_t nd = (uint64_t)vu + (is_sssp ? w : 1u);
      if (nd >= INF32) return false;
      cand = (uint32_t)nd;
    }
    if (cand >= cur) return false;
    const uint64_t idx = (uint64_t)v * WLANES + q;
    return relax_mirror_packed(&val[idx], &st[idx], cand, u);
  }
};

// Parent-tree reset of one lane: a child whose parent is u is reset once
// (CAS on the packed word), the mirror with it; resets are counted per lane.
struct WideInvalidateOp {
  static constexpr bool kNeedsSourceValues = false;
  static constexpr bool kRestrict = false;
  using Pre = unsigned long long;
  unsigned long long *st;
  uint32_t *val;
  WideAlgo algo;
  const unsigned long long *only = nullptr;
  unsigned long long *mark = nullptr;  // per vertex: the lanes reset there (OR-ed in)
  __device__ __forceinline__ Pre pre(uint32_t v, int q) const {
    return __ldcg(&st[(uint64_t)v * WLANES + q]);
  }
  __device__ __forceinline__ bool lane(uint32_t u, uint32_t v, uint32_t w, uint32_t vu, int q,
                                       bool is_sssp, bool is_cc) const {
    return fin(u, v, w, vu, q, is_sssp, is_cc, pre(v, q));
  }
  __device__ __forceinline__ bool fin(uint32_t u, uint32_t v, uint32_t, uint32_t, int q, bool,
                                      bool is_cc, Pre cu) const {
    const uint64_t idx = (uint64_t)v * WLANES + q;
    if ((uint32_t)cu != u) return false;
    const unsigned long long rst = is_cc ? (((unsigned long long)v << 32) | INF32) : ~0ull;
    if (atomicCAS(&st[idx], cu, rst) != cu) return false;
    val[idx] = is_cc ? v : INF32;
    return true;
  }
};

// Load-balanced map for wide ops: CTAs take ranges of 2048-slot units of
// the frontier's edge space (as seg_map / group_map); entries are staged in
// shared memory, then each warp takes 32 consecutive slots per step.  Per
// lane counts: the CTA that holds an entry's first slot adds live[v] for
// every lane of its mask (the traversed-edge count of the frontier);
// lane_changes counts the lanes changed (resets for the invalidation op);
// edge_stat receives the (lane, edge) pairs actually evaluated -- fewer than
// the traversed count when a restricted round skips destinations.
// H = false: every block is in HBM and the host-tier logic is compiled out.
template <class Op, bool H>
__device__ __forceinline__ void wide_map_body(const GraphView &g, FrontierView in, FrontierView out,
                                              const Op &op, const unsigned long long *m_in,
                                              unsigned long long *m_out, const uint32_t *prev_vtx,
                                              const unsigned long long *prev_cnt,
                                              unsigned long long *prev_mask,
                                              unsigned long long *lane_edges,
                                              unsigned long long *lane_changes,
                                              unsigned long long *edge_stat) {
  constexpr int GC = WCHUNK;
  __shared__ uint64_t s_eb[GC + 1];
  __shared__ uint64_t s_off[GC];
  __shared__ unsigned long long s_mask[GC];
  __shared__ uint32_t s_len[GC];
  __shared__ uint32_t s_vtx[GC];
  __shared__ unsigned long long s_lane[WLANES];
  __shared__ unsigned long long s_chg[WLANES];
  clear_prev_masks64(prev_vtx, prev_cnt, prev_mask);
  const int t = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  constexpr int NW = RELAX_THREADS / 32;
  if (threadIdx.x < WLANES) {
    s_lane[threadIdx.x] = 0;
    s_chg[threadIdx.x] = 0;
  }
  const bool sssp0 = op.algo.sssp >> t & 1ull, sssp1 = op.algo.sssp >> (t + 32) & 1ull;
  const bool cc0 = op.algo.cc >> t & 1ull, cc1 = op.algo.cc >> (t + 32) & 1ull;
  unsigned long long acc0 = 0, acc1 = 0, chg0 = 0, chg1 = 0;
  uint32_t evald = 0;  // (lane, edge) pairs evaluated by this thread's lanes
  uint32_t miss_acc = 0;  // host-tier slots this thread read over the link
  __shared__ unsigned long long s_host;  // host-tier slots of the entries this CTA owns
  if (threadIdx.x == 0) s_host = 0;
  __shared__ unsigned long long s_eval;
  if (threadIdx.x == 0) s_eval = 0;
  const uint64_t packed = __ldcg((const unsigned long long *)in.counter);
  const uint32_t n = (uint32_t)(packed >> CNT_SHIFT);
  const uint64_t T = packed & EDGE_MASK;
  const uint64_t nunits = (T + UNIT - 1) / UNIT;
  const uint64_t ub = (uint64_t)blockIdx.x * nunits / gridDim.x;
  const uint64_t ue = (uint64_t)(blockIdx.x + 1) * nunits / gridDim.x;
  __syncthreads();
  if (n != 0 && ub < ue) {
    const uint64_t E0 = ub * UNIT;
    const uint64_t E1 = min(ue * (uint64_t)UNIT, T);
    uint32_t s = __ldcg(&in.ustart[ub]);
    for (;;) {
      __syncthreads();
      for (int h = threadIdx.x; h < GC; h += RELAX_THREADS) {
        const uint32_t idx = s + h;
        const uint64_t eb = idx < n ? __ldcg((const unsigned long long *)&in.ebase[idx]) : T;
        s_eb[h] = eb;
        s_mask[h] = 0ull;
        if (h == 0) {
          const uint32_t j = s + GC;
          s_eb[GC] = j < n ? __ldcg((const unsigned long long *)&in.ebase[j]) : T;
        }
        if (idx < n && eb < E1) {
          const uint32_t v = __ldcg(&in.vtx[idx]);
          s_vtx[h] = v;
          s_len[h] = __ldcg(&in.len[idx]);
          const uint64_t o = g.off[v];
          s_mask[h] = __ldcg(&m_in[v]);
          if (H && (o & HOST_BIT)) {
            if (eb >= E0) {
              hot_bump(g, v, o);
              if (g.cstat) atomicAdd(&s_host, (unsigned long long)s_len[h]);
            }
            s_off[h] = resolve_block(g, o, s_len[h]);
          } else {
            s_off[h] = o;
          }
        }
      }
      __syncthreads();
      // per-lane (query, edge) counts of the entries whose first slot is ours
      for (int h = warp * 32; h < GC; h += RELAX_THREADS) {
        const uint32_t idx = s + h + t;
        const uint64_t eb = s_eb[h + t];
        const bool own = idx < n && eb >= E0 && eb < E1;
        const uint32_t l = own ? g.live[s_vtx[h + t]] : 0u;
        const unsigned long long m = own ? s_mask[h + t] : 0ull;
#pragma unroll 4
        for (int i = 0; i < 32; ++i) {
          const uint32_t li = __shfl_sync(0xFFFFFFFFu, l, i);
          const unsigned long long mi = __shfl_sync(0xFFFFFFFFu, m, i);
          acc0 += (mi >> t & 1ull) ? li : 0u;
          acc1 += (mi >> (t + 32) & 1ull) ? li : 0u;
        }
      }
      const uint64_t lo = max(E0, s_eb[0]);
      const uint64_t hi = min(E1, s_eb[GC]);
      // The work of 32 slots, one per thread: the slot (ok: it holds an edge)
      // of entry le leads to v with weight w, and mk holds the lanes to
      // evaluate on it -- (edge, active lane) pairs.  Dense windows (many
      // lanes per edge) take the per-edge path, every thread on two lanes of
      // each edge; sparse ones -- the common case after the first rounds --
      // spread the pairs over the warp's threads, one pair per thread per
      // step, so no thread idles on an inactive lane.
      auto pairs = [&](bool ok, uint32_t v, uint32_t w, int le, unsigned long long mk) {
        const uint32_t c = (uint32_t)__popcll(mk);
        uint32_t incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
          if (t >= d) incl += y;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        const uint32_t excl = incl - c;
        if (total > 32u * WIDE_DENSE_LANES) {
          bool want = false;
          // two edges per step: their destination rows (and source rows) are
          // all requested before any decision, so a thread keeps 8 loads in
          // flight instead of waiting once per edge
          constexpr int D = 2;
          uint32_t rem = __ballot_sync(0xFFFFFFFFu, ok);
          while (rem) {
            int ii[D], li[D];
            uint32_t vi[D], wi[D], uu[D];
            bool a0[D], a1[D];
#pragma unroll
            for (int q = 0; q < D; ++q) {
              ii[q] = rem ? __ffs(rem) - 1 : -1;
              rem = rem ? rem & (rem - 1) : 0u;
              const int src = ii[q] < 0 ? 0 : ii[q];
              li[q] = __shfl_sync(0xFFFFFFFFu, le, src);
              vi[q] = __shfl_sync(0xFFFFFFFFu, v, src);
              wi[q] = __shfl_sync(0xFFFFFFFFu, w, src);
              uu[q] = s_vtx[li[q]];
              // no edge left for this step (ii < 0): evaluate nothing.  (A
              // repeat of edge 0 here could succeed with no thread to append
              // its destination, and the improvement would never be pushed.)
              unsigned long long mkq = __shfl_sync(0xFFFFFFFFu, mk, src);
              if (ii[q] < 0) mkq = 0ull;
              a0[q] = mkq >> t & 1ull;
              a1[q] = mkq >> (t + 32) & 1ull;
            }
            typename Op::Pre c0[D], c1[D];
            uint32_t vu0[D], vu1[D];
#pragma unroll
            for (int q = 0; q < D; ++q) {
              c0[q] = a0[q] ? op.pre(vi[q], t) : typename Op::Pre(0);
              c1[q] = a1[q] ? op.pre(vi[q], t + 32) : typename Op::Pre(0);
              vu0[q] = INF32;
              vu1[q] = INF32;
              if (Op::kNeedsSourceValues) {
                // read through L2 (not the non-coherent path: this kernel
                // writes the rows, and a persistent launch runs every round
                // in one kernel).  A value that drops after this read is
                // harmless: its vertex is appended and pushes again.
                const uint32_t *row = op.val + (uint64_t)uu[q] * WLANES;
                if (a0[q]) vu0[q] = __ldcg(row + t);
                if (a1[q]) vu1[q] = __ldcg(row + t + 32);
              }
            }
#pragma unroll
            for (int q = 0; q < D; ++q) {
              evald += (uint32_t)a0[q] + (uint32_t)a1[q];
              const bool x0 = a0[q] && op.fin(uu[q], vi[q], wi[q], vu0[q], t, sssp0, cc0, c0[q]);
              const bool x1 = a1[q] && op.fin(uu[q], vi[q], wi[q], vu1[q], t + 32, sssp1, cc1, c1[q]);
              chg0 += x0;
              chg1 += x1;
              const unsigned long long bits = ballot64(x0, x1);
              if (bits && t == ii[q] && op.mark) atomicOr(&op.mark[vi[q]], bits);
              if (bits && t == ii[q] && g.slots[vi[q]])
                want = atomicOr(&m_out[vi[q]], bits) == 0ull;
            }
          }
          frontier_append(out, want, v, want ? g.slots[v] : 0u);
        } else if (total) {
          const uint32_t nonempty = __ballot_sync(0xFFFFFFFFu, c > 0);
          for (uint32_t ib = 0; ib < total; ib += 32) {
            // the pair of this thread: item ib + t belongs to the nonempty
            // edge whose items start last at or before it -- the edge that
            // covers item ib (carry) plus the starts inside this step
            const uint32_t item = ib + t;
            const uint32_t carry = __popc(__ballot_sync(0xFFFFFFFFu, c > 0 && excl <= ib)) - 1u;
            const uint32_t sb = (c > 0 && excl > ib && excl < ib + 32) ? 1u << (excl - ib) : 0u;
            const uint32_t ms = __reduce_or_sync(0xFFFFFFFFu, sb);
            const bool has = item < total;
            const uint32_t rank = carry + __popc(ms & (0xFFFFFFFFu >> (31 - t)));
            const int sl = has ? (int)__fns(nonempty, 0, (int)rank + 1) : 0;
            const uint32_t r = item - __shfl_sync(0xFFFFFFFFu, excl, sl);
            const unsigned long long mj = __shfl_sync(0xFFFFFFFFu, mk, sl);
            const uint32_t vj = __shfl_sync(0xFFFFFFFFu, v, sl);
            const uint32_t wj = __shfl_sync(0xFFFFFFFFu, w, sl);
            const int lej = __shfl_sync(0xFFFFFFFFu, le, sl);
            bool want = false;
            if (has) {
              // lane = the r-th active lane of the edge's source
              const uint32_t m0 = (uint32_t)mj, m1 = (uint32_t)(mj >> 32);
              const uint32_t p0 = __popc(m0);
              const int q = r < p0 ? (int)__fns(m0, 0, (int)r + 1) : 32 + (int)__fns(m1, 0, (int)(r - p0) + 1);
              const uint32_t u = s_vtx[lej];
              uint32_t vu = INF32;
              if (Op::kNeedsSourceValues) vu = __ldcg(op.val + (uint64_t)u * WLANES + q);
              ++evald;
              if (op.lane(u, vj, wj, vu, q, op.algo.sssp >> q & 1ull, op.algo.cc >> q & 1ull)) {
                atomicAdd(&s_chg[q], 1ull);
                if (op.mark) atomicOr(&op.mark[vj], 1ull << q);
                want = g.slots[vj] && atomicOr(&m_out[vj], 1ull << q) == 0ull;
              }
            }
            frontier_append(out, want, vj, want ? g.slots[vj] : 0u);
          }
        }
      };
      if constexpr (Op::kRestrict && !H) {
        // Restricted round (the repair's first), every block in HBM: almost
        // no edge leads into a vertex reset in one of its source's lanes, so
        // the round is a walk of ids and reset-lane probes.  It walks like
        // group_map: each warp its own contiguous share of the chunk, 32
        // quads (128 slots) per window, lane i on quad i (coalesced 512-B id
        // reads), owners from the OR of entry starts, the next window's ids
        // loaded before this window's probes; the four probes of a quad are
        // issued together.  Only a slot whose probe meets a lane of its
        // source takes the pair path above, one slot of the quad at a time.
        const uint64_t nq = hi > lo ? (hi - lo) >> 2 : 0;
        uint64_t wq = (lo >> 2) + nq * (uint64_t)warp / NW;
        const uint64_t wqe = (lo >> 2) + nq * (uint64_t)(warp + 1) / NW;
        if (wq < wqe) {
          int s0;
          {  // owner of the share's first quad
            const uint64_t e = wq << 2;
            int a = 0, b = GC - 1;
            while (a < b) {
              const int m = (a + b + 1) >> 1;
              if (s_eb[m] <= e) a = m;
              else b = m - 1;
            }
            s0 = a;
          }
          // owner and first slot of this thread's quad in the window at
          // quad q (consecutive windows, all threads together); true when the
          // quad holds slots.  Leaves s0 at the next window's first owner.
          auto window = [&](uint64_t q, int &own, uint32_t &j0) -> bool {
            const uint64_t p0 = q << 2, pe = p0 + 4 * 32;
            const int j = s0 + t;
            const uint64_t bj = j <= GC ? s_eb[j] : ~0ull;
            const uint32_t bit = (t >= 1 && bj < pe) ? 1u << (uint32_t)((bj - p0) >> 2) : 0u;
            const uint32_t m = __reduce_or_sync(0xFFFFFFFFu, bit);
            own = s0 + __popc(m & (0xFFFFFFFFu >> (31 - t)));
            int ns = s0 + __popc(m);
            if (ns < GC && s_eb[ns + 1] <= pe) ++ns;  // an entry starting exactly at pe
            s0 = ns;
            j0 = (uint32_t)(p0 + 4 * (uint32_t)t - s_eb[own]);
            return q + (uint64_t)t < wqe && j0 < s_len[own];
          };
          const uint4 none = make_uint4(SGS_TOMB, SGS_TOMB, SGS_TOMB, SGS_TOMB);
          int oc = 0;
          uint32_t jc = 0;
          bool hc = window(wq, oc, jc);
          uint4 ic = hc ? ld_quad_stream(g.adj_d + s_off[oc] + jc) : none;
          for (; wq < wqe; wq += 32) {
            int on = 0;
            uint32_t jn = 0;
            bool hn = false;
            uint4 in4 = none;
            if (wq + 32 < wqe) {
              hn = window(wq + 32, on, jn);
              if (hn) in4 = ld_quad_stream(g.adj_d + s_off[on] + jn);
            }
            const unsigned long long sm = hc ? s_mask[oc] : 0ull;
            const uint32_t ln = hc ? s_len[oc] : 0u;
            uint32_t d[4];
            unsigned long long mk[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              d[k] = quad_at(ic, k);
              const bool okk = jc + k < ln && d[k] != SGS_TOMB;
              mk[k] = okk ? __ldcg(&op.only[d[k]]) : 0ull;
            }
            uint32_t hitm = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              mk[k] &= sm;
              hitm |= (mk[k] != 0ull ? 1u : 0u) << k;
            }
            const uint32_t wh = __reduce_or_sync(0xFFFFFFFFu, hitm);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              if (!(wh >> k & 1u)) continue;
              uint32_t w = 1;
              if (mk[k] & op.algo.sssp)
                w = g.wmode == W_EXPLICIT ? __ldcg(g.wgt_d + s_off[oc] + jc + k)
                    : g.wmode == W_SYNTH  ? (s_vtx[oc] + d[k]) % 128u + 1u
                                          : 1u;
              pairs(mk[k] != 0ull, d[k], w, oc, mk[k]);
            }
            oc = on;
            jc = jn;
            ic = in4;
            hc = hn;
          }
        }
      } else {
        // Windows of 32 slots, lane t on slot t (one coalesced id read), dealt
        // round-robin to the warps so that they share the chunk's heavy and
        // light entries evenly.  A window's first owner s0 comes from one
        // warp-uniform search; the others need none (as in group_map): lane j
        // holds the start of entry s0 + j, every start inside the window sets
        // bit (start - window) of a warp-wide OR, and a slot's owner is s0 plus
        // the set bits at or below it (every entry has at least one slot).
        for (uint64_t wb = lo + (uint64_t)warp * 32; wb < hi; wb += (uint64_t)NW * 32) {
          int le;
          {
            int a = 0, b = GC - 1;
            while (a < b) {
              const int m = (a + b + 1) >> 1;
              if (s_eb[m] <= wb) a = m;
              else b = m - 1;
            }
            const int s0 = a;
            const int j = s0 + t;
            const uint64_t bj = j <= GC ? s_eb[j] : ~0ull;
            const uint32_t bit = (t >= 1 && bj < wb + 32) ? 1u << (uint32_t)(bj - wb) : 0u;
            const uint32_t m = __reduce_or_sync(0xFFFFFFFFu, bit);
            le = s0 + __popc(m & (0xFFFFFFFFu >> (31 - t)));
          }
          const uint64_t e = wb + t;
          bool ok = false;
          uint32_t v = 0, w = 1;
          unsigned long long rl = ~0ull;  // the lanes this edge may relax
          if (e < hi) {
            const int l = le;
            const uint32_t j = (uint32_t)(e - s_eb[l]);
            if (j < s_len[l]) {
              // slot position in its arena: HBM, cache line or host
              uint64_t x = s_off[l] + j;
              int tier = 0;
              if (H && (x & HOST_BIT)) {
                x &= OFF_MASK;
                const uint32_t m = cache_line(g, x);
                tier = m != NO_LINE ? 1 : 2;
                if (m != NO_LINE) x = ((uint64_t)m << CLINE_SHIFT) + (x & (CLINE - 1));
                miss_acc += tier == 2;
              }
              v = __ldcg((tier == 0 ? g.adj_d : tier == 1 ? g.adj_c : g.adj_h) + x);
              ok = v != SGS_TOMB;
              if constexpr (Op::kRestrict) {
                if (ok) rl = __ldcg(&op.only[v]);
                ok = ok && rl != 0ull;
              }
              if (ok && op.algo.sssp && s_mask[l] & op.algo.sssp)
                w = g.wmode == W_EXPLICIT ? __ldcg((tier == 0 ? g.wgt_d : tier == 1 ? g.wgt_c : g.wgt_h) + x)
                    : g.wmode == W_SYNTH  ? (s_vtx[l] + v) % 128u + 1u
                                          : 1u;
            }
          }
          const unsigned long long mk = ok ? s_mask[le] & rl : 0ull;
          pairs(ok, v, w, le, mk);
        }
      }
      if (s_eb[GC] >= E1 || s + GC >= n) break;
      s += GC;
    }
  }
  // per-lane sums (thread t holds lanes t and t + 32): shared, then 64
  // global atomics per CTA
  atomicAdd(&s_lane[t], acc0);
  atomicAdd(&s_lane[t + 32], acc1);
  atomicAdd(&s_chg[t], chg0);
  atomicAdd(&s_chg[t + 32], chg1);
  const unsigned long long ev = warp_sum((unsigned long long)evald);
  if (t == 0 && ev) atomicAdd(&s_eval, ev);
  const unsigned long long miss = warp_sum((unsigned long long)miss_acc);
  if (g.cstat && t == 0 && miss) atomicAdd(&g.cstat[1], miss);
  __syncthreads();
  if (threadIdx.x < WLANES) {
    const unsigned long long x = s_lane[threadIdx.x], c = s_chg[threadIdx.x];
    if (x && lane_edges) atomicAdd(&lane_edges[threadIdx.x], x);
    if (c && lane_changes) atomicAdd(&lane_changes[threadIdx.x], c);
  }
  if (threadIdx.x == 0 && s_eval && edge_stat) atomicAdd(edge_stat, s_eval);
  if (threadIdx.x == 0 && g.cstat && s_host) atomicAdd(&g.cstat[0], s_host);
  __syncthreads();  // shared state is reused when the body runs again
}

template <class Op, bool H>
__global__ void __launch_bounds__(RELAX_THREADS, 3)
    wide_map(GraphView g, FrontierView in, FrontierView out, Op op,
             const unsigned long long *m_in, unsigned long long *m_out, const uint32_t *prev_vtx,
             const unsigned long long *prev_cnt, unsigned long long *prev_mask,
             unsigned long long *lane_edges, unsigned long long *lane_changes,
             unsigned long long *edge_stat) {
  wide_map_body<Op, H>(g, in, out, op, m_in, m_out, prev_vtx, prev_cnt, prev_mask, lane_edges,
                       lane_changes, edge_stat);
}

// Rounds r0, r0+1, ... of a wide phase in one cooperative launch (see
// group_rounds).
template <class Op, bool H>
__global__ void __launch_bounds__(RELAX_THREADS, 3)
    wide_rounds(GraphView g, RoundBufs<unsigned long long> rb, Op op, uint32_t r0, uint32_t max_rounds,
                unsigned long long *lane_edges, unsigned long long *lane_changes,
                unsigned long long *rstat, uint32_t *rounds_out) {
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  uint32_t r = r0;
  bool conv = false;
  for (; r < max_rounds; ++r) {
    const bool hp = r >= 1;
    wide_map_body<Op, H>(g, rb.view(r), rb.view(r + 1), op, rb.mask[r % 3], rb.mask[(r + 1) % 3],
                  hp ? rb.vtx[(r - 1) % 3] : nullptr, hp ? rb.cnt + r - 1 : nullptr,
                  hp ? rb.mask[(r - 1) % 3] : nullptr, lane_edges, lane_changes, rstat + r);
    __threadfence();
    grid.sync();
    if ((__ldcg(rb.cnt + r + 1) >> CNT_SHIFT) == 0) {
      conv = true;
      ++r;
      break;
    }
  }
  if (r >= 1) clear_prev_masks64(rb.vtx[(r - 1) % 3], rb.cnt + r - 1, rb.mask[(r - 1) % 3]);
  if (!conv) clear_prev_masks64(rb.vtx[r % 3], rb.cnt + r, rb.mask[r % 3]);
  if (blockIdx.x == 0 && threadIdx.x == 0) *rounds_out = r;
}

// ---------------------------------------------------------------------------
// Frontier builders and per-lane helpers
// ---------------------------------------------------------------------------

// Summaries of the lanes of a wide group in one pass over its 512-B state
// rows: a warp per vertex, thread t holding lanes t and t+32 across the
// vertices it visits; slot[q] >= 0 selects lane q and its 4 counters at
// out + 4 * slot[q] (reached, sum of values, max value, sum of parents).
struct WideSlots {
  int slot[WLANES];
};
__global__ void __launch_bounds__(RELAX_THREADS)
    k_wide_summary_lanes(const unsigned long long *st, uint32_t nv, WideSlots ws,
                         unsigned long long *out) {
  __shared__ unsigned long long s_acc[WLANES][4];
  for (int i = threadIdx.x; i < WLANES * 4; i += RELAX_THREADS) s_acc[i / 4][i % 4] = 0;
  __syncthreads();
  const int t = threadIdx.x & 31;
  const bool on0 = ws.slot[t] >= 0, on1 = ws.slot[t + 32] >= 0;
  unsigned long long r0 = 0, su0 = 0, m0 = 0, p0 = 0, r1 = 0, su1 = 0, m1 = 0, p1 = 0;
  const uint32_t nwarp = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv; v += nwarp) {
    const unsigned long long *row = st + (uint64_t)v * WLANES;
    if (on0) {
      const unsigned long long x = __ldcs(row + t);
      const uint32_t val = (uint32_t)(x >> 32);
      if (val != INF32) {
        ++r0;
        su0 += val;
        m0 = val > m0 ? val : m0;
        if ((uint32_t)x != INF32) p0 += (uint32_t)x;
      }
    }
    if (on1) {
      const unsigned long long x = __ldcs(row + t + 32);
      const uint32_t val = (uint32_t)(x >> 32);
      if (val != INF32) {
        ++r1;
        su1 += val;
        m1 = val > m1 ? val : m1;
        if ((uint32_t)x != INF32) p1 += (uint32_t)x;
      }
    }
  }
  if (on0) {
    atomicAdd(&s_acc[t][0], r0);
    atomicAdd(&s_acc[t][1], su0);
    atomicMax(&s_acc[t][2], m0);
    atomicAdd(&s_acc[t][3], p0);
  }
  if (on1) {
    atomicAdd(&s_acc[t + 32][0], r1);
    atomicAdd(&s_acc[t + 32][1], su1);
    atomicMax(&s_acc[t + 32][2], m1);
    atomicAdd(&s_acc[t + 32][3], p1);
  }
  __syncthreads();
  if (threadIdx.x < WLANES && ws.slot[threadIdx.x] >= 0) {
    unsigned long long *o = out + 4 * ws.slot[threadIdx.x];
    const unsigned long long *a = s_acc[threadIdx.x];
    if (a[0]) atomicAdd(&o[0], a[0]);
    if (a[1]) atomicAdd(&o[1], a[1]);
    atomicMax(&o[2], a[2]);
    if (a[3]) atomicAdd(&o[3], a[3]);
  }
}

// Initial state of the lanes in `lanes` on every vertex: CC lanes v's own id,
// the others unreached; one warp per vertex row.
__global__ void k_wide_init_lanes(unsigned long long *st, uint32_t *val, uint32_t nv,
                                  unsigned long long lanes, unsigned long long cc) {
  const int t = threadIdx.x & 31;
  const uint32_t nwarp = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv; v += nwarp) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = t + 32 * h;
      if (!(lanes >> q & 1ull)) continue;
      const bool c = cc >> q & 1ull;
      const uint64_t idx = (uint64_t)v * WLANES + q;
      st[idx] = c ? (((unsigned long long)v << 32) | INF32) : ~0ull;
      val[idx] = c ? v : INF32;
    }
  }
}

// Sources of new BFS/SSSP lanes: value 0 at the source, mask bit set, the
// source appended once.  One thread per new lane.
__global__ void k_wide_seed_sources(GraphView g, unsigned long long *st, uint32_t *val,
                                    const uint32_t *src, const uint32_t *lane, uint32_t n,
                                    unsigned long long *m_out, FrontierView out) {
  for (uint32_t b = blockIdx.x * blockDim.x; b < n; b += gridDim.x * blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    bool want = false;
    uint32_t v = 0, d = 0;
    if (i < n) {
      v = src[i];
      const uint32_t q = lane[i];
      const uint64_t idx = (uint64_t)v * WLANES + q;
      st[idx] = (unsigned long long)INF32;  // value 0, no parent
      val[idx] = 0u;
      d = g.slots[v];
      want = d && atomicOr(&m_out[v], 1ull << q) == 0ull;
    }
    frontier_append(out, want, v, d);
  }
}

// Every vertex with a non-empty block; mask = lanes of `lanes` whose value is
// finite there (CC lanes always).  A warp reads 32 rows, one per step, and
// appends the 32 vertices together.  With `only_if_reset`, nothing unless a
// lane of `lanes` was reset by the last invalidation.
__global__ void k_wide_dense(GraphView g, const uint32_t *val, unsigned long long lanes,
                             unsigned long long cc, unsigned long long *m_out, FrontierView out,
                             const unsigned long long *only_if_reset = nullptr) {
  if (only_if_reset && !block_any_lane(only_if_reset, lanes)) return;
  const int t = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const bool l0 = lanes >> t & 1ull, l1 = lanes >> (t + 32) & 1ull;
  const bool c0 = cc >> t & 1ull, c1 = cc >> (t + 32) & 1ull;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < g.nv; b += stride) {
    const uint64_t base = b + (threadIdx.x & ~31u);
    const uint32_t myv = (uint32_t)(base + t);
    const uint32_t myd = myv < g.nv ? g.slots[myv] : 0u;
    bool want = false;
    uint32_t dm = __ballot_sync(0xFFFFFFFFu, myd != 0u);
    for (; dm; dm &= dm - 1) {
      const int i = __ffs(dm) - 1;
      const uint32_t v = (uint32_t)(base + i);
      const uint32_t *row = val + (uint64_t)v * WLANES;
      const bool f0 = l0 && (c0 || __ldcg(row + t) != INF32);
      const bool f1 = l1 && (c1 || __ldcg(row + t + 32) != INF32);
      const unsigned long long m = ballot64(f0, f1);
      if (t == i && m) {
        m_out[v] = m;
        want = true;
      }
    }
    frontier_append_block(out, want, myv, want ? myd : 0u);
  }
}

// Deletion seeds: deleted (u,v) whose lane-q parent of v is u reset lane q.
// A warp handles 32 deleted edges, one per step.
__global__ void k_wide_seed_deleted(GraphView g, unsigned long long *st, uint32_t *val,
                                    unsigned long long lanes, unsigned long long cc,
                                    const uint64_t *keys, uint32_t n, unsigned long long *inval,
                                    unsigned long long *mark, unsigned long long *m_out, FrontierView out) {
  const int t = threadIdx.x & 31;
  const bool l0 = lanes >> t & 1ull, l1 = lanes >> (t + 32) & 1ull;
  const bool c0 = cc >> t & 1ull, c1 = cc >> (t + 32) & 1ull;
  WideInvalidateOp op{st, val, WideAlgo{0, cc}};
  unsigned long long r0 = 0, r1 = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t base = b + (threadIdx.x & ~31u);
    const uint64_t mi = base + t;
    const uint64_t key = mi < n ? keys[mi] : 0ull;
    bool want = false;
    uint32_t okm = __ballot_sync(0xFFFFFFFFu, mi < n);
    for (; okm; okm &= okm - 1) {
      const int i = __ffs(okm) - 1;
      const uint64_t k = __shfl_sync(0xFFFFFFFFu, (unsigned long long)key, i);
      const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
      const bool x0 = l0 && op.lane(u, v, 0, 0, t, false, c0);
      const bool x1 = l1 && op.lane(u, v, 0, 0, t + 32, false, c1);
      r0 += x0;
      r1 += x1;
      const unsigned long long bits = ballot64(x0, x1);
      if (bits && t == i) atomicOr(&mark[v], bits);
      if (bits && t == i && g.slots[v]) want = atomicOr(&m_out[v], bits) == 0ull;
    }
    const uint32_t v = (uint32_t)key;
    frontier_append(out, want, v, want ? g.slots[v] : 0u);
  }
  if (r0) atomicAdd(&inval[t], r0);
  if (r1) atomicAdd(&inval[t + 32], r1);
}

// Insert-only fast path: relax just the kept inserted edges in the lanes of
// `lanes`; each inserted edge counts once per lane.
__global__ void k_wide_relax_inserted(GraphView g, unsigned long long *st, uint32_t *val,
                                      unsigned long long lanes, WideAlgo algo,
                                      const uint64_t *keys, const uint32_t *w,
                                      const uint32_t *n_ptr, unsigned long long *m_out,
                                      FrontierView out, unsigned long long *lane_edges) {
  const uint32_t n = *n_ptr;
  const int t = threadIdx.x & 31;
  const bool l0 = lanes >> t & 1ull, l1 = lanes >> (t + 32) & 1ull;
  const bool s0 = algo.sssp >> t & 1ull, s1 = algo.sssp >> (t + 32) & 1ull;
  const bool c0 = algo.cc >> t & 1ull, c1 = algo.cc >> (t + 32) & 1ull;
  WideRelaxOp<> op{st, val, algo};
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t counted = 0;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t base = b + (threadIdx.x & ~31u);
    const uint64_t mi = base + t;
    const uint64_t key = mi < n ? keys[mi] : 0ull;
    uint32_t wt = 1u;
    if (mi < n) {
      const uint32_t u = (uint32_t)(key >> 32), v = (uint32_t)key;
      wt = g.wmode == W_EXPLICIT ? w[mi] : g.wmode == W_SYNTH ? (u + v) % 128u + 1u : 1u;
      ++counted;
    }
    bool want = false;
    uint32_t okm = __ballot_sync(0xFFFFFFFFu, mi < n);
    for (; okm; okm &= okm - 1) {
      const int i = __ffs(okm) - 1;
      const uint64_t k = __shfl_sync(0xFFFFFFFFu, (unsigned long long)key, i);
      const uint32_t wi = __shfl_sync(0xFFFFFFFFu, wt, i);
      const uint32_t u = (uint32_t)(k >> 32), v = (uint32_t)k;
      const uint32_t *row = val + (uint64_t)u * WLANES;
      const uint32_t vu0 = l0 ? __ldcg(row + t) : INF32;
      const uint32_t vu1 = l1 ? __ldcg(row + t + 32) : INF32;
      const bool x0 = l0 && op.lane(u, v, wi, vu0, t, s0, c0);
      const bool x1 = l1 && op.lane(u, v, wi, vu1, t + 32, s1, c1);
      const unsigned long long bits = ballot64(x0, x1);
      if (bits && t == i && g.slots[v]) want = atomicOr(&m_out[v], bits) == 0ull;
    }
    const uint32_t v = (uint32_t)key;
    frontier_append(out, want, v, want ? g.slots[v] : 0u);
  }
  const uint32_t c = warp_sum(counted);
  if (t == 0 && c) {
    for (int q = 0; q < WLANES; ++q)
      if (lanes >> q & 1ull) atomicAdd(&lane_edges[q], (unsigned long long)c);
  }
}

__global__ void k_clear_masks64(const uint32_t *vtx, const unsigned long long *cnt,
                                unsigned long long *mask) {
  clear_prev_masks64(vtx, cnt, mask);
}

}  // namespace sgs
