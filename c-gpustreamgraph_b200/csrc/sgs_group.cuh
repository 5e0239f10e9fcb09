// sgs_group.cuh -- query groups: up to GMAX integer queries (BFS / SSSP / CC,
// any sources) relaxed together over one edge stream.
//
// Layout: st[v * S + lane] u64 packed (value << 32 | parent), S = 1, 2 or 4,
// so one vertex's states share one 32-B sector and a random access to a
// destination serves every lane.  Lane masks mask[k][v] (u32, three rotating
// buffers) record which lanes improved v in a round; the thread whose
// atomicOr turns the mask non-zero appends v, which replaces per-query
// de-duplication stamps.  Round r reads mask[r%3], writes mask[(r+1)%3] and
// clears the masks of frontier r-1 in mask[(r+2)%3], which round r+1 writes
// next; frontier buffers rotate the same way, so no grid barrier is needed.
//
// Reference semantics per lane are those of the single-query ops
// (hybrid_sssp.cu:97-118 min relaxation, hybrid_cc.cu:96-110 label
// propagation, reset_del_edges / SyncPushDDB_del parent-tree invalidation,
// driver.cuh:398-430 and :1985-2031).
#pragma once
#include <cooperative_groups.h>

#include "sgs_device.cuh"
#include "sgs_segmap.cuh"

namespace sgs {

constexpr int GMAX = 4;
constexpr int GCHUNK = 512;  // entries staged per chunk by group_map

struct LaneAlgo {
  uint32_t packed;  // 8 bits per lane: A_BFS / A_SSSP / A_CC
  // the same as lane bit masks (bit q = lane q), so a relaxation picks a
  // lane's step from kernel-parameter constants instead of decoding `packed`:
  // candidate = source value + (w: the edge weight, inc: 1, cc: 0)
  uint32_t cc, w, inc;
  __device__ __forceinline__ int at(int q) const { return (packed >> (8 * q)) & 0xFF; }
  static LaneAlgo of(uint32_t packed) {
    LaneAlgo a{packed, 0, 0, 0};
    for (int q = 0; q < 4; ++q) {
      const uint32_t k = (packed >> (8 * q)) & 0xFF;
      if (k == A_CC) a.cc |= 1u << q;
      else if (k == A_SSSP) a.w |= 1u << q;
      else a.inc |= 1u << q;
    }
    return a;
  }
};

template <int S>
struct GPay {
  uint64_t off;
  uint32_t mask;
  uint32_t val[S];
};

// S u32 values of vertex v (one 16-B load for S = 4).
template <int S>
__device__ __forceinline__ void load_vals(const uint32_t *val, uint32_t v, uint32_t (&o)[S]) {
  if constexpr (S == 4) {
    const uint4 x = __ldcg(reinterpret_cast<const uint4 *>(val + (uint64_t)v * 4));
    o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = x.w;
  } else if constexpr (S == 2) {
    const uint2 x = __ldcg(reinterpret_cast<const uint2 *>(val + (uint64_t)v * 2));
    o[0] = x.x; o[1] = x.y;
  } else {
    o[0] = __ldcg(val + v);
  }
}

// Clears the masks of the previous frontier (grid-stride, all threads).
__device__ __forceinline__ void clear_prev_masks(const uint32_t *vtx, const unsigned long long *cnt,
                                                 uint32_t *mask) {
  if (!cnt) return;
  const uint32_t n = (uint32_t)(__ldcg(cnt) >> CNT_SHIFT);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    mask[__ldcg(&vtx[i])] = 0;
}

// Relaxation of every active lane of every source over its out-edges.  The
// u32 mirror `val` filters candidates with one 16-B read per destination; a
// candidate below it lowers the mirror first and, if that strictly lowered
// it, the packed (value,parent) word (relax_mirror_packed: equal candidates
// never swap a parent).
//
// Per entry the payload holds each lane's candidate base -- the source's
// value, plus 1 in BFS lanes -- and INF32 in the lanes that do not push, so
// the per-edge test is compare-only: candidate = base (+ the weight in SSSP
// lanes, saturating at INF32) against the destination's mirror.  Most edges
// of a sweep improve nothing; only the quads with some candidate below the
// mirror take the atomic path.
template <int S>
struct RPay {
  uint64_t off;
  uint32_t mask;     // lanes that push from this vertex
  uint32_t base[S];  // candidate base per lane (INF32: the lane does not push)
};

template <int S>
struct GroupRelaxOp {
  using Payload = RPay<S>;
  GraphView g;
  unsigned long long *st;
  uint32_t *val;
  const uint32_t *m_in;
  uint32_t *m_out;
  LaneAlgo algo;
  uint32_t any_w;  // some lane reads stored weights
  __device__ __forceinline__ Payload load(uint32_t v) const {
    Payload p;
    p.off = g.off[v];
    p.mask = __ldcg(&m_in[v]);
    uint32_t x[S];
    load_vals<S>(val, v, x);
    // a BFS/SSSP lane that has not reached v pushes nothing: drop it here,
    // once per entry, instead of testing it for every edge.  A reached BFS
    // value is below INF32, so value + 1 does not wrap.
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const bool on = (p.mask >> q & 1u) && (x[q] != INF32 || (algo.cc >> q & 1u));
      if (!on) p.mask &= ~(1u << q);
      p.base[q] = on ? x[q] + (algo.inc >> q & 1u) : INF32;
    }
    return p;
  }
  // The quad's ids (and weights), loaded one step ahead by group_map.
  struct Quad {
    uint4 ids, ws;
  };
  // slots of an appended vertex (its range in the next frontier)
  __device__ __forceinline__ uint32_t append_len(uint32_t v) const { return g.slots[v]; }
  // H: the graph has a host tier (blocks may be host-resident or cached)
  template <bool H>
  __device__ __forceinline__ Quad fetch(const Payload &p, uint32_t j0) const {
    Quad q;
    if constexpr (H) {
      q.ids = ld_quad_stream(adj_at(g, p.off, j0));
      q.ws = any_w ? ld_quad_stream(wgt_at(g, p.off, j0)) : make_uint4(1, 1, 1, 1);
    } else {
      q.ids = ld_quad_stream(g.adj_d + p.off + j0);
      q.ws = any_w ? ld_quad_stream(g.wgt_d + p.off + j0) : make_uint4(1, 1, 1, 1);
    }
    return q;
  }
  // candidate of lane q for an edge of weight w: base + w in SSSP lanes,
  // saturating (min(base, INF32 - w) + w), else base; INF32 is never below
  // a mirror value
  __device__ __forceinline__ uint32_t cand_of(uint32_t base, uint32_t w, int q) const {
    const uint32_t wq = w & (0u - (algo.w >> q & 1u));
    return min(base, ~wq) + wq;
  }
  __device__ __forceinline__ uint32_t weight_of(const uint4 &ws, int k, uint32_t u, uint32_t d) const {
    return g.wmode == W_EXPLICIT ? quad_at(ws, k) : g.wmode == W_SYNTH ? (u + d) % 128u + 1u : 1u;
  }
  // Returns a 4-bit mask of destinations to append; dst[] holds them.
  __device__ __forceinline__ uint32_t visit4(uint32_t u, const Payload &pr, uint32_t j0, uint32_t len,
                                             const Quad &qd, uint32_t (&dst)[4]) const {
    const uint4 ids = qd.ids;
    const uint4 ws = qd.ws;
    uint32_t okm = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      dst[k] = quad_at(ids, k);
      if (j0 + k < len && dst[k] != SGS_TOMB) okm |= 1u << k;
    }
    uint32_t cur[4][S];
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (okm >> k & 1u) load_vals<S>(val, dst[k], cur[k]);
    // compare-only pass: bit 4k+q = lane q's candidate is below the mirror
    // of destination k
    uint32_t lt = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!(okm >> k & 1u)) continue;
      const uint32_t w = weight_of(ws, k, u, dst[k]);
#pragma unroll
      for (int q = 0; q < S; ++q)
        lt |= (cand_of(pr.base[q], w, q) < cur[k][q] ? 1u : 0u) << (4 * k + q);
    }
    if (!lt) return 0;
    uint32_t app = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t lk = lt >> (4 * k) & 0xFu;
      if (!lk) continue;
      const uint32_t w = weight_of(ws, k, u, dst[k]);
      uint32_t bits = 0;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        if (!(lk >> q & 1u)) continue;
        const uint64_t idx = (uint64_t)dst[k] * S + q;
        if (relax_mirror_packed(&val[idx], &st[idx], cand_of(pr.base[q], w, q), u)) bits |= 1u << q;
      }
      if (bits && g.slots[dst[k]] && atomicOr(&m_out[dst[k]], bits) == 0u) app |= 1u << k;
    }
    return app;
  }
};

// Parent-tree invalidation per lane: a child whose lane-q parent is u (and u
// was reset in lane q) is reset exactly once (CAS on the packed word); the
// mirror is reset with it.
template <int S>
struct GroupInvalidateOp {
  struct Payload {
    uint64_t off;
    uint32_t mask;
    uint32_t pad;
  };
  GraphView g;
  unsigned long long *st;
  uint32_t *val;
  const uint32_t *m_in;
  uint32_t *m_out;
  LaneAlgo algo;
  unsigned long long *inval;  // [GMAX] per-lane reset counts
  uint32_t *mark;             // bitmap of reset vertices (may be null)
  __device__ __forceinline__ Payload load(uint32_t v) const {
    Payload p;
    p.off = g.off[v];
    p.mask = __ldcg(&m_in[v]);
    p.pad = 0;
    return p;
  }
  struct Quad {
    uint4 ids;
  };
  __device__ __forceinline__ uint32_t append_len(uint32_t v) const { return g.slots[v]; }
  template <bool H>
  __device__ __forceinline__ Quad fetch(const Payload &p, uint32_t j0) const {
    if constexpr (H) return Quad{ld_quad_stream(adj_at(g, p.off, j0))};
    else return Quad{ld_quad_stream(g.adj_d + p.off + j0)};
  }
  __device__ __forceinline__ uint32_t visit4(uint32_t u, const Payload &p, uint32_t j0, uint32_t len,
                                             const Quad &qd, uint32_t (&dst)[4]) const {
    const uint4 ids = qd.ids;
    uint32_t okm = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      dst[k] = quad_at(ids, k);
      if (j0 + k < len && dst[k] != SGS_TOMB) okm |= 1u << k;
    }
    uint32_t app = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!(okm >> k & 1u)) continue;
      uint32_t bits = 0;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        if (!(p.mask >> q & 1u)) continue;
        const uint64_t idx = (uint64_t)dst[k] * S + q;
        const unsigned long long cu = __ldcg(&st[idx]);
        if ((uint32_t)cu != u) continue;
        const bool cc = algo.at(q) == A_CC;
        const unsigned long long rst = cc ? (((unsigned long long)dst[k] << 32) | INF32) : ~0ull;
        if (atomicCAS(&st[idx], cu, rst) == cu) {
          val[idx] = cc ? dst[k] : INF32;
          bits |= 1u << q;
          atomicAdd(&inval[q], 1ull);
        }
      }
      if (bits && mark) bit_set(mark, dst[k]);
      if (bits && g.slots[dst[k]] && atomicOr(&m_out[dst[k]], bits) == 0u) app |= 1u << k;
    }
    return app;
  }
};

// Load-balanced map for group ops (same unit/chunk scheme as seg_map).
// Edges are attributed per entry: the CTA whose range holds an entry's first
// position adds live[v] for every lane of its mask, which counts exactly the
// (query, edge) pairs relaxed.  The kernel also clears the previous
// frontier's masks.
#ifndef SGS_GROUP_MIN_BLOCKS
#define SGS_GROUP_MIN_BLOCKS 4  // resident CTAs per SM the register budget allows
#endif
// H = false when every block is in HBM (no host tier): the host-tier logic
// (hotness, cache lookups, link accounting) is compiled out.
template <class Op, bool H>
__device__ __forceinline__ void group_map_body(FrontierView in, FrontierView out, const Op &op,
                                               const uint32_t *prev_vtx,
                                               const unsigned long long *prev_cnt, uint32_t *prev_mask,
                                               unsigned long long *lane_edges,
                                               unsigned long long *edge_stat,
                                               unsigned long long *host_stat) {
  using P = typename Op::Payload;
  constexpr int GC = GCHUNK;
  __shared__ uint64_t s_eb[GC + 1];
  __shared__ uint32_t s_len[GC];
  __shared__ P s_pay[GC];
  __shared__ uint32_t s_vtx[GC];
  __shared__ unsigned long long s_lane[GMAX];
  __shared__ unsigned long long s_host, s_all;  // host-tier slots read over the link / owned
  clear_prev_masks(prev_vtx, prev_cnt, prev_mask);
  if (threadIdx.x < GMAX) s_lane[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_host = s_all = 0;
  uint32_t host_acc = 0;
  const uint64_t packed = __ldcg((const unsigned long long *)in.counter);
  const uint32_t n = (uint32_t)(packed >> CNT_SHIFT);
  const uint64_t T = packed & EDGE_MASK;
  const uint64_t nunits = (T + UNIT - 1) / UNIT;
  const uint64_t ub = (uint64_t)blockIdx.x * nunits / gridDim.x;
  const uint64_t ue = (uint64_t)(blockIdx.x + 1) * nunits / gridDim.x;
  if (n != 0 && ub < ue) {
    const uint64_t E0 = ub * UNIT;
    const uint64_t E1 = min(ue * (uint64_t)UNIT, T);
    uint32_t s = __ldcg(&in.ustart[ub]);
    for (;;) {
      __syncthreads();
      bool host = false;  // this thread staged a host-tier entry
      uint32_t lane_acc[GMAX] = {0, 0, 0, 0};  // (query, edge) pairs of owned entries
#pragma unroll
      for (int h = 0; h < GC / RELAX_THREADS; ++h) {
        const uint32_t t = threadIdx.x + h * RELAX_THREADS;
        const uint32_t idx = s + t;
        const uint64_t eb = idx < n ? __ldcg((const unsigned long long *)&in.ebase[idx]) : T;
        s_eb[t] = eb;
        if (t == 0) {
          const uint32_t j = s + GC;
          s_eb[GC] = j < n ? __ldcg((const unsigned long long *)&in.ebase[j]) : T;
        }
        if (idx < n && eb < E1) {
          const uint32_t v = __ldcg(&in.vtx[idx]);
          s_vtx[t] = v;
          s_len[t] = __ldcg(&in.len[idx]);
          P pay = op.load(v);
          if constexpr (H) {
            if (pay.off & HOST_BIT) {
              host = true;
              if (eb >= E0) {
                hot_bump(op.g, v, pay.off);
                if (op.g.cstat) atomicAdd(&s_all, (unsigned long long)s_len[t]);
              }
              pay.off = resolve_block(op.g, pay.off, s_len[t]);
            }
          }
          s_pay[t] = pay;
          if (eb >= E0 && pay.mask) {
            const uint32_t l = op.g.live[v];
#pragma unroll
            for (int q = 0; q < GMAX; ++q) lane_acc[q] += (pay.mask >> q & 1u) ? l : 0u;
          }
        }
      }
      // the chunk's pair counts go to shared memory now, so no register
      // holds them through the walk
#pragma unroll
      for (int q = 0; q < GMAX; ++q) {
        const uint32_t x = warp_sum(lane_acc[q]);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(&s_lane[q], (unsigned long long)x);
      }
      // the barrier also tells every thread whether the chunk holds
      // host-tier entries (only then does the walk account host reads)
      bool chunk_host = false;
      if constexpr (H) chunk_host = __syncthreads_or(host) != 0;
      else __syncthreads();
      const uint64_t lo = max(E0, s_eb[0]);
      const uint64_t hi = min(E1, s_eb[GC]);
      // Each warp walks its own contiguous share of the chunk's positions,
      // one window of 32 quads (128 slots) per step, lane i on quad i of the
      // window (coalesced 512-B id reads).  Owners need no search: lane j
      // holds the start of entry s0 + j (s0 = owner of the window's first
      // quad), every start inside the window sets bit (start - window) / 4
      // of a warp-wide OR, and a lane's owner is s0 plus the set bits at or
      // below its quad.  This relies on every frontier entry having at least
      // one slot (every append site checks it), so a window meets at most 32
      // entries and no two starts share a bit.  The same bits give the next
      // window's first owner.  Software pipeline: the next window's owners
      // and id loads are issued before the current window's state reads.
      constexpr uint32_t NW = RELAX_THREADS / 32;
      const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      const uint64_t nq = hi > lo ? (hi - lo) >> 2 : 0;
      uint64_t wq = (lo >> 2) + nq * wid / NW;  // this warp's share [wq, wqe) in quads
      const uint64_t wqe = (lo >> 2) + nq * (wid + 1) / NW;
      if (wq < wqe) {
        int s0;
        {  // owner of the share's first quad: one warp-uniform search per chunk
          const uint64_t e = wq << 2;
          int a = 0, b = GC - 1;
          while (a < b) {
            const int m = (a + b + 1) >> 1;
            if (s_eb[m] <= e) a = m;
            else b = m - 1;
          }
          s0 = a;
        }
        // Owner and first slot of this lane's quad in the window at quad q
        // (called for consecutive windows, all lanes together); true when
        // the quad holds slots.  Leaves s0 at the next window's first owner.
        auto window = [&](uint64_t q, int &own, uint32_t &j0) -> bool {
          const uint64_t p0 = q << 2, pe = p0 + 4 * 32;
          const int j = s0 + (int)lane;
          const uint64_t bj = j <= GC ? s_eb[j] : ~0ull;
          const uint32_t bit = (lane >= 1 && bj < pe) ? 1u << (uint32_t)((bj - p0) >> 2) : 0u;
          const uint32_t m = __reduce_or_sync(0xFFFFFFFFu, bit);
          own = s0 + __popc(m & (0xFFFFFFFFu >> (31 - lane)));
          int ns = s0 + __popc(m);
          if (ns < GC && s_eb[ns + 1] <= pe) ++ns;  // an entry starting exactly at pe
          s0 = ns;
          j0 = (uint32_t)(p0 + 4 * lane - s_eb[own]);
          return q + lane < wqe && j0 < s_len[own];
        };
        int oc = 0;
        uint32_t jc = 0;
        typename Op::Quad qc{};
        bool hc = window(wq, oc, jc);
        if (hc) qc = op.template fetch<H>(s_pay[oc], jc);
        for (; wq < wqe; wq += 32) {
          int on = 0;
          uint32_t jn = 0;
          typename Op::Quad qn{};
          bool hn = false;
          if (wq + 32 < wqe) {
            hn = window(wq + 32, on, jn);
            if (hn) qn = op.template fetch<H>(s_pay[on], jn);
          }
          uint32_t app = 0;
          uint32_t dst[4] = {0, 0, 0, 0};
          if (hc) {
            app = op.visit4(s_vtx[oc], s_pay[oc], jc, s_len[oc], qc, dst);
            if (H && chunk_host) {
              const uint64_t o = s_pay[oc].off;
              if ((o & HOST_BIT) && cache_line(op.g, (o & OFF_MASK) + jc) == NO_LINE)
                host_acc += min(4u, s_len[oc] - jc);
            }
          }
          oc = on;
          jc = jn;
          qc = qn;
          hc = hn;
          if (__ballot_sync(0xFFFFFFFFu, app != 0u)) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const bool w = app >> k & 1u;
              frontier_append(out, w, dst[k], w ? op.append_len(dst[k]) : 0u);
            }
          }
        }
      }
      if (s_eb[GC] >= E1 || s + GC >= n) break;
      s += GC;
    }
  }
  const unsigned long long hs = warp_sum((unsigned long long)host_acc);
  if ((threadIdx.x & 31) == 0 && hs) atomicAdd(&s_host, hs);
  __syncthreads();
  if (threadIdx.x < GMAX && s_lane[threadIdx.x]) {
    if (lane_edges) atomicAdd(&lane_edges[threadIdx.x], s_lane[threadIdx.x]);
    if (edge_stat) atomicAdd(edge_stat, s_lane[threadIdx.x]);
  }
  if (threadIdx.x == 0 && s_host && host_stat) atomicAdd(host_stat, s_host);
  if (threadIdx.x == 0 && op.g.cstat) {
    if (s_all) atomicAdd(&op.g.cstat[0], s_all);
    if (s_host) atomicAdd(&op.g.cstat[1], s_host);
  }
  __syncthreads();  // shared state is reused when the body runs again
}

template <class Op, bool H>
__global__ void __launch_bounds__(RELAX_THREADS, SGS_GROUP_MIN_BLOCKS)
    group_map(FrontierView in, FrontierView out, Op op, const uint32_t *prev_vtx,
              const unsigned long long *prev_cnt, uint32_t *prev_mask,
              unsigned long long *lane_edges, unsigned long long *edge_stat,
              unsigned long long *host_stat) {
  group_map_body<Op, H>(in, out, op, prev_vtx, prev_cnt, prev_mask, lane_edges, edge_stat, host_stat);
}

// The three rotating frontier buffers, their counters and lane masks, as one
// persistent launch sees them: round r reads buffer r % 3 / cnt[r] and masks
// r % 3, and writes buffer (r+1) % 3 / cnt[r+1].
template <class M>
struct RoundBufs {
  uint32_t *vtx[3];
  uint32_t *len[3];
  uint64_t *ebase[3];
  uint32_t *ustart[3];
  unsigned long long *cnt;
  M *mask[3];
  uint32_t ucap;
  __device__ __forceinline__ FrontierView view(uint32_t r) const {
    FrontierView f;
    f.vtx = vtx[r % 3];
    f.len = len[r % 3];
    f.ebase = ebase[r % 3];
    f.ustart = ustart[r % 3];
    f.counter = (uint64_t *)(cnt + r);
    f.ucap = ucap;
    return f;
  }
};

// Rounds r0, r0+1, ... of a phase in one cooperative launch: round r, a
// grid-wide barrier (cooperative_groups grid sync; the cooperative launch
// makes every block resident), then the next round unless round r appended
// nothing.  The masks of the last non-empty frontier are cleared before the
// kernel returns; *rounds_out = the first empty frontier's index (or
// max_rounds when the limit is hit).
template <class Op, bool H>
__global__ void __launch_bounds__(RELAX_THREADS, SGS_GROUP_MIN_BLOCKS)
    group_rounds(RoundBufs<uint32_t> rb, Op op, uint32_t r0, uint32_t max_rounds,
                 unsigned long long *lane_edges, unsigned long long *rstat, unsigned long long *hstat,
                 uint32_t *rounds_out) {
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  uint32_t r = r0;
  bool conv = false;
  for (; r < max_rounds; ++r) {
    Op o = op;
    o.m_in = rb.mask[r % 3];
    o.m_out = rb.mask[(r + 1) % 3];
    const bool hp = r >= 1;
    group_map_body<Op, H>(rb.view(r), rb.view(r + 1), o, hp ? rb.vtx[(r - 1) % 3] : nullptr,
                   hp ? rb.cnt + r - 1 : nullptr, hp ? rb.mask[(r - 1) % 3] : nullptr, lane_edges,
                   rstat + r, hstat + r);
    __threadfence();
    grid.sync();
    if ((__ldcg(rb.cnt + r + 1) >> CNT_SHIFT) == 0) {
      conv = true;
      ++r;
      break;
    }
  }
  // r: the first empty frontier (converged) or max_rounds
  if (r >= 1) clear_prev_masks(rb.vtx[(r - 1) % 3], rb.cnt + r - 1, rb.mask[(r - 1) % 3]);
  if (!conv) clear_prev_masks(rb.vtx[r % 3], rb.cnt + r, rb.mask[r % 3]);
  if (blockIdx.x == 0 && threadIdx.x == 0) *rounds_out = r;
}

// ---------------------------------------------------------------------------
// Group frontier builders
// ---------------------------------------------------------------------------
template <int S>
__global__ void k_group_init_lane(unsigned long long *st, uint32_t *val, uint32_t nv, int lane,
                                  int algo, uint32_t source) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    unsigned long long s;
    if (algo == A_CC) s = (v << 32) | INF32;
    else s = v == source ? (unsigned long long)INF32 : ~0ull;
    st[v * S + lane] = s;
    val[v * S + lane] = (uint32_t)(s >> 32);
  }
}

// Every vertex with a non-empty block; mask = selected lanes whose value is
// finite there (CC lanes always).  One writer per vertex: plain stores.
// With `only_if_reset`, the launch does nothing unless a selected lane was
// reset by the last invalidation (its per-lane counts).
template <int S>
__global__ void k_group_dense(GraphView g, const uint32_t *val, uint32_t lanes,
                              LaneAlgo algo, uint32_t *m_out, FrontierView out,
                              const unsigned long long *only_if_reset = nullptr) {
  if (only_if_reset && !block_any_lane(only_if_reset, lanes)) return;
  // eight consecutive vertices per thread, one block append per 2048
  constexpr int N = 8;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * N;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x * N; b < g.nv; b += stride) {
    const uint64_t v0 = b + (uint64_t)threadIdx.x * N;
    bool want[N];
    uint32_t d[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const uint64_t v = v0 + i;
      want[i] = false;
      d[i] = 0;
      if (v < g.nv) {
        d[i] = g.slots[v];
        if (d[i]) {
          uint32_t blk[S];
          load_vals<S>(val, (uint32_t)v, blk);
          uint32_t m = 0;
#pragma unroll
          for (int q = 0; q < S; ++q)
            if ((lanes >> q & 1u) && (algo.at(q) == A_CC || blk[q] != INF32)) m |= 1u << q;
          if (m) {
            m_out[v] = m;
            want[i] = true;
          }
        }
      }
    }
    frontier_append_block_n<N>(out, want, (uint32_t)v0, d);
  }
}

// One vertex, given lanes (the source of new BFS/SSSP lanes).
__global__ void k_group_seed_one(GraphView g, uint32_t v, uint32_t bits, uint32_t *m_out,
                                 FrontierView out) {
  if (threadIdx.x >= 32) return;
  const uint32_t d = g.slots[v];
  bool want = false;
  if (threadIdx.x == 0 && d) want = atomicOr(&m_out[v], bits) == 0u;
  frontier_append(out, want, v, d);
}

// Deletion seeds: deleted (u,v) whose lane-q parent of v is u reset lane q.
template <int S>
__global__ void k_group_seed_deleted(GraphView g, unsigned long long *st, uint32_t *val, uint32_t lanes,
                                     LaneAlgo algo, const uint64_t *keys, uint32_t n,
                                     unsigned long long *inval, uint32_t *mark, uint32_t *m_out,
                                     FrontierView out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    bool want = false;
    uint32_t v = 0, d = 0;
    if (i < n) {
      const uint64_t k = keys[i];
      const uint32_t u = (uint32_t)(k >> 32);
      v = (uint32_t)k;
      uint32_t bits = 0;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        if (!(lanes >> q & 1u)) continue;
        const uint64_t idx = (uint64_t)v * S + q;
        const unsigned long long cu = __ldcg(&st[idx]);
        if ((uint32_t)cu != u) continue;
        const bool cc = algo.at(q) == A_CC;
        const unsigned long long rst = cc ? (((unsigned long long)v << 32) | INF32) : ~0ull;
        if (atomicCAS(&st[idx], cu, rst) == cu) {
          val[idx] = cc ? v : INF32;
          bits |= 1u << q;
          atomicAdd(&inval[q], 1ull);
        }
      }
      if (bits) {
        if (mark) bit_set(mark, v);
        d = g.slots[v];
        want = d && atomicOr(&m_out[v], bits) == 0u;
      }
    }
    frontier_append(out, want, v, d);
  }
}

// Relaxes just the kept inserted edges in the selected lanes: the whole
// repair of an insert-only batch, and the inserted-edge half of the repair
// after an invalidation (the other half is the restricted first round).
// With `skip_if_reset`, the launch does nothing when a selected lane was
// reset by the last invalidation (the full sweep covers the inserted edges).
template <int S>
__global__ void k_group_relax_inserted(GraphView g, unsigned long long *st, uint32_t *val, uint32_t lanes,
                                       LaneAlgo algo, const uint64_t *keys, const uint32_t *w,
                                       const uint32_t *n_ptr, uint32_t *m_out, FrontierView out,
                                       unsigned long long *lane_edges,
                                       const unsigned long long *skip_if_reset = nullptr) {
  if (skip_if_reset && block_any_lane(skip_if_reset, lanes)) return;
  const uint32_t n = *n_ptr;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t counted = 0;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    bool want = false;
    uint32_t v = 0, d = 0;
    if (i < n) {
      const uint64_t k = keys[i];
      const uint32_t u = (uint32_t)(k >> 32);
      v = (uint32_t)k;
      ++counted;
      uint32_t su[S], sv[S];
      load_vals<S>(val, u, su);
      load_vals<S>(val, v, sv);
      uint32_t bits = 0;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        if (!(lanes >> q & 1u)) continue;
        const int a = algo.at(q);
        uint32_t cand;
        if (a == A_CC) {
          cand = su[q];
        } else {
          if (su[q] == INF32) continue;
          uint32_t wt = 1;
          if (a == A_SSSP)
            wt = g.wmode == W_EXPLICIT ? w[i] : g.wmode == W_SYNTH ? (u + v) % 128u + 1u : 1u;
          const uint64_t nd = (uint64_t)su[q] + wt;
          if (nd >= INF32) continue;
          cand = (uint32_t)nd;
        }
        if (cand >= sv[q]) continue;
        const uint64_t idx = (uint64_t)v * S + q;
        if (relax_mirror_packed(&val[idx], &st[idx], cand, u)) bits |= 1u << q;
      }
      if (bits) {
        d = g.slots[v];
        want = d && atomicOr(&m_out[v], bits) == 0u;
      }
    }
    frontier_append(out, want, v, d);
  }
  if (counted) {
#pragma unroll
    for (int q = 0; q < S; ++q)
      if (lanes >> q & 1u) atomicAdd(&lane_edges[q], (unsigned long long)counted);
  }
}

template <int S>
__global__ void k_group_split(const unsigned long long *st, uint32_t nv, int lane, uint32_t *val,
                              uint32_t *par) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    const unsigned long long s = st[v * S + lane];
    if (val) val[v] = (uint32_t)(s >> 32);
    if (par) par[v] = (uint32_t)s;
  }
}

template <int S>
__global__ void k_group_summary(const unsigned long long *st, uint32_t nv, int lane,
                                unsigned long long *out) {
  unsigned long long reached = 0, sum = 0, mx = 0, psum = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    const unsigned long long s = st[v * S + lane];
    const uint32_t val = (uint32_t)(s >> 32);
    if (val == INF32) continue;
    reached += 1;
    sum += val;
    mx = val > mx ? val : mx;
    if ((uint32_t)s != INF32) psum += (uint32_t)s;
  }
  reached = warp_sum(reached);
  sum = warp_sum(sum);
  psum = warp_sum(psum);
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, mx, s);
    mx = o > mx ? o : mx;
  }
  if ((threadIdx.x & 31) == 0) {
    if (reached) atomicAdd(&out[0], reached);
    if (sum) atomicAdd(&out[1], sum);
    atomicMax(&out[2], mx);
    if (psum) atomicAdd(&out[3], psum);
  }
}

// The same summaries for several lanes of a narrow group in one pass over
// the state rows (one 32-B row per vertex read once for all of them):
// slot[q] >= 0 selects lane q and its 4 counters at out + 4 * slot[q].
struct LaneSlots {
  int slot[GMAX];
};
__global__ void k_group_summary_lanes(const unsigned long long *st, uint32_t nv, LaneSlots ls,
                                      unsigned long long *out) {
  unsigned long long reached[GMAX] = {}, sum[GMAX] = {}, mx[GMAX] = {}, psum[GMAX] = {};
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    const ulonglong2 a = __ldcs(reinterpret_cast<const ulonglong2 *>(st + v * GMAX));
    const ulonglong2 b = __ldcs(reinterpret_cast<const ulonglong2 *>(st + v * GMAX + 2));
    const unsigned long long row[GMAX] = {a.x, a.y, b.x, b.y};
#pragma unroll
    for (int q = 0; q < GMAX; ++q) {
      if (ls.slot[q] < 0) continue;
      const uint32_t val = (uint32_t)(row[q] >> 32);
      if (val == INF32) continue;
      reached[q] += 1;
      sum[q] += val;
      mx[q] = val > mx[q] ? val : mx[q];
      if ((uint32_t)row[q] != INF32) psum[q] += (uint32_t)row[q];
    }
  }
#pragma unroll
  for (int q = 0; q < GMAX; ++q) {
    if (ls.slot[q] < 0) continue;
    const unsigned long long r = warp_sum(reached[q]), su = warp_sum(sum[q]), ps = warp_sum(psum[q]);
    unsigned long long m = mx[q];
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
      const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, m, sh);
      m = o > m ? o : m;
    }
    if ((threadIdx.x & 31) == 0) {
      unsigned long long *o = out + 4 * ls.slot[q];
      if (r) atomicAdd(&o[0], r);
      if (su) atomicAdd(&o[1], su);
      atomicMax(&o[2], m);
      if (ps) atomicAdd(&o[3], ps);
    }
  }
}

// Lanes present in a frontier: per-lane counts of its entries' mask bits
// (narrow u32 or wide u64 masks), for a serving loop that retires a lane as
// soon as no entry carries it.
template <class M>
__global__ void k_lane_counts(const uint32_t *vtx, const unsigned long long *cnt, const M *mask,
                              unsigned long long *out) {
  __shared__ unsigned long long s[64];
  if (threadIdx.x < 64) s[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t n = (uint32_t)(__ldcg(cnt) >> CNT_SHIFT);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long m = (unsigned long long)__ldcg(&mask[__ldcg(&vtx[i])]);
    while (m) {
      const int q = __ffsll((long long)m) - 1;
      atomicAdd(&s[q], 1ull);
      m &= m - 1;
    }
  }
  __syncthreads();
  if (threadIdx.x < 64 && s[threadIdx.x]) atomicAdd(&out[threadIdx.x], s[threadIdx.x]);
}

// Dense seeding of CC lanes into a frontier that may already hold entries:
// OR the lanes in, append only vertices whose mask was empty.
template <class M>
__global__ void k_seed_all_or(GraphView g, M bits, M *m_out, FrontierView out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < g.nv; b += stride) {
    const uint64_t v = b + threadIdx.x;
    bool want = false;
    uint32_t d = 0;
    if (v < g.nv) {
      d = g.slots[v];
      if (d) want = atomicOr(&m_out[v], bits) == (M)0;
    }
    frontier_append_block(out, want, (uint32_t)v, d);
  }
}

// Masks of the last non-empty frontier (after convergence).
__global__ void k_clear_masks(const uint32_t *vtx, const unsigned long long *cnt, uint32_t *mask) {
  clear_prev_masks(vtx, cnt, mask);
}

}  // namespace sgs
