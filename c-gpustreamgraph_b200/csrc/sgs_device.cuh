// sgs_device.cuh -- device-side data layout and shared helpers of the
// B200 streaming-graph engine.
//
// Layout in HBM (one engine = one dynamic graph + N registered queries):
//
//   per vertex (struct-of-arrays, 20 B/vertex):
//     off[v]   u64  start of v's edge block in an arena; bit 63 selects the
//                   pinned-host arena (out-of-HBM tier) instead of HBM
//     slots[v] u32  used slots of the block (live edges + tombstones)
//     live[v]  u32  live out-degree (what PageRank divides by)
//     cap[v]   u32  capacity of the block (multiple of 4, block 16-B aligned)
//   arenas (per tier): adj[] u32 destination ids, wgt[] u32 weights (only
//     when weights are stored explicitly); a deleted edge becomes a tombstone
//     (adj == SGS_TOMB) until its block is relocated or compacted.
//
//   per query: st[v] u64 packed (value << 32 | parent) for BFS/SSSP/CC; a
//     single 64-bit atomic keeps value and parent consistent, which is what
//     makes parent-tree invalidation after deletions exact.  PageRank keeps
//     x[v], r[v] in FP64.
//
//   frontier (shared scratch): entries (vertex, edge-prefix) appended with
//     one packed 64-bit atomicAdd per warp: count in the high 27 bits, the
//     running sum of block sizes in the low 37 bits.  So the append itself
//     produces the exclusive prefix sum of degrees, and it also writes, for
//     every unit of UNIT edges, the first entry covering it.  The next round
//     splits its edges into equal units with no scan kernel and no host sync.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sgs {

constexpr uint32_t INF32 = 0xFFFFFFFFu;
constexpr uint32_t SGS_TOMB = 0xFFFFFFFFu;   // tombstoned edge slot
constexpr uint64_t HOST_BIT = 1ull << 63;
constexpr uint64_t OFF_MASK = HOST_BIT - 1;
constexpr int CNT_SHIFT = 37;                 // packed frontier counter
constexpr uint64_t EDGE_MASK = (1ull << CNT_SHIFT) - 1;
constexpr uint32_t UNIT = 2048;               // edges per load-balanced unit
constexpr int RELAX_THREADS = 256;

enum Algo : int { A_BFS = 0, A_SSSP = 1, A_CC = 2, A_PR = 3 };
enum WMode : int { W_EXPLICIT = 0, W_SYNTH = 1, W_UNIT = 2 };

struct GraphView {
  uint32_t nv;
  uint64_t *off;
  uint32_t *slots;
  uint32_t *live;
  uint32_t *cap;
  uint32_t *adj_d;   // HBM arena
  uint32_t *wgt_d;
  uint32_t *adj_h;   // pinned, mapped host arena (may be null)
  uint32_t *wgt_h;
  int wmode;
  // device edge cache of the host tier (all null when the cache is off):
  // cmap[c] = cache line holding host-arena line c (slots [c*CLINE,
  // (c+1)*CLINE)) or NO_LINE; adj_c/wgt_c hold the cached lines
  const uint32_t *cmap;
  uint32_t *adj_c;  // = adj_d + cbase: the cache lines follow the HBM arena
  uint32_t *wgt_c;
  uint64_t cbase;
  // hotness: per vertex four u8 counters of activations (one per snapshot of
  // a four-snapshot window); relaxation kernels add 1 to byte hot_sh / 8 of
  // every host-tier vertex they expand
  uint32_t *hot;
  uint32_t hot_sh;
  // [0] host-tier slots the relaxation maps walked, [1] of those, slots read
  // over the host link (the rest came from the cache)
  unsigned long long *cstat;
};

struct FrontierView {
  uint32_t *vtx;       // [cap] vertex of each entry
  uint32_t *len;       // [cap] slots of the entry (its range is padded to 4)
  uint64_t *ebase;     // [cap] exclusive prefix of padded block sizes
  uint32_t *ustart;    // [ucap] first entry of each UNIT-edge unit
  uint64_t *counter;   // packed (count << 37 | edges)
  uint32_t ucap;
};

__device__ __forceinline__ uint64_t pack(uint32_t val, uint32_t par) {
  return ((uint64_t)val << 32) | par;
}
__device__ __forceinline__ uint32_t val_of(uint64_t s) { return (uint32_t)(s >> 32); }
__device__ __forceinline__ uint32_t par_of(uint64_t s) { return (uint32_t)s; }

__device__ __forceinline__ const uint32_t *adj_ptr(const GraphView &g, uint64_t o) {
  return ((o & HOST_BIT) ? g.adj_h : g.adj_d) + (o & OFF_MASK);
}
__device__ __forceinline__ const uint32_t *wgt_ptr(const GraphView &g, uint64_t o) {
  return ((o & HOST_BIT) ? g.wgt_h : g.wgt_d) + (o & OFF_MASK);
}
__device__ __forceinline__ uint32_t *adj_wptr(const GraphView &g, uint64_t o) {
  return ((o & HOST_BIT) ? g.adj_h : g.adj_d) + (o & OFF_MASK);
}
__device__ __forceinline__ uint32_t *wgt_wptr(const GraphView &g, uint64_t o) {
  return ((o & HOST_BIT) ? g.wgt_h : g.wgt_d) + (o & OFF_MASK);
}

// Device edge cache.  The host arena is cut into lines of CLINE slots (512 B
// of ids, and as much of weights); a line the cache holds is read from HBM
// instead of over the host link.  The host copy stays authoritative and the
// cache is written through (every write of a snapshot into a cached line is
// made to both copies), so the two never differ and any reader may use
// either.
// Blocks and the quads read from them are 16-B aligned, so a quad never
// straddles two lines.
constexpr uint32_t CLINE_SHIFT = 7;
constexpr uint32_t CLINE = 1u << CLINE_SHIFT;
constexpr uint32_t NO_LINE = 0xFFFFFFFFu;

// Cache line holding host-arena slot h, or NO_LINE.
__device__ __forceinline__ uint32_t cache_line(const GraphView &g, uint64_t h) {
  return g.cmap ? __ldg(g.cmap + (h >> CLINE_SHIFT)) : NO_LINE;
}
// Slots j.. of the block at offset o, for reading: HBM arena, cached line or
// host arena.
__device__ __forceinline__ const uint32_t *adj_at(const GraphView &g, uint64_t o, uint32_t j) {
  if (!(o & HOST_BIT)) return g.adj_d + o + j;
  const uint64_t h = (o & OFF_MASK) + j;
  const uint32_t m = cache_line(g, h);
  if (m != NO_LINE) return g.adj_c + ((uint64_t)m << CLINE_SHIFT) + (h & (CLINE - 1));
  return g.adj_h + h;
}
__device__ __forceinline__ const uint32_t *wgt_at(const GraphView &g, uint64_t o, uint32_t j) {
  if (!(o & HOST_BIT)) return g.wgt_d + o + j;
  const uint64_t h = (o & OFF_MASK) + j;
  const uint32_t m = cache_line(g, h);
  if (m != NO_LINE) return g.wgt_c + ((uint64_t)m << CLINE_SHIFT) + (h & (CLINE - 1));
  return g.wgt_h + h;
}
// Offset to read the block at o (len slots) from: when the whole block lies
// in one cached line, its place in the cache region of the HBM arena (an HBM
// offset, so no per-read lookup follows); otherwise o.
__device__ __forceinline__ uint64_t resolve_block(const GraphView &g, uint64_t o, uint32_t len) {
  if (!(o & HOST_BIT) || !g.cmap || !len) return o;
  const uint64_t h0 = o & OFF_MASK;
  if ((h0 >> CLINE_SHIFT) != ((h0 + len - 1) >> CLINE_SHIFT)) return o;
  const uint32_t m = __ldg(g.cmap + (h0 >> CLINE_SHIFT));
  return m == NO_LINE ? o : g.cbase + ((uint64_t)m << CLINE_SHIFT) + (h0 & (CLINE - 1));
}

// Write-through of slot j of the block at offset o: the cached copy of its
// line, or null (HBM block, or line not cached).
__device__ __forceinline__ uint32_t *cache_slot_w(const GraphView &g, uint32_t *base, uint64_t o,
                                                  uint32_t j) {
  if (!(o & HOST_BIT) || !g.cmap) return nullptr;
  const uint64_t h = (o & OFF_MASK) + j;
  const uint32_t m = g.cmap[h >> CLINE_SHIFT];
  return m == NO_LINE ? nullptr : base + ((uint64_t)m << CLINE_SHIFT) + (h & (CLINE - 1));
}
// Stores id (and weight) into slot j of the block at o, and into its cached
// line if there is one.
__device__ __forceinline__ void store_slot(const GraphView &g, uint64_t o, uint32_t j, uint32_t id,
                                           bool has_w, uint32_t w) {
  uint32_t *a = ((o & HOST_BIT) ? g.adj_h : g.adj_d) + (o & OFF_MASK) + j;
  *a = id;
  if (has_w) ((o & HOST_BIT) ? g.wgt_h : g.wgt_d)[(o & OFF_MASK) + j] = w;
  if (uint32_t *c = cache_slot_w(g, g.adj_c, o, j)) {
    *c = id;
    if (has_w) g.wgt_c[c - g.adj_c] = w;
  }
}

// One activation of host-tier vertex v in the current snapshot's counter
// (saturating at 255; the counters of the window are summed at admission).
// Called by the one thread that owns v's frontier entry.
__device__ __forceinline__ void hot_bump(const GraphView &g, uint32_t v, uint64_t o) {
  if (!g.hot || !(o & HOST_BIT)) return;
  const uint32_t h = g.hot[v];
  if ((h >> g.hot_sh & 0xFFu) != 0xFFu) g.hot[v] = h + (1u << g.hot_sh);
}

// One relaxation of a lane: the u32 value mirror *m first, then the packed
// (value << 32 | parent) word *p; true when cand strictly lowered the mirror.
// Only the thread whose atomicMin lowers the mirror to cand offers cand to
// the packed word, so two equal candidates never both reach it, and the
// packed word's parent changes only with a strictly better value.  (A 64-bit
// atomicMin alone also replaces the parent when the values tie and the new
// parent id is smaller.  CC labels are equal along tight parents, so such tie
// swaps could close a parent cycle that the parent-tree invalidation never
// reaches; SSSP/BFS parents have strictly smaller values.)  The packed update
// is a reduction nobody waits for: when a smaller candidate overtakes this
// one between the two atomics, the caller's "improved" only costs a redundant
// frontier entry.  The mirror may run ahead of the packed value for a moment,
// never below the value the packed word is about to take, so a pre-check
// against it still rejects only candidates that cannot improve.
__device__ __forceinline__ bool relax_mirror_packed(uint32_t *m, unsigned long long *p, uint32_t cand,
                                                    uint32_t u) {
  if (atomicMin(m, cand) <= cand) return false;
  atomicMin(p, ((unsigned long long)cand << 32) | u);
  return true;
}

// Weight of slot j of u's block.  Synthesized mode reproduces the
// reference's per-edge (src+dst)%128+1 (push_functor.h:306).
__device__ __forceinline__ uint32_t edge_weight(const GraphView &g, uint64_t o,
                                                uint32_t j, uint32_t u,
                                                uint32_t dst) {
  if (g.wmode == W_EXPLICIT) return wgt_ptr(g, o)[j];
  if (g.wmode == W_SYNTH) return (u + dst) % 128u + 1u;
  return 1u;
}

// True when some lane of `lanes` has a non-zero count in cnt[] (per-lane
// reset counts of a group's last invalidation); one read per block, so a
// whole launch can be skipped on the device without a host round trip.
// Block-uniform; must be called by every thread of the block.
__device__ __forceinline__ bool block_any_lane(const unsigned long long *cnt, uint64_t lanes) {
  __shared__ int s_any;
  if (threadIdx.x == 0) {
    int a = 0;
    for (int q = 0; q < 64; ++q)
      if ((lanes >> q & 1ull) && cnt[q]) a = 1;
    s_any = a;
  }
  __syncthreads();
  return s_any != 0;
}

// Vertex bitmaps (one bit per vertex): `only` restricts a relaxation round to
// destinations whose bit is set; `mark` records vertices reset by the
// parent-tree invalidation.
__device__ __forceinline__ bool bit_at(const uint32_t *bm, uint32_t v) {
  return __ldcg(&bm[v >> 5]) >> (v & 31) & 1u;
}
__device__ __forceinline__ void bit_set(uint32_t *bm, uint32_t v) {
  atomicOr(&bm[v >> 5], 1u << (v & 31));
}

// Warp-aggregated append of (v, d) into a frontier.  Must be called by all 32
// lanes of a converged warp; `want` selects the lanes that append.  One packed
// 64-bit atomicAdd per warp reserves the slots and the edge range together.
// Block-aggregated append of up to N consecutive vertices per thread
// (v0 + i for want[i]): one atomic per block call for N x blockDim items,
// entries in thread order, so a block's vertices stay in vertex order.
template <int N>
__device__ __forceinline__ void frontier_append_block_n(const FrontierView &f, const bool (&want)[N],
                                                        uint32_t v0, const uint32_t (&d)[N]) {
  constexpr int NW = RELAX_THREADS / 32;
  __shared__ unsigned long long s_warp[NW];
  __shared__ unsigned long long s_base;
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long inc = 0;
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (want[i]) inc += (1ull << CNT_SHIFT) | (unsigned long long)((d[i] + 3u) & ~3u);
  unsigned long long x = inc;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const unsigned long long y = __shfl_up_sync(full, x, s);
    if (lane >= s) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (int w = 0; w < NW; ++w) {
      const unsigned long long t = s_warp[w];
      s_warp[w] = run;
      run += t;
    }
    s_base = run ? atomicAdd((unsigned long long *)f.counter, run) : 0ull;
  }
  __syncthreads();
  if (inc) {
    unsigned long long pos = s_base + s_warp[wid] + (x - inc);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if (!want[i]) continue;
      const uint32_t dp = (d[i] + 3u) & ~3u;
      const uint32_t slot = (uint32_t)(pos >> CNT_SHIFT);
      const uint64_t eb = pos & EDGE_MASK;
      f.vtx[slot] = v0 + i;
      f.len[slot] = d[i];
      f.ebase[slot] = eb;
      if (dp) {
        const uint64_t u0 = (eb + UNIT - 1) / UNIT, u1 = (eb + dp - 1) / UNIT;
        for (uint64_t u = u0; u <= u1 && u < f.ucap; ++u) f.ustart[u] = slot;
      }
      pos += (1ull << CNT_SHIFT) | (unsigned long long)dp;
    }
  }
  __syncthreads();  // s_warp / s_base are reused by the next call
}

__device__ __forceinline__ void frontier_append(const FrontierView &f, bool want,
                                                uint32_t v, uint32_t d,
                                                uint32_t *aux = nullptr,
                                                uint32_t aux_val = 0) {
  const unsigned full = 0xFFFFFFFFu;
  unsigned m = __ballot_sync(full, want);
  if (!m) return;
  const int lane = threadIdx.x & 31;
  const uint32_t dp = (d + 3u) & ~3u;  // ranges padded to whole 16-B quads
  uint64_t inc = want ? ((1ull << CNT_SHIFT) | (uint64_t)dp) : 0ull;
  // inclusive warp scan of inc
  uint64_t x = inc;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    uint64_t y = __shfl_up_sync(full, x, s);
    if (lane >= s) x += y;
  }
  uint64_t total = __shfl_sync(full, x, 31);
  uint64_t base = 0;
  if (lane == 31) base = atomicAdd((unsigned long long *)f.counter, (unsigned long long)total);
  base = __shfl_sync(full, base, 31);
  if (want) {
    uint64_t excl = x - inc;
    uint32_t slot = (uint32_t)((base >> CNT_SHIFT) + (excl >> CNT_SHIFT));
    uint64_t eb = (base & EDGE_MASK) + (excl & EDGE_MASK);
    f.vtx[slot] = v;
    f.len[slot] = d;
    f.ebase[slot] = eb;
    if (aux) aux[slot] = aux_val;
    if (dp) {
      uint64_t u0 = (eb + UNIT - 1) / UNIT, u1 = (eb + dp - 1) / UNIT;
      for (uint64_t u = u0; u <= u1 && u < f.ucap; ++u) f.ustart[u] = slot;
    }
  }
}

// Block-aggregated append: one atomic per CTA instead of one per warp, for
// builders where most threads append.  Every thread of the CTA (blockDim.x ==
// RELAX_THREADS) must call it the same number of times.
__device__ __forceinline__ void frontier_append_block(const FrontierView &f, bool want,
                                                      uint32_t v, uint32_t d,
                                                      uint32_t *aux = nullptr,
                                                      uint32_t aux_val = 0) {
  constexpr int NW = RELAX_THREADS / 32;
  __shared__ unsigned long long s_warp[NW];
  __shared__ unsigned long long s_base;
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t dp = (d + 3u) & ~3u;
  const unsigned long long inc = want ? ((1ull << CNT_SHIFT) | (unsigned long long)dp) : 0ull;
  unsigned long long x = inc;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const unsigned long long y = __shfl_up_sync(full, x, s);
    if (lane >= s) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long run = 0;
    for (int w = 0; w < NW; ++w) {
      const unsigned long long t = s_warp[w];
      s_warp[w] = run;
      run += t;
    }
    s_base = run ? atomicAdd((unsigned long long *)f.counter, run) : 0ull;
  }
  __syncthreads();
  if (want) {
    const unsigned long long pos = s_base + s_warp[wid] + (x - inc);
    const uint32_t slot = (uint32_t)(pos >> CNT_SHIFT);
    const uint64_t eb = pos & EDGE_MASK;
    f.vtx[slot] = v;
    f.len[slot] = d;
    f.ebase[slot] = eb;
    if (aux) aux[slot] = aux_val;
    if (dp) {
      const uint64_t u0 = (eb + UNIT - 1) / UNIT, u1 = (eb + dp - 1) / UNIT;
      for (uint64_t u = u0; u <= u1 && u < f.ucap; ++u) f.ustart[u] = slot;
    }
  }
  __syncthreads();  // s_warp / s_base are reused by the next call
}

// Warp-aggregated atomicAdd: lanes with want add val to *p; returns each
// lane's old value (exclusive prefix within the warp added).  All 32 lanes of
// a converged warp must call it.
__device__ __forceinline__ unsigned long long warp_atomic_add(unsigned long long *p, bool want,
                                                              unsigned long long val) {
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  unsigned long long x = want ? val : 0ull;
  const unsigned long long inc = x;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const unsigned long long y = __shfl_up_sync(full, x, s);
    if (lane >= s) x += y;
  }
  const unsigned long long total = __shfl_sync(full, x, 31);
  unsigned long long base = 0;
  if (lane == 31 && total) base = atomicAdd(p, total);
  base = __shfl_sync(full, base, 31);
  return base + x - inc;
}

// 16-B read-only load of four consecutive u32 slots (block starts and j0 are
// multiples of 4 elements, so the address is 16-B aligned).
__device__ __forceinline__ uint4 ld_quad(const uint32_t *p) {
  return __ldg(reinterpret_cast<const uint4 *>(p));
}
// The same for a stream read exactly once per pass (a frontier's ids and
// weights): no L1 allocation, and the line is the first the L2 evicts, so
// the randomly re-read per-vertex state keeps more of the L2.
// (A 128-bit load takes its L2 priority from a cache policy operand; the
// plain .L2::evict_first qualifier is for 256-bit loads only.)
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint4 ld_quad_stream(const uint32_t *p) {
  uint4 r;
  // (not volatile: a pure read of data no kernel writes while it runs, so
  // the compiler may schedule it freely)
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p), "l"(l2_evict_first_policy()));
  return r;
}
__device__ __forceinline__ uint32_t quad_at(const uint4 &q, int k) {
  return k == 0 ? q.x : k == 1 ? q.y : k == 2 ? q.z : q.w;
}

// Block-wide helpers --------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, s);
  return v;
}

}  // namespace sgs
