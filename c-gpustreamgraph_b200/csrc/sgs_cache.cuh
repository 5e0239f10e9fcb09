// sgs_cache.cuh -- device edge cache of the host tier: hotness window,
// per-snapshot admission / eviction and the line copies.
//
// Reference behaviour (include/framework/variants/driver.cuh:437-516,
// include/framework/graph_datum.cuh:151-189,258-269, framework.cuh:149-308):
// every vertex carries four u8 activation counters, one per snapshot of a
// sliding window (csr_graph.cuh:308; bumped by the push kernels,
// sync_push_dd.cuh:224,326; shifted once per snapshot, driver.cuh:505-515);
// the hotness of a vertex is their sum (driver.cuh:448); vertices are sorted
// by hotness and the prefix whose degrees fit the cache capacity is admitted,
// the rest evicted, survivors compacted and new lists copied from host.
//
// Here the same window and score drive a cache of fixed-size LINES of the
// host arena (CLINE = 128 slots) instead of whole vertex lists:
//   * line score = sum over the slots it holds of the owning vertex's
//     hotness, i.e. the slot reads the window saw from that line;
//   * admission = the top lines by score that fit the capacity, found with a
//     histogram over the (bounded) score range and a threshold instead of a
//     sort; ties at the threshold take tickets, lines already cached first;
//   * lines have one size, so a freed cache line is reused as it is: no
//     allocator and no compaction pass;
//   * the copy of newly admitted lines runs on a side stream while the
//     snapshot's queries run, and the lines become visible (cmap) after it.
// The snapshot's writes into cached lines (tombstones, appended edges,
// relocated blocks) are made to both copies, so the cache never differs from
// the host arena and hot lines survive the updates that touch them; lines of
// blocks that moved away score zero and are evicted by the next admission.
#pragma once
#include <cub/block/block_scan.cuh>

#include "sgs_device.cuh"

namespace sgs {

constexpr uint32_t HOT_BINS = 1u << 17;  // line scores are < 4 * 255 * CLINE
// lines with a smaller score are never admitted (1: any read in the window,
// so a cache larger than the hot part of the host tier holds all of it, as the
// reference admits its whole sorted prefix)
constexpr uint32_t LINE_MIN_SCORE = 1;

// Counter block of the cache (device, u64):
//   [0] host-tier slots walked  [1] of those, slots read over the host link
//   [2] tie tickets  [3] new lines picked  [4] free cache lines found
//   [5] lines admitted (copies)  [6] lines evicted  [7] threshold t_hi
//   [8] tie score t_tie  [9] tie quota
enum : int {
  CC_WALK = 0, CC_MISS, CC_TICK, CC_NEW, CC_FREE, CC_ADMIT, CC_EVICT, CC_THI, CC_TTIE, CC_REM, CC_N
};

// Line scores from the hotness window; clears byte `clear_sh / 8` of every
// counter when clear_sh < 32 (the byte the next snapshot fills).
__global__ void k_cache_score(GraphView g, uint32_t clear_sh, uint32_t *score, uint64_t nlines) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < g.nv; v += stride) {
    const uint64_t o = g.off[v];
    if (!(o & HOST_BIT)) continue;
    const uint32_t h = g.hot[v];
    if (!h) continue;
    const uint32_t sum = (h & 0xFFu) + (h >> 8 & 0xFFu) + (h >> 16 & 0xFFu) + (h >> 24);
    if (clear_sh < 32) g.hot[v] = h & ~(0xFFu << clear_sh);
    const uint32_t n = g.slots[v];
    if (!n) continue;
    const uint64_t h0 = o & OFF_MASK, h1 = h0 + n;  // [h0, h1)
    for (uint64_t c = h0 >> CLINE_SHIFT; c <= (h1 - 1) >> CLINE_SHIFT && c < nlines; ++c) {
      const uint64_t a = max(h0, c << CLINE_SHIFT), b = min(h1, (c + 1) << CLINE_SHIFT);
      atomicAdd(&score[c], sum * (uint32_t)(b - a));
    }
  }
}

__global__ void k_cache_hist(const uint32_t *score, uint64_t nlines, uint32_t *hist) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nlines; c += stride) {
    const uint32_t s = score[c];
    if (s >= LINE_MIN_SCORE) atomicAdd(&hist[min(s, HOT_BINS - 1)], 1u);
  }
}

// Threshold for a capacity of `cap` lines (one block of 1024 threads, 128
// bins each, highest scores first): every line with score >= t_hi fits, and
// `rem` more of those with score == t_tie.  When all candidates fit, t_hi is
// the minimum score and no tie is taken.
__global__ void __launch_bounds__(1024) k_cache_threshold(const uint32_t *hist, uint64_t cap,
                                                          unsigned long long *cc) {
  constexpr int PER = HOT_BINS / 1024;
  typedef cub::BlockScan<unsigned long long, 1024> BS;
  __shared__ typename BS::TempStorage tmp;
  const int k = threadIdx.x;
  const uint32_t top = HOT_BINS - (uint32_t)k * PER;  // bins [top - PER, top)
  unsigned long long mine = 0;
  for (int i = 1; i <= PER; ++i) mine += hist[top - i];
  unsigned long long before = 0;
  BS(tmp).ExclusiveSum(mine, before);
  if (k == 0) {
    cc[CC_THI] = LINE_MIN_SCORE;
    cc[CC_TTIE] = 0xFFFFFFFFull;
    cc[CC_REM] = 0;
  }
  __syncthreads();
  if (before <= cap && before + mine > cap) {  // the crossing is in my bins
    unsigned long long cum = before;
    for (int i = 1; i <= PER; ++i) {
      const uint32_t b = top - i;
      const uint32_t hb = hist[b];
      if (cum + hb > cap) {
        cc[CC_THI] = b + 1;
        cc[CC_TTIE] = b;
        cc[CC_REM] = cap - cum;
        break;
      }
      cum += hb;
    }
  }
}

__device__ __forceinline__ bool line_takes(uint32_t s, const unsigned long long *cc,
                                           unsigned long long *tick) {
  if (s >= cc[CC_THI]) return true;
  return s == cc[CC_TTIE] && atomicAdd(tick, 1ull) < cc[CC_REM];
}

// Cached lines that stay (score above the threshold, or a tie ticket) keep
// their place; the others are evicted.
__global__ void k_cache_keep(uint32_t *cmap, uint32_t *cown, const uint32_t *score, uint64_t ncache,
                             unsigned long long *cc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t ev = 0;
  for (uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; m < ncache; m += stride) {
    const uint32_t c = cown[m];
    if (c == NO_LINE) continue;
    if (line_takes(score[c], cc, &cc[CC_TICK])) continue;
    cmap[c] = NO_LINE;
    cown[m] = NO_LINE;
    ++ev;
  }
  if (ev) atomicAdd(&cc[CC_EVICT], (unsigned long long)ev);
}

// Lines to admit: not cached and above the threshold (ties after the cached
// ones took their tickets).
__global__ void k_cache_pick(const uint32_t *cmap, const uint32_t *score, uint64_t nlines,
                             uint64_t ncache, uint32_t *newl, unsigned long long *cc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nlines; c += stride) {
    const uint32_t s = score[c];
    if (s < LINE_MIN_SCORE || cmap[c] != NO_LINE) continue;
    if (!line_takes(s, cc, &cc[CC_TICK])) continue;
    const unsigned long long i = atomicAdd(&cc[CC_NEW], 1ull);
    if (i < ncache) newl[i] = (uint32_t)c;
  }
}

__global__ void k_cache_free(const uint32_t *cown, uint64_t ncache, uint32_t *freel,
                             unsigned long long *cc) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; m < ncache; m += stride)
    if (cown[m] == NO_LINE) freel[atomicAdd(&cc[CC_FREE], 1ull)] = (uint32_t)m;
}

// Pairs the i-th new line with the i-th free cache line and reserves it;
// the pair list is what the copy and the publish read.
__global__ void k_cache_pair(const uint32_t *newl, const uint32_t *freel, uint64_t ncache,
                             uint32_t *cown, uint2 *pend, unsigned long long *cc) {
  const unsigned long long n = min(min(cc[CC_NEW], cc[CC_FREE]), (unsigned long long)ncache);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t c = newl[i], m = freel[i];
    pend[i] = make_uint2(c, m);
    cown[m] = c;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cc[CC_ADMIT] = n;
}

// Copies the pending lines host -> cache: one warp per line, 16 B per thread
// of ids (and of weights).  Runs on the side stream.
__global__ void k_cache_copy(const uint2 *pend, const unsigned long long *cc, const uint32_t *adj_h,
                             const uint32_t *wgt_h, uint32_t *adj_c, uint32_t *wgt_c) {
  const unsigned long long n = cc[CC_ADMIT];
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nwarp = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarp) {
    const uint2 p = pend[i];
    const uint64_t src = ((uint64_t)p.x << CLINE_SHIFT) + 4 * lane;
    const uint64_t dst = ((uint64_t)p.y << CLINE_SHIFT) + 4 * lane;
    *reinterpret_cast<uint4 *>(adj_c + dst) = __ldcv(reinterpret_cast<const uint4 *>(adj_h + src));
    if (wgt_h)
      *reinterpret_cast<uint4 *>(wgt_c + dst) = __ldcv(reinterpret_cast<const uint4 *>(wgt_h + src));
  }
}

// Makes the copied lines visible.
__global__ void k_cache_publish(const uint2 *pend, const unsigned long long *cc, uint32_t *cmap) {
  const unsigned long long n = cc[CC_ADMIT];
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint2 p = pend[i];
    cmap[p.x] = p.y;
  }
}

}  // namespace sgs
