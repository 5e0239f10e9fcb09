// sgs_segmap.cuh -- the engine's load-balanced segmented map kernel
// (template only, so several translation units can instantiate it).
#pragma once
#include <cub/block/block_reduce.cuh>

#include "sgs_device.cuh"

namespace sgs {

// ---------------------------------------------------------------------------
// Generic load-balanced segmented map.
//
// The input frontier is a list of entries (vertex v, ebase) whose ranges
// [ebase_s, ebase_{s+1}) tile [0, T).  Units of UNIT consecutive positions are
// spread over a fixed grid; a CTA stages up to CHUNK entries of its unit in
// shared memory (the per-entry payload is loaded once, coalesced) and then
// its threads walk consecutive positions, so consecutive lanes touch
// consecutive slots of the same block (coalesced 128-B lines).  Every thread
// of a CTA runs the same trip count, so warp-aggregated appends always see
// full warps.
// ---------------------------------------------------------------------------
constexpr int CHUNK = 256;

template <class Op>
__global__ void __launch_bounds__(RELAX_THREADS)
    seg_map(FrontierView in, FrontierView out, Op op, unsigned long long *edge_stat) {
  using P = typename Op::Payload;
  __shared__ uint64_t s_eb[CHUNK + 1];
  __shared__ P s_pay[CHUNK];
  __shared__ uint32_t s_vtx[CHUNK];
  const uint64_t packed = __ldcg((const unsigned long long *)in.counter);
  const uint32_t n = (uint32_t)(packed >> CNT_SHIFT);
  const uint64_t T = packed & EDGE_MASK;
  if (n == 0 || T == 0) return;
  const uint64_t nunits = (T + UNIT - 1) / UNIT;
  uint64_t counted = 0;
  for (uint64_t unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
    const uint64_t E0 = unit * UNIT;
    const uint64_t E1 = min(E0 + (uint64_t)UNIT, T);
    uint32_t s = __ldcg(&in.ustart[unit]);
    for (;;) {
      __syncthreads();  // previous chunk fully consumed
      {
        const uint32_t t = threadIdx.x;
        const uint32_t idx = s + t;
        uint64_t eb = idx < n ? __ldcg((const unsigned long long *)&in.ebase[idx]) : T;
        s_eb[t] = eb;
        if (t == 0) {
          const uint32_t j = s + CHUNK;
          s_eb[CHUNK] = j < n ? __ldcg((const unsigned long long *)&in.ebase[j]) : T;
        }
        if (idx < n && eb < E1) {
          const uint32_t v = __ldcg(&in.vtx[idx]);
          s_vtx[t] = v;
          s_pay[t] = op.load(idx, v);
        }
      }
      __syncthreads();
      const uint64_t lo = max(E0, s_eb[0]);
      const uint64_t hi = min(E1, s_eb[CHUNK]);
      for (uint64_t base = lo; base < hi; base += RELAX_THREADS) {
        const uint64_t e = base + threadIdx.x;
        const bool valid = e < hi;
        bool app = false;
        uint32_t av = 0, ad = 0;
        if (valid) {
          // largest i with s_eb[i] <= e
          int l = 0, r = CHUNK - 1;
          while (l < r) {
            int m = (l + r + 1) >> 1;
            if (s_eb[m] <= e) l = m;
            else r = m - 1;
          }
          const uint32_t j = (uint32_t)(e - s_eb[l]);
          counted += op.visit(s_vtx[l], s_pay[l], j, app, av, ad);
        }
        if (Op::kAppends) frontier_append(out, app, av, ad);
      }
      if (s_eb[CHUNK] >= E1 || s + CHUNK >= n) break;
      s += CHUNK;
    }
  }
  if (edge_stat) {
    typedef cub::BlockReduce<unsigned long long, RELAX_THREADS> BR;
    __shared__ typename BR::TempStorage tmp;
    unsigned long long tot = BR(tmp).Sum((unsigned long long)counted);
    if (threadIdx.x == 0 && tot) atomicAdd(edge_stat, tot);
  }
}

}  // namespace sgs
