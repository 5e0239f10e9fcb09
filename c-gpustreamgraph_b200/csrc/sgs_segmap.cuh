// sgs_segmap.cuh -- the engine's load-balanced segmented map kernel
// (template only, so several translation units can instantiate it).
#pragma once
#include <cub/block/block_reduce.cuh>
#include <type_traits>
#include <utility>

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

// Ops that define touch(v, payload) are told once per frontier entry (by the
// CTA that owns the entry's first slot); PageRank's push counts hotness there.
template <class Op, class = void>
struct op_touches : std::false_type {};
template <class Op>
struct op_touches<Op, std::void_t<decltype(std::declval<const Op &>().touch(
                          0u, std::declval<const typename Op::Payload &>()))>> : std::true_type {};

// Ops either implement visit (one slot) or, with kQuad, visit4 (four
// consecutive slots j0..j0+3 of one block, j0 a multiple of 4; slots >= len
// are padding and must be ignored).
template <class Op>
__device__ __forceinline__ uint32_t visit_quad(const Op &op, uint32_t u,
                                               const typename Op::Payload &p, uint32_t j0,
                                               uint32_t len, bool (&app)[4], uint32_t (&av)[4],
                                               uint32_t (&ad)[4]) {
  if constexpr (Op::kQuad) {
    return op.visit4(u, p, j0, len, app, av, ad);
  } else {
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (j0 + k < len) c += op.visit(u, p, j0 + k, app[k], av[k], ad[k]);
    return c;
  }
}

// Each CTA walks one contiguous run of units [u_begin, u_end), staging up to
// CHUNK entries at a time in shared memory; each thread takes four
// consecutive positions per iteration.
template <class Op>
__global__ void __launch_bounds__(RELAX_THREADS)
    seg_map(FrontierView in, FrontierView out, Op op, unsigned long long *edge_stat) {
  using P = typename Op::Payload;
  __shared__ uint64_t s_eb[CHUNK + 1];
  __shared__ uint32_t s_len[CHUNK];
  __shared__ P s_pay[CHUNK];
  __shared__ uint32_t s_vtx[CHUNK];
  const uint64_t packed = __ldcg((const unsigned long long *)in.counter);
  const uint32_t n = (uint32_t)(packed >> CNT_SHIFT);
  const uint64_t T = packed & EDGE_MASK;
  uint64_t counted = 0;
  const uint64_t nunits = (T + UNIT - 1) / UNIT;
  const uint64_t ub = (uint64_t)blockIdx.x * nunits / gridDim.x;
  const uint64_t ue = (uint64_t)(blockIdx.x + 1) * nunits / gridDim.x;
  if (n != 0 && ub < ue) {
    const uint64_t E0 = ub * UNIT;
    const uint64_t E1 = min(ue * (uint64_t)UNIT, T);
    uint32_t s = __ldcg(&in.ustart[ub]);
    for (;;) {
      __syncthreads();  // previous chunk fully consumed
      {
        const uint32_t t = threadIdx.x;
        const uint32_t idx = s + t;
        const uint64_t eb = idx < n ? __ldcg((const unsigned long long *)&in.ebase[idx]) : T;
        s_eb[t] = eb;
        if (t == 0) {
          const uint32_t j = s + CHUNK;
          s_eb[CHUNK] = j < n ? __ldcg((const unsigned long long *)&in.ebase[j]) : T;
        }
        if (idx < n && eb < E1) {
          const uint32_t v = __ldcg(&in.vtx[idx]);
          s_vtx[t] = v;
          s_len[t] = __ldcg(&in.len[idx]);
          s_pay[t] = op.load(idx, v);
          if constexpr (op_touches<Op>::value)
            if (eb >= E0) op.touch(v, s_pay[t]);
        }
      }
      __syncthreads();
      const uint64_t lo = max(E0, s_eb[0]);
      const uint64_t hi = min(E1, s_eb[CHUNK]);
      for (uint64_t base = lo; base < hi; base += 4 * RELAX_THREADS) {
        const uint64_t e = base + 4 * threadIdx.x;
        bool app[4] = {false, false, false, false};
        uint32_t av[4] = {0, 0, 0, 0}, ad[4] = {0, 0, 0, 0};
        if (e < hi) {
          // largest i with s_eb[i] <= e
          int l = 0, r = CHUNK - 1;
          while (l < r) {
            const int m = (l + r + 1) >> 1;
            if (s_eb[m] <= e) l = m;
            else r = m - 1;
          }
          const uint32_t j0 = (uint32_t)(e - s_eb[l]);
          if (j0 < s_len[l]) counted += visit_quad(op, s_vtx[l], s_pay[l], j0, s_len[l], app, av, ad);
        }
        if (Op::kAppends) {
#pragma unroll
          for (int k = 0; k < 4; ++k) frontier_append(out, app[k], av[k], ad[k]);
        }
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
