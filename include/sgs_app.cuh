// sgs_app.cuh -- user algorithms written as AppBase functors, run by the
// streaming-graph engine on its snapshot path.
//
// The reference's plugin surface is sepgraph::api::AppBase<TValue, TBuffer,
// TWeight> (include/framework/variants/api.cuh:22-160): a user derives a
// functor struct from it -- GetInitValue / GetInitBuffer /
// GetIdentityElement, CombineValueBuffer(Amend), AccumulateBuffer(_add,
// _del), IsActiveNode(_INC) -- and instantiates
// Engine<TValue, TBuffer, TWeight, TAppImpl, Args...> with it
// (include/framework/framework.cuh:77-140); samples/hybrid_{bfs,sssp,cc,pr}
// are such structs.  This header keeps those names and signatures.  The
// engine (libsgs.so) is compiled once; this header's kernels are templates,
// instantiated for the user's functor in the user's own translation unit, so
// every functor call is a direct, inlinable call -- no device virtual
// functions (CUDA leaves a virtual call on an object built in host code
// undefined, and the reference passes host-built functors to its kernels).
// The library reaches the functor kernels through the plain-C hooks of
// sgs.h (sgs_app_attach): every sgs_apply_batch updates the graph, the
// built-in queries and every attached user algorithm in one snapshot.
//
// Build: nvcc -std=c++17 -gencode arch=compute_100a,code=sm_100a
//        -I <repo>/include -I <repo>/c-gpustreamgraph_b200/csrc ... -lsgs
//
// What the engine does with a functor (per the reference's data-driven
// push variant, framework.cuh:549-584 and variants/sync_push_dd.cuh:170-268):
//
//   state     value[v] (TValue), and one record per vertex holding parent[v]
//             (TValue) and buffer[v] (TBuffer) side by side: when both are 4
//             bytes the record is one aligned 8-byte word, parent in the low
//             half, so a functor may update (buffer, parent) with one 64-bit
//             atomic (min_with_parent / max_with_parent below) and parents
//             stay consistent with the values they explain.
//   start     value = GetInitValue(v), buffer = GetInitBuffer(v), parent = all
//             ones; the first frontier = vertices IsActiveNode (or _INC).
//   round     for each frontier vertex v: (b, push) = CombineValueBuffer(v,
//             &value[v], &buffer[v]); if push, for every live out-edge (v,u,w)
//             AccumulateBuffer(v, u, w, &parent[u], &buffer[u], b); a
//             destination that IsActiveNode (or _INC) afterwards joins the
//             next frontier (once).  Combine runs in its own launch, so no
//             accumulation races with the fold of value and buffer.  Rounds
//             end when a frontier is empty.
//   snapshot  two families (app_traits<App>::accumulative; default: floating
//             point TValue):
//     monotone (BFS/SSSP/CC style): before the graph changes,
//             AccumulateBuffer_del(u, v, &parent[v], &buffer[v], &value[v])
//             for every deleted edge, then for every out-edge of each vertex
//             the functor marked with m_vcsr_graph.vertices_[v].deletion =
//             true, until no new vertex is marked (the reference's
//             reset_del_edges + SyncPushDDB_del, variants/driver.cuh:398-430);
//             after it, if anything was marked, every vertex whose value is
//             not GetIdentityElement() pushes its value along its out-edges
//             (the reference's SyncPushDDBAll, framework.cuh:1507-1560),
//             else only the kept inserted edges are accumulated; then rounds.
//     accumulative (PageRank style): each source whose out-list changes
//             pushes CombineValueBufferAmend(v, type, ...) along its old list
//             with *type = -1 before the update and along its new list with
//             *type = +1 after it (Cancelation / Compensate,
//             framework.cuh:1110-1301); then the active vertices run rounds.
//   weights   TWeight(w): stored weights (SGS_W_EXPLICIT), the reference's
//             synthesized (u+v)%128+1 (SGS_W_SYNTH, push_functor.h:306) or 1.
//
// Device graph view the functors read: m_vcsr_graph.vertices_[v].degree and
// .sync_vertices_[v].degree (live out-degree), vertices_[v].deletion (read
// and set), plus m_nnodes, m_nedges and *m_p_current_round.
//
// Drop-in names: unless SGS_APP_NO_REFERENCE_NAMES is defined, the header
// also declares sepgraph::api::AppBase, sepgraph::engine::Engine, utils::pair
// and a global index_t, the names the sample sources use.  The samples mark
// their overrides with `override`; here the base has no virtual functions, so
// either drop the keyword or define SGS_APP_ACCEPT_OVERRIDE before including
// this header (it then defines `override` away; include it after the
// standard headers the file uses).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "sgs.h"
#include "sgs_engine.hpp"
#include "sgs_segmap.cuh"

namespace sgs {
namespace api {

using index_t = uint32_t;

template <typename A, typename B>
struct pair {
  A first;
  B second;
  __host__ __device__ pair() : first(), second() {}
  __host__ __device__ pair(const A &a, const B &b) : first(a), second(b) {}
};

// ---- the device view of the dynamic graph that functors read ------------
struct DegreeRef {  // live out-degree of one vertex
  const uint32_t *live;
  index_t v;
  __device__ __forceinline__ operator uint32_t() const { return __ldg(live + v); }
};
struct DeletionRef {  // the "reset in this snapshot" mark of one vertex
  uint32_t *bits;
  index_t v;
  __device__ __forceinline__ const DeletionRef &operator=(bool b) const {
    if (b) atomicOr(&bits[v >> 5], 1u << (v & 31));
    else atomicAnd(&bits[v >> 5], ~(1u << (v & 31)));
    return *this;
  }
  __device__ __forceinline__ operator bool() const { return (__ldcg(&bits[v >> 5]) >> (v & 31)) & 1u; }
};
struct VertexRef {
  DegreeRef degree;
  DeletionRef deletion;
};
struct VertexArray {
  const uint32_t *live = nullptr;
  uint32_t *del_bits = nullptr;
  __device__ __forceinline__ VertexRef operator[](index_t v) const {
    return VertexRef{DegreeRef{live, v}, DeletionRef{del_bits, v}};
  }
};
struct PMAView {
  uint32_t nnodes = 0;
  uint64_t nedges = 0;
  VertexArray vertices_;       // .degree, .deletion
  VertexArray sync_vertices_;  // .degree (the reference's synced copy)
  __device__ __forceinline__ uint32_t out_degree(index_t v) const { return __ldg(vertices_.live + v); }
};

// ---- the functor base ----------------------------------------------------
// Non-virtual: the engine calls the derived struct's own members (a missing
// required one is a compile error where the engine needs it).  Defaults are
// given for the members some algorithm families never use.
template <typename TValue, typename TBuffer, typename TWeight>
struct AppBase {
  // AccumulateBuffer return codes of the reference ([ACCUMULATE][CONTINUE])
  static constexpr int ACCUMULATE_SUCCESS_BREAK = 0;
  static constexpr int ACCUMULATE_SUCCESS_CONTINUE = 1;
  static constexpr int ACCUMULATE_FAILURE_BREAK = 2;
  static constexpr int ACCUMULATE_FAILURE_CONTINUE = 3;

  PMAView m_vcsr_graph;
  uint32_t m_nnodes = 0;
  uint32_t m_nedges = 0;
  uint32_t *m_p_current_round = nullptr;

  // PageRank-style amend: unused by monotone algorithms.
  __device__ __forceinline__ pair<TBuffer, bool> CombineValueBufferAmend(index_t, int *, TValue *,
                                                                        TBuffer *p_buffer) {
    return pair<TBuffer, bool>(*p_buffer, false);
  }
  // Never called by the engine (nor by the reference's framework).
  __device__ __forceinline__ int AccumulateBuffer_add(index_t, index_t, TWeight, TValue *, TBuffer *,
                                                     TBuffer *) {
    return 0;
  }
  __device__ __forceinline__ bool IsActiveNode_INC(index_t, TBuffer, TValue) const { return false; }
  // Scheduling hints of the reference's priority variants; unused here.
  __device__ __forceinline__ TValue sum_value(index_t, TValue value, TBuffer) const { return value; }
  __device__ __forceinline__ bool IsHighPriority(TBuffer, TBuffer) const { return true; }
  __device__ __forceinline__ void PostComputation() {}
};

// Strict minimum of the (buffer, parent) record of one vertex: stores
// (cand, src) only when cand is strictly below the current buffer, so a
// parent changes only with a strictly better value and parent chains cannot
// form cycles (which the deletion phase relies on).  Needs the 8-byte record
// layout (4-byte TValue and TBuffer, buffer an unsigned integer); p_buffer
// must be the buffer of the record that p_parent starts.  Returns true when
// it stored.
template <typename TValue, typename TBuffer>
__device__ __forceinline__ bool min_with_parent(TValue *p_parent, TBuffer *p_buffer, TBuffer cand,
                                                index_t src) {
  static_assert(sizeof(TValue) == 4 && sizeof(TBuffer) == 4 && std::is_unsigned<TBuffer>::value,
                "min_with_parent needs 4-byte parents and unsigned 4-byte buffers");
  (void)p_buffer;
  unsigned long long *w = reinterpret_cast<unsigned long long *>(p_parent);
  unsigned long long old = __ldcg(w);
  const unsigned long long nw = ((unsigned long long)cand << 32) | src;
  while ((uint32_t)(old >> 32) > (uint32_t)cand) {
    const unsigned long long prev = atomicCAS(w, old, nw);
    if (prev == old) return true;
    old = prev;
  }
  return false;
}
// The same for maximisation (widest paths and the like).
template <typename TValue, typename TBuffer>
__device__ __forceinline__ bool max_with_parent(TValue *p_parent, TBuffer *p_buffer, TBuffer cand,
                                                index_t src) {
  static_assert(sizeof(TValue) == 4 && sizeof(TBuffer) == 4 && std::is_unsigned<TBuffer>::value,
                "max_with_parent needs 4-byte parents and unsigned 4-byte buffers");
  (void)p_buffer;
  unsigned long long *w = reinterpret_cast<unsigned long long *>(p_parent);
  unsigned long long old = __ldcg(w);
  const unsigned long long nw = ((unsigned long long)cand << 32) | src;
  while ((uint32_t)(old >> 32) < (uint32_t)cand) {
    const unsigned long long prev = atomicCAS(w, old, nw);
    if (prev == old) return true;
    old = prev;
  }
  return false;
}

// ---- traits ----------------------------------------------------------------
template <class App, class = void>
struct has_accumulative_flag : std::false_type {};
template <class App>
struct has_accumulative_flag<App, std::void_t<decltype(App::kAccumulative)>> : std::true_type {};

// accumulative: the PageRank family (deltas pushed and summed, snapshots by
// cancel/compensate); otherwise the monotone family (parent-tree
// invalidation).  A functor states it with `static constexpr bool
// kAccumulative`; without it, floating-point values mean accumulative.
template <class App, class TValue>
struct app_traits {
  static constexpr bool accumulative = [] {
    if constexpr (has_accumulative_flag<App>::value) return (bool)App::kAccumulative;
    else return std::is_floating_point<TValue>::value;
  }();
};

}  // namespace api

namespace app_detail {

using api::index_t;

// One vertex's parent and buffer, adjacent (see the header comment).
template <class V, class B>
struct alignas((sizeof(V) + sizeof(B) <= 8) ? 8 : 16) Rec {
  V parent;
  B buffer;
};

template <class T>
__device__ __forceinline__ T ld_fresh(const T *p) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte value types");
  T t;
  if constexpr (sizeof(T) == 4) {
    const unsigned int x = __ldcg(reinterpret_cast<const unsigned int *>(p));
    memcpy(&t, &x, 4);
  } else {
    const unsigned long long x = __ldcg(reinterpret_cast<const unsigned long long *>(p));
    memcpy(&t, &x, 8);
  }
  return t;
}

template <class V, class B>
struct State {
  V *value;
  Rec<V, B> *rec;
  B *pushval;         // what a scheduled vertex pushes this round
  uint32_t *stamp;    // frontier claims (tag of the frontier a vertex joined last)
  uint32_t *del_bits; // vertices marked by the deletion phase of this snapshot
  uint32_t *round;    // *m_p_current_round
  unsigned long long *resets;  // vertices marked in this snapshot
};

__device__ __forceinline__ bool claim(uint32_t *stamp, uint32_t v, uint32_t tag) {
  return __ldcg(&stamp[v]) != tag && atomicExch(&stamp[v], tag) != tag;
}

template <class App, class V, class B>
__device__ __forceinline__ bool active(App &app, uint32_t v, B buf, V val) {
  return app.IsActiveNode(v, buf, val) || app.IsActiveNode_INC(v, buf, val);
}

__device__ __forceinline__ uint32_t weight_at(const GraphView &g, uint64_t off, uint32_t j, uint32_t u,
                                              uint32_t dst) {
  if (g.wmode == W_EXPLICIT) return __ldg(wgt_at(g, off, j));
  if (g.wmode == W_SYNTH) return (u + dst) % 128u + 1u;
  return 1u;
}

template <class App, class V, class B>
__global__ void k_init(App app, State<V, B> s, uint32_t nv) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    s.value[v] = app.GetInitValue((index_t)v);
    s.rec[v].buffer = app.GetInitBuffer((index_t)v);
    memset(&s.rec[v].parent, 0xFF, sizeof(V));
    s.stamp[v] = 0;
  }
}

// Every vertex the functor calls active joins `out` (claimed with tag).
template <class App, class V, class B>
__global__ void __launch_bounds__(RELAX_THREADS) k_active_scan(App app, State<V, B> s, uint32_t nv,
                                                               uint32_t tag, FrontierView out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < nv; b += stride) {
    const uint64_t v = b + threadIdx.x;
    bool want = false;
    if (v < nv)
      want = active(app, (uint32_t)v, s.rec[v].buffer, s.value[v]) && claim(s.stamp, (uint32_t)v, tag);
    frontier_append_block(out, want, (uint32_t)v, 0u);
  }
}

// Combine of one round: the frontier's vertices fold their buffers; those
// that schedule a push join `pout` with their out-block.
template <class App, class V, class B>
__global__ void k_combine(App app, GraphView g, State<V, B> s, FrontierView fin, FrontierView pout,
                          uint32_t round) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *s.round = round;
  const uint32_t n = (uint32_t)(__ldcg((const unsigned long long *)fin.counter) >> CNT_SHIFT);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    bool want = false;
    uint32_t v = 0, d = 0;
    if (i < n) {
      v = __ldcg(&fin.vtx[i]);
      const api::pair<B, bool> pr = app.CombineValueBuffer(v, &s.value[v], &s.rec[v].buffer);
      if (pr.second) {
        d = g.slots[v];
        if (d) {
          s.pushval[v] = pr.first;
          want = true;
        }
      }
    }
    frontier_append(pout, want, v, d);
  }
}

// AccumulateBuffer over the out-blocks of a push frontier; destinations that
// become active join the next frontier (when `activate`).
template <class App, class V, class B, class W>
struct PushOp {
  static constexpr bool kAppends = true;
  static constexpr bool kQuad = false;
  struct Payload {
    uint64_t off;
    B buf;
  };
  mutable App app;
  GraphView g;
  State<V, B> s;
  uint32_t tag;
  int activate;
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const {
    Payload p;
    p.off = g.off[v];
    p.buf = s.pushval[v];
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t u, const Payload &p, uint32_t j, bool &ap, uint32_t &av,
                                            uint32_t &ad) const {
    const uint32_t dst = __ldg(adj_at(g, p.off, j));
    if (dst == SGS_TOMB) return 0;
    const uint32_t w = weight_at(g, p.off, j, u, dst);
    app.AccumulateBuffer(u, dst, (W)w, &s.rec[dst].parent, &s.rec[dst].buffer, p.buf);
    if (activate && active(app, dst, ld_fresh(&s.rec[dst].buffer), ld_fresh(&s.value[dst])) &&
        claim(s.stamp, dst, tag)) {
      ap = true;
      av = dst;
      ad = 0;
    }
    return 1;
  }
};

// Deletion phase, seeds: every deleted edge (u,v) meets v's state.
template <class App, class V, class B>
__global__ void k_del_seed(App app, GraphView g, State<V, B> s, const uint64_t *keys, uint64_t n,
                           uint32_t tag, FrontierView out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    bool want = false;
    uint32_t v = 0, d = 0;
    if (i < n) {
      const uint64_t k = keys[i];
      const uint32_t u = (uint32_t)(k >> 32);
      v = (uint32_t)k;
      app.AccumulateBuffer_del(u, v, &s.rec[v].parent, &s.rec[v].buffer, &s.value[v]);
      if (bit_at(s.del_bits, v) && claim(s.stamp, v, tag)) {
        atomicAdd(s.resets, 1ull);
        d = g.slots[v];
        want = d != 0;
      }
    }
    frontier_append(out, want, v, d);
  }
}

// Deletion phase, propagation over the out-edges of marked vertices.
template <class App, class V, class B>
struct DelOp {
  static constexpr bool kAppends = true;
  static constexpr bool kQuad = false;
  struct Payload {
    uint64_t off;
  };
  mutable App app;
  GraphView g;
  State<V, B> s;
  uint32_t tag;
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const { return Payload{g.off[v]}; }
  __device__ __forceinline__ uint32_t visit(uint32_t u, const Payload &p, uint32_t j, bool &ap, uint32_t &av,
                                            uint32_t &ad) const {
    const uint32_t dst = __ldg(adj_at(g, p.off, j));
    if (dst == SGS_TOMB) return 0;
    app.AccumulateBuffer_del(u, dst, &s.rec[dst].parent, &s.rec[dst].buffer, &s.value[dst]);
    if (bit_at(s.del_bits, dst) && claim(s.stamp, dst, tag)) {
      atomicAdd(s.resets, 1ull);
      const uint32_t d = g.slots[dst];
      if (d) {
        ap = true;
        av = dst;
        ad = d;
      }
    }
    return 1;
  }
};

// Repair after marks: every vertex whose value is not the identity pushes
// its value along its out-block.
template <class App, class V, class B>
__global__ void __launch_bounds__(RELAX_THREADS) k_sweep(App app, GraphView g, State<V, B> s,
                                                         FrontierView pout) {
  const V id = static_cast<V>(app.GetIdentityElement());
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < g.nv; b += stride) {
    const uint64_t v = b + threadIdx.x;
    bool want = false;
    uint32_t d = 0;
    if (v < g.nv) {
      d = g.slots[v];
      const V val = s.value[v];
      if (d && !(val == id)) {
        s.pushval[v] = static_cast<B>(val);
        want = true;
      }
    }
    frontier_append_block(pout, want, (uint32_t)v, want ? d : 0u);
  }
}

// Repair without marks: only the kept inserted edges (u,v,w).
template <class App, class V, class B, class W>
__global__ void k_inserted(App app, GraphView g, State<V, B> s, const uint64_t *keys, const uint32_t *wts,
                           const uint32_t *n_ptr, uint32_t tag, FrontierView out, unsigned long long *edges) {
  const uint32_t n = *n_ptr;
  const V id = static_cast<V>(app.GetIdentityElement());
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t counted = 0;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    bool want = false;
    uint32_t v = 0;
    if (i < n) {
      const uint64_t k = keys[i];
      const uint32_t u = (uint32_t)(k >> 32);
      v = (uint32_t)k;
      const V val = s.value[u];
      if (!(val == id)) {
        const uint32_t w = g.wmode == W_EXPLICIT ? wts[i] : g.wmode == W_SYNTH ? (u + v) % 128u + 1u : 1u;
        app.AccumulateBuffer(u, v, (W)w, &s.rec[v].parent, &s.rec[v].buffer, static_cast<B>(val));
        ++counted;
        want = active(app, v, ld_fresh(&s.rec[v].buffer), ld_fresh(&s.value[v])) && claim(s.stamp, v, tag);
      }
    }
    frontier_append(out, want, v, 0u);
  }
  if (counted) atomicAdd(edges, (unsigned long long)counted);
}

// Accumulative family: the distinct sources of the deleted and kept inserted
// edges amend once each (CombineValueBufferAmend with *type), and those that
// schedule a push join `pout` with their current out-block.
template <class App, class V, class B>
__global__ void k_amend(App app, GraphView g, State<V, B> s, const uint64_t *dkeys, uint64_t nd,
                        const uint64_t *ikeys, const uint32_t *ni_ptr, uint32_t tag, int *type,
                        FrontierView pout) {
  const uint64_t ni = ikeys ? *ni_ptr : 0;
  const uint64_t n = nd + ni;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x; b < n; b += stride) {
    const uint64_t i = b + threadIdx.x;
    bool want = false;
    uint32_t v = 0, d = 0;
    if (i < n) {
      const bool del = i < nd;
      const uint64_t *ks = del ? dkeys : ikeys;
      const uint64_t k = del ? i : i - nd;
      v = (uint32_t)(ks[k] >> 32);
      const bool head = k == 0 || (uint32_t)(ks[k - 1] >> 32) != v;
      if (head && claim(s.stamp, v, tag)) {
        const api::pair<B, bool> pr = app.CombineValueBufferAmend(v, type, &s.value[v], &s.rec[v].buffer);
        if (pr.second) {
          d = g.slots[v];
          if (d) {
            s.pushval[v] = pr.first;
            want = true;
          }
        }
      }
    }
    frontier_append(pout, want, v, d);
  }
}

template <int = 0>
__global__ void k_set_types(int *t) {
  t[0] = -1;
  t[1] = 1;
}

inline GraphView graph_of(const sgs_graph_view &v) {
  GraphView g{};
  g.nv = v.nv;
  g.off = v.off;
  g.slots = v.slots;
  g.live = v.live;
  g.cap = v.cap;
  g.adj_d = v.adj_d;
  g.wgt_d = v.wgt_d;
  g.adj_h = v.adj_h;
  g.wgt_h = v.wgt_h;
  g.wmode = v.weight_mode;
  g.cmap = v.cmap;
  g.adj_c = v.adj_c;
  g.wgt_c = v.wgt_c;
  g.cbase = v.cbase;
  return g;
}

inline void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(SGS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

template <class T>
struct DevArr {
  T *p = nullptr;
  size_t n = 0;
  void ensure(size_t m) {
    if (m <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (cudaMalloc((void **)&p, sizeof(T) * m) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      throw Error(SGS_ERR_OOM, "device allocation failed (user algorithm state)");
    }
    n = m;
  }
  ~DevArr() {
    if (p) cudaFree(p);
  }
};

}  // namespace app_detail

namespace app {

// Statistics of the last start or snapshot of a user algorithm.
struct Stats {
  uint64_t edges_traversed = 0;  // out-edges walked by pushes and the deletion phase
  uint64_t resets = 0;           // vertices the deletion phase marked
  uint32_t rounds = 0;           // combine/push rounds
  uint32_t converged = 0;
  double ms = 0;                 // device time
};

// One user algorithm (functor App over TValue/TBuffer/TWeight) attached to an
// engine: its state lives in HBM, and every snapshot the engine applies
// updates it through the hooks.  Not copyable; detaches on destruction.
template <class App, typename TValue, typename TBuffer, typename TWeight>
class Query {
  using V = TValue;
  using B = TBuffer;
  using W = TWeight;
  using St = app_detail::State<V, B>;
  static constexpr bool kAcc = api::app_traits<App, V>::accumulative;
  static_assert(sizeof(V) <= 8 && sizeof(B) <= 8, "value and buffer types of at most 8 bytes");

 public:
  Query(sgs_engine *e, const App &app, uint32_t max_rounds = 1000) : e_(e), app_(app), max_rounds_(max_rounds) {
    sgs_graph_view g{};
    check(sgs_get_graph_view(e_, &g));
    app_detail::ck(cudaSetDevice(g.device), "cudaSetDevice");
    nv_ = g.nv;
    s_ = (cudaStream_t)g.stream;
    int dev = g.device;
    app_detail::ck(cudaDeviceGetAttribute(&nsm_, cudaDevAttrMultiProcessorCount, dev), "attribute");
    value_.ensure(nv_);
    rec_.ensure(nv_);
    push_.ensure(nv_);
    stamp_.ensure(nv_);
    bits_.ensure(nv_ / 32 + 1);
    misc_.ensure(4);
    types_.ensure(2);
    cnt_.ensure(3 * (size_t)(max_rounds_ + 2));
    for (auto &f : fr_) {
      f.vtx.ensure((size_t)nv_ + 1);
      f.len.ensure((size_t)nv_ + 1);
      f.ebase.ensure((size_t)nv_ + 1);
    }
    app_detail::k_set_types<><<<1, 1, 0, s_>>>(types_.p);
    app_detail::ck(cudaEventCreate(&ev0_), "event");
    app_detail::ck(cudaEventCreate(&ev1_), "event");
    sgs_app_hooks h{this, &Query::hook_before, &Query::hook_after};
    check(sgs_app_attach(e_, &h, &id_));
  }
  ~Query() {
    if (id_ > 0) sgs_app_detach(e_, id_);
    if (s_) cudaStreamSynchronize(s_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
  }
  Query(const Query &) = delete;
  Query &operator=(const Query &) = delete;

  App &app() { return app_; }
  const Stats &stats() const { return st_; }
  uint32_t nv() const { return nv_; }

  // InitGraph + Start: initial state and convergence on the current graph.
  void start() {
    sgs_graph_view g{};
    check(sgs_get_graph_view(e_, &g));
    prepare(g);
    st_ = Stats{};
    phase_begin();
    app_detail::k_init<App, V, B><<<grid_elem(nv_), 256, 0, s_>>>(app_, state(), nv_);
    reset_counters();
    const uint32_t t = next_tag();
    app_detail::k_active_scan<App, V, B><<<grid_elem(nv_), RELAX_THREADS, 0, s_>>>(app_, state(), nv_, t,
                                                                                 fview(0, fcnt(0)));
    launch_check();
    rounds_from(g, 0);
    phase_end(true);
    started_ = true;
  }

  // Per-vertex results (host copies).
  std::vector<V> values() {
    std::vector<V> out(nv_);
    app_detail::ck(cudaMemcpyAsync(out.data(), value_.p, sizeof(V) * nv_, cudaMemcpyDeviceToHost, s_), "copy");
    sync();
    return out;
  }
  std::vector<app_detail::Rec<V, B>> records() {
    std::vector<app_detail::Rec<V, B>> out(nv_);
    app_detail::ck(cudaMemcpyAsync(out.data(), rec_.p, sizeof(out[0]) * nv_, cudaMemcpyDeviceToHost, s_), "copy");
    sync();
    return out;
  }
  std::vector<V> parents() {
    std::vector<V> out(nv_);
    auto r = records();
    for (uint32_t v = 0; v < nv_; ++v) out[v] = r[v].parent;
    return out;
  }
  std::vector<B> buffers() {
    std::vector<B> out(nv_);
    auto r = records();
    for (uint32_t v = 0; v < nv_; ++v) out[v] = r[v].buffer;
    return out;
  }

 private:
  struct Buf {
    app_detail::DevArr<uint32_t> vtx, len, ustart;
    app_detail::DevArr<uint64_t> ebase;
  };

  static int hook_before(void *ctx, const sgs_graph_view *g, const sgs_update_view *u) {
    return guard([&] { static_cast<Query *>(ctx)->before_update(*g, *u); });
  }
  static int hook_after(void *ctx, const sgs_graph_view *g, const sgs_update_view *u) {
    return guard([&] { static_cast<Query *>(ctx)->after_update(*g, *u); });
  }
  template <class F>
  static int guard(F &&f) {
    try {
      f();
      return SGS_OK;
    } catch (const Error &err) {
      sgs_set_last_error(err.what());
      return err.code;
    } catch (const std::exception &err) {
      sgs_set_last_error(err.what());
      return SGS_ERR_CUDA;
    }
  }

  // the deletion phase (monotone) or the cancellation (accumulative), on
  // the old graph
  void before_update(const sgs_graph_view &g, const sgs_update_view &u) {
    if (!started_) return;
    prepare(g);
    st_ = Stats{};
    phase_begin();
    reset_counters();
    const GraphView gv = app_detail::graph_of(g);
    marked_ = false;
    if constexpr (kAcc) {
      amend(gv, u, 0);
    } else if (u.n_del) {
      app_detail::ck(cudaMemsetAsync(bits_.p, 0, sizeof(uint32_t) * (nv_ / 32 + 1), s_), "memset");
      const uint32_t t = next_tag();
      app_detail::k_del_seed<App, V, B><<<grid_elem(u.n_del), 256, 0, s_>>>(app_, gv, state(), u.del_keys,
                                                                           u.n_del, t, fview(0, dcnt(0)));
      launch_check();
      // propagation rounds until no vertex is newly marked
      uint32_t r = 0;
      for (;; ++r) {
        if (r >= max_rounds_) throw Error(SGS_ERR_NOCONV, "deletion phase of a user algorithm did not converge");
        unsigned long long c = 0;
        app_detail::ck(cudaMemcpyAsync(&c, dcnt(r), sizeof(c), cudaMemcpyDeviceToHost, s_), "copy");
        sync();
        if ((c >> CNT_SHIFT) == 0) break;
        app_detail::DelOp<App, V, B> op{app_, gv, state(), t};
        seg_map<<<grid_map(), RELAX_THREADS, 0, s_>>>(fview(r % 2, dcnt(r)), fview((r + 1) % 2, dcnt(r + 1)), op,
                                                        misc_.p + 0);
        launch_check();
      }
      unsigned long long resets = 0;
      app_detail::ck(cudaMemcpyAsync(&resets, misc_.p + 1, sizeof(resets), cudaMemcpyDeviceToHost, s_), "copy");
      sync();
      marked_ = resets != 0;
    }
    phase_end(false);
  }

  // the repair and convergence (monotone) or the compensation and
  // convergence (accumulative), on the new graph
  void after_update(const sgs_graph_view &g, const sgs_update_view &u) {
    if (!started_) return;
    prepare(g);
    phase_begin();
    const GraphView gv = app_detail::graph_of(g);
    if constexpr (kAcc) {
      amend(gv, u, 1);
      reset_round_counters();
      const uint32_t t = next_tag();
      app_detail::k_active_scan<App, V, B><<<grid_elem(nv_), RELAX_THREADS, 0, s_>>>(app_, state(), nv_, t,
                                                                                   fview(0, fcnt(0)));
      launch_check();
      rounds_from(g, 0);
    } else {
      reset_round_counters();
      const uint32_t t = next_tag();
      if (marked_) {
        // every reached vertex re-pushes (into frontier 1 of round 0), then
        // the marked vertices that are active by themselves join it
        app_detail::k_sweep<App, V, B><<<grid_elem(nv_), RELAX_THREADS, 0, s_>>>(app_, gv, state(),
                                                                               pview(pcnt(0)));
        app_detail::PushOp<App, V, B, W> op{app_, gv, state(), t, 1};
        seg_map<<<grid_map(), RELAX_THREADS, 0, s_>>>(pview(pcnt(0)), fview(1, fcnt(1)), op, misc_.p + 0);
        app_detail::k_active_scan<App, V, B><<<grid_elem(nv_), RELAX_THREADS, 0, s_>>>(app_, state(), nv_, t,
                                                                                     fview(1, fcnt(1)));
      } else if (u.n_ins_max) {
        app_detail::k_inserted<App, V, B, W><<<grid_elem(u.n_ins_max), 256, 0, s_>>>(
            app_, gv, state(), u.ins_keys, u.ins_w, u.n_ins, t, fview(1, fcnt(1)), misc_.p + 0);
      }
      launch_check();
      rounds_from(g, 1);
    }
    phase_end(true);
  }

  // accumulative: CombineValueBufferAmend of the touched sources with
  // *type = -1 (before) or +1 (after), pushed along their current lists
  void amend(const GraphView &gv, const sgs_update_view &u, int which) {
    if (!u.n_del && !u.n_ins_max) return;
    const uint32_t t = next_tag();
    unsigned long long *pc = pcnt(which);
    app_detail::ck(cudaMemsetAsync(pc, 0, sizeof(unsigned long long), s_), "memset");
    app_detail::k_amend<App, V, B><<<grid_elem(u.n_del + u.n_ins_max), 256, 0, s_>>>(
        app_, gv, state(), u.del_keys, u.n_del, u.n_ins_max ? u.ins_keys : nullptr, u.n_ins, t,
        types_.p + which, pview(pc));
    app_detail::PushOp<App, V, B, W> op{app_, gv, state(), 0u, 0};
    seg_map<<<grid_map(), RELAX_THREADS, 0, s_>>>(pview(pc), fview(1, fcnt(max_rounds_ + 1)), op, misc_.p + 0);
    launch_check();
  }

  // Rounds from frontier `r0` (buffer r0 % 2, counter fcnt(r0)) until one is
  // empty; the counters of a batch of rounds are read once.
  void rounds_from(const sgs_graph_view &g, uint32_t r0) {
    const GraphView gv = app_detail::graph_of(g);
    uint32_t r = r0, nb = 2;
    std::vector<unsigned long long> h(20);
    st_.converged = 0;
    while (r < max_rounds_) {
      const uint32_t k = std::min(nb, max_rounds_ - r);
      for (uint32_t q = 0; q < k; ++q) {
        const uint32_t rr = r + q;
        app_detail::k_combine<App, V, B><<<grid_elem(nv_), 256, 0, s_>>>(app_, gv, state(), fview(rr % 2, fcnt(rr)),
                                                                        pview(pcnt(rr)), rr);
        app_detail::PushOp<App, V, B, W> op{app_, gv, state(), next_tag(), 1};
        seg_map<<<grid_map(), RELAX_THREADS, 0, s_>>>(pview(pcnt(rr)), fview((rr + 1) % 2, fcnt(rr + 1)), op,
                                                        misc_.p + 0);
      }
      launch_check();
      app_detail::ck(cudaMemcpyAsync(h.data(), fcnt(r + 1), sizeof(unsigned long long) * k,
                                     cudaMemcpyDeviceToHost, s_),
                     "copy");
      sync();
      for (uint32_t q = 0; q < k; ++q)
        if ((h[q] >> CNT_SHIFT) == 0) {
          st_.rounds = r + q + 1 - r0;
          st_.converged = 1;
          return;
        }
      r += k;
      nb = std::min<uint32_t>(nb * 2, 16);
    }
    st_.rounds = r - r0;
    throw Error(SGS_ERR_NOCONV, "user algorithm: round limit reached before convergence");
  }

  // Sizes the frontiers for the current layout and refreshes the functor's
  // graph view.
  void prepare(const sgs_graph_view &g) {
    if (g.nv != nv_) throw Error(SGS_ERR_STATE, "the engine's graph changed size under a user algorithm");
    const uint64_t max_pos = g.slots_total + 3ull * nv_;
    const uint32_t need = (uint32_t)std::min<uint64_t>(max_pos / UNIT + 2, 0xFFFFFFF0ull);
    for (auto &f : fr_) f.ustart.ensure(need);
    ucap_ = need;
    app_.m_vcsr_graph.nnodes = nv_;
    app_.m_vcsr_graph.nedges = g.ne;
    app_.m_vcsr_graph.vertices_.live = g.live;
    app_.m_vcsr_graph.vertices_.del_bits = bits_.p;
    app_.m_vcsr_graph.sync_vertices_ = app_.m_vcsr_graph.vertices_;
    app_.m_nnodes = nv_;
    app_.m_nedges = (uint32_t)std::min<uint64_t>(g.ne, 0xFFFFFFFFull);
    app_.m_p_current_round = round_p();
  }

  St state() {
    return St{value_.p, rec_.p, push_.p, stamp_.p, bits_.p, round_p(), misc_.p + 1};
  }
  uint32_t *round_p() { return reinterpret_cast<uint32_t *>(misc_.p + 2); }
  // frontier views: buffers 0 and 1 for frontiers, 2 for the push list
  FrontierView fview(uint32_t b, unsigned long long *c) {
    FrontierView f;
    f.vtx = fr_[b].vtx.p;
    f.len = fr_[b].len.p;
    f.ebase = fr_[b].ebase.p;
    f.ustart = fr_[b].ustart.p;
    f.counter = (uint64_t *)c;
    f.ucap = ucap_;
    return f;
  }
  FrontierView pview(unsigned long long *c) { return fview(2, c); }
  unsigned long long *fcnt(uint32_t r) { return cnt_.p + r; }
  unsigned long long *pcnt(uint32_t r) { return cnt_.p + (max_rounds_ + 2) + r; }
  unsigned long long *dcnt(uint32_t r) { return cnt_.p + 2 * (max_rounds_ + 2) + r; }
  void reset_counters() {
    app_detail::ck(cudaMemsetAsync(cnt_.p, 0, sizeof(unsigned long long) * cnt_.n, s_), "memset");
    app_detail::ck(cudaMemsetAsync(misc_.p, 0, sizeof(unsigned long long) * 2, s_), "memset");
  }
  void reset_round_counters() {
    app_detail::ck(cudaMemsetAsync(cnt_.p, 0, sizeof(unsigned long long) * 2 * (max_rounds_ + 2), s_), "memset");
  }
  uint32_t next_tag() {
    if (tag_ >= 0xFFFFFFF0u) {  // wrap: clear every claim
      app_detail::ck(cudaMemsetAsync(stamp_.p, 0, sizeof(uint32_t) * nv_, s_), "memset");
      tag_ = 0;
    }
    return ++tag_;
  }
  uint32_t grid_elem(uint64_t n) const {
    const uint64_t b = (n + 255) / 256;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)nsm_ * 8));
  }
  uint32_t grid_map() const { return (uint32_t)nsm_ * 8; }
  void launch_check() { app_detail::ck(cudaGetLastError(), "kernel launch"); }
  void sync() { app_detail::ck(cudaStreamSynchronize(s_), "cudaStreamSynchronize"); }
  // Device time of a phase (added to the stats); the last phase of a start
  // or snapshot also reads the edge and reset counters.
  void phase_begin() { app_detail::ck(cudaEventRecord(ev0_, s_), "event"); }
  void phase_end(bool last) {
    app_detail::ck(cudaEventRecord(ev1_, s_), "event");
    unsigned long long m[2] = {0, 0};
    if (last) app_detail::ck(cudaMemcpyAsync(m, misc_.p, sizeof(m), cudaMemcpyDeviceToHost, s_), "copy");
    sync();
    float ms = 0;
    app_detail::ck(cudaEventElapsedTime(&ms, ev0_, ev1_), "event time");
    st_.ms += ms;
    if (last) {
      st_.edges_traversed = m[0];
      st_.resets = m[1];
    }
  }

  sgs_engine *e_;
  App app_;
  uint32_t max_rounds_;
  uint32_t nv_ = 0;
  int nsm_ = 148;
  cudaStream_t s_ = nullptr;
  int id_ = 0;
  uint32_t tag_ = 0;
  uint32_t ucap_ = 0;
  bool marked_ = false;
  bool started_ = false;  // the hooks do nothing before start()
  Stats st_;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  app_detail::DevArr<V> value_;
  app_detail::DevArr<app_detail::Rec<V, B>> rec_;
  app_detail::DevArr<B> push_;
  app_detail::DevArr<uint32_t> stamp_, bits_;
  app_detail::DevArr<unsigned long long> misc_, cnt_;  // misc: [0] edges, [1] resets, [2] round
  app_detail::DevArr<int> types_;
  Buf fr_[3];
};

// Results of a user algorithm, as GraphDatum exposes them after Gather*.
template <typename TValue, typename TBuffer>
struct AppDatum {
  uint32_t nnodes = 0;
  std::vector<TValue> host_value, host_parent;
  std::vector<TBuffer> host_buffer;
};

// The reference's Engine<TValue, TBuffer, TWeight, TAppImpl, Args...>
// (framework.cuh:77-140) for a user functor template TAppImpl: the graph and
// snapshot calls of EngineBase, InitGraph(args...) constructing
// TAppImpl<TValue, TBuffer, TWeight, Args...>(args...), Start, Gather*.
template <typename TValue, typename TBuffer, typename TWeight,
          template <typename, typename, typename, typename...> class TAppImpl, typename... UnusedData>
class Engine : public EngineBase {
 public:
  using AppImplDeviceObject = TAppImpl<TValue, TBuffer, TWeight, UnusedData...>;
  explicit Engine(const sgs_config *cfg = nullptr) : EngineBase(cfg) {}
  ~Engine() override { q_.reset(); }

  void InitGraph(const UnusedData &...data) {
    q_.reset();
    q_ = std::make_unique<Query<AppImplDeviceObject, TValue, TBuffer, TWeight>>(h_, AppImplDeviceObject(data...));
  }
  void Start() {
    if (!q_) throw Error(SGS_ERR_STATE, "InitGraph before Start");
    q_->start();
  }
  void GatherValue() { datum_.host_value = q().values(); datum_.nnodes = q().nv(); }
  void GatherParent() { datum_.host_parent = q().parents(); datum_.nnodes = q().nv(); }
  void GatherBuffer() { datum_.host_buffer = q().buffers(); datum_.nnodes = q().nv(); }
  const AppDatum<TValue, TBuffer> &GetGraphDatum() const { return datum_; }
  const Stats &AppStats() { return q().stats(); }
  Query<AppImplDeviceObject, TValue, TBuffer, TWeight> &query() { return q(); }

 private:
  Query<AppImplDeviceObject, TValue, TBuffer, TWeight> &q() {
    if (!q_) throw Error(SGS_ERR_STATE, "InitGraph first");
    return *q_;
  }
  std::unique_ptr<Query<AppImplDeviceObject, TValue, TBuffer, TWeight>> q_;
  AppDatum<TValue, TBuffer> datum_;
};

}  // namespace app
}  // namespace sgs

#ifndef SGS_APP_NO_REFERENCE_NAMES
// The names the reference's sample sources use.
typedef uint32_t index_t;
namespace utils {
using sgs::api::pair;
}
namespace sepgraph {
namespace api {
using sgs::api::AppBase;
}
namespace engine {
template <typename TValue, typename TBuffer, typename TWeight,
          template <typename, typename, typename, typename...> class TAppImpl, typename... UnusedData>
using Engine = sgs::app::Engine<TValue, TBuffer, TWeight, TAppImpl, UnusedData...>;
}
}  // namespace sepgraph
#endif

#ifdef SGS_APP_ACCEPT_OVERRIDE
// The base has no virtual functions; the samples' `override` marks become
// nothing (see the header comment).
#define override
#endif
