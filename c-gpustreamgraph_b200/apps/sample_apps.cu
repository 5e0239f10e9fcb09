// sample_apps.cu -- algorithms written as AppBase functors (include/sgs_app.cuh),
// the way a user of the reference writes one (samples/hybrid_*/hybrid_*.cu
// derive from sepgraph::api::AppBase), run on the engine's snapshot path.
//
//   Bfs, Sssp, Cc   the monotone family: minimum relaxation, parent-tree
//                   invalidation after deletions (the same algorithms as the
//                   engine's built-in lanes, so the two can be compared);
//   Widest          a fifth algorithm the engine has no built-in for: the
//                   widest (maximum-bottleneck) path from a source -- value =
//                   the largest, over paths, of the smallest edge weight;
//   PageRank        the accumulative family in FP64: delta pushes, snapshots
//                   by cancel/compensate of the changed out-lists.
//
// The C entry points at the end (sgs_sample_app_*) let tests drive them
// through a plain ABI; they are not part of the engine's API.
#include <cstdint>
#include <memory>
#include <string>

#include "sgs_app.cuh"

namespace samples {

using sgs::api::AppBase;
using sgs::api::index_t;
using sgs::api::max_with_parent;
using sgs::api::min_with_parent;
using sgs::api::pair;

constexpr uint32_t INF = 0xFFFFFFFFu;

// Shortest paths with integer weights (BFS: every weight 1).
template <typename TValue, typename TBuffer, typename TWeight, bool kUnit>
struct MinPath : AppBase<TValue, TBuffer, TWeight> {
  index_t source;
  explicit MinPath(index_t s) : source(s) {}
  __device__ TValue GetInitValue(index_t) const { return INF; }
  __device__ TBuffer GetInitBuffer(index_t v) const { return v == source ? 0u : INF; }
  __host__ __device__ TBuffer GetIdentityElement() const { return INF; }
  __device__ pair<TBuffer, bool> CombineValueBuffer(index_t, TValue *value, TBuffer *buffer) {
    const TBuffer b = *buffer;
    if (*value > b) {
      *value = b;
      return pair<TBuffer, bool>(b, true);
    }
    return pair<TBuffer, bool>(b, false);
  }
  __device__ int AccumulateBuffer(index_t src, index_t, TWeight w, TValue *parent, TBuffer *buffer,
                                  TBuffer b) {
    if (b == INF) return this->ACCUMULATE_FAILURE_CONTINUE;
    const uint64_t cand = (uint64_t)b + (kUnit ? 1u : (uint32_t)w);
    if (cand >= INF) return this->ACCUMULATE_FAILURE_CONTINUE;
    return min_with_parent(parent, buffer, (TBuffer)cand, src) ? this->ACCUMULATE_SUCCESS_CONTINUE
                                                               : this->ACCUMULATE_FAILURE_CONTINUE;
  }
  // A vertex whose parent edge is gone loses its value; its children follow
  // through the deletion rounds.
  __device__ int AccumulateBuffer_del(index_t src, index_t dst, TValue *parent, TBuffer *buffer,
                                      TValue *value) {
    if (*(volatile TValue *)parent != src) return 0;
    *reinterpret_cast<unsigned long long *>(parent) = ~0ull;  // buffer and parent together
    *value = INF;
    (void)buffer;
    this->m_vcsr_graph.vertices_[dst].deletion = true;
    return 1;
  }
  __device__ bool IsActiveNode(index_t, TBuffer buffer, TValue value) const { return buffer < value; }
};
template <typename V, typename B, typename W, typename... U>
using Sssp = MinPath<V, B, W, false>;
template <typename V, typename B, typename W, typename... U>
using Bfs = MinPath<V, B, W, true>;

// Directed CC of the reference (hybrid_cc.cu:96-110): the smallest id that
// reaches v along out-edges.
template <typename TValue, typename TBuffer, typename TWeight, typename... U>
struct Cc : AppBase<TValue, TBuffer, TWeight> {
  __device__ TValue GetInitValue(index_t) const { return INF; }
  __device__ TBuffer GetInitBuffer(index_t v) const { return v; }
  __host__ __device__ TBuffer GetIdentityElement() const { return INF; }
  __device__ pair<TBuffer, bool> CombineValueBuffer(index_t, TValue *value, TBuffer *buffer) {
    const TBuffer b = *buffer;
    if (*value > b) {
      *value = b;
      return pair<TBuffer, bool>(b, true);
    }
    return pair<TBuffer, bool>(b, false);
  }
  __device__ int AccumulateBuffer(index_t src, index_t, TWeight, TValue *parent, TBuffer *buffer, TBuffer b) {
    return min_with_parent(parent, buffer, b, src) ? 1 : 0;
  }
  // reset to the vertex's own label, which it then pushes again
  __device__ int AccumulateBuffer_del(index_t src, index_t dst, TValue *parent, TBuffer *, TValue *value) {
    if (*(volatile TValue *)parent != src) return 0;
    *reinterpret_cast<unsigned long long *>(parent) = ((unsigned long long)dst << 32) | INF;
    *value = INF;
    this->m_vcsr_graph.vertices_[dst].deletion = true;
    return 1;
  }
  __device__ bool IsActiveNode(index_t, TBuffer buffer, TValue value) const { return buffer < value; }
};

// Widest path: value(v) = max over paths s -> v of the smallest weight on the
// path (the source itself: INF); 0 = unreachable.
template <typename TValue, typename TBuffer, typename TWeight, typename... U>
struct Widest : AppBase<TValue, TBuffer, TWeight> {
  index_t source;
  explicit Widest(index_t s) : source(s) {}
  __device__ TValue GetInitValue(index_t) const { return 0u; }
  __device__ TBuffer GetInitBuffer(index_t v) const { return v == source ? INF : 0u; }
  __host__ __device__ TBuffer GetIdentityElement() const { return 0u; }
  __device__ pair<TBuffer, bool> CombineValueBuffer(index_t, TValue *value, TBuffer *buffer) {
    const TBuffer b = *buffer;
    if (*value < b) {
      *value = b;
      return pair<TBuffer, bool>(b, true);
    }
    return pair<TBuffer, bool>(b, false);
  }
  __device__ int AccumulateBuffer(index_t src, index_t, TWeight w, TValue *parent, TBuffer *buffer, TBuffer b) {
    const TBuffer cand = b < (TBuffer)w ? b : (TBuffer)w;
    if (cand == 0u) return 0;
    return max_with_parent(parent, buffer, cand, src) ? 1 : 0;
  }
  __device__ int AccumulateBuffer_del(index_t src, index_t dst, TValue *parent, TBuffer *, TValue *value) {
    if (*(volatile TValue *)parent != src) return 0;
    *reinterpret_cast<unsigned long long *>(parent) = 0xFFFFFFFFull;  // buffer 0, parent none
    *value = 0u;
    this->m_vcsr_graph.vertices_[dst].deletion = true;
    return 1;
  }
  __device__ bool IsActiveNode(index_t, TBuffer buffer, TValue value) const { return buffer > value; }
};

// Delta PageRank in FP64 (hybrid_pr.cu:26-151's fixed point: x_v = (1-a) +
// a * sum over in-edges u of x_u / outdeg(u); mass at dangling vertices is
// dropped).  A vertex is active while |buffer| > err.
template <typename TValue, typename TBuffer, typename TWeight, typename... U>
struct PageRank : AppBase<TValue, TBuffer, TWeight> {
  static constexpr bool kAccumulative = true;
  double err;
  double alpha;
  PageRank(double e, double a) : err(e), alpha(a) {}
  __device__ TValue GetInitValue(index_t) const { return 0.0; }
  __device__ TBuffer GetInitBuffer(index_t) const { return 1.0 - alpha; }
  __host__ __device__ TBuffer GetIdentityElement() const { return 0.0; }
  __device__ pair<TBuffer, bool> CombineValueBuffer(index_t v, TValue *value, TBuffer *buffer) {
    const unsigned long long bits = atomicExch(reinterpret_cast<unsigned long long *>(buffer), 0ull);
    const double b = __longlong_as_double((long long)bits);
    if (b == 0.0) return pair<TBuffer, bool>(0.0, false);
    *value += b;
    const uint32_t deg = this->m_vcsr_graph.sync_vertices_[v].degree;
    if (!deg) return pair<TBuffer, bool>(0.0, false);
    return pair<TBuffer, bool>(alpha * b / deg, true);
  }
  __device__ pair<TBuffer, bool> CombineValueBufferAmend(index_t v, int *type, TValue *value, TBuffer *) {
    const double b = *value * type[0];
    const uint32_t deg = this->m_vcsr_graph.sync_vertices_[v].degree;
    if (b == 0.0 || !deg) return pair<TBuffer, bool>(0.0, false);
    return pair<TBuffer, bool>(alpha * b / deg, true);
  }
  __device__ int AccumulateBuffer(index_t, index_t, TWeight, TValue *, TBuffer *buffer, TBuffer b) {
    atomicAdd(buffer, b);
    return 0;
  }
  __device__ bool IsActiveNode(index_t, TBuffer buffer, TValue) const { return buffer > err; }
  __device__ bool IsActiveNode_INC(index_t, TBuffer buffer, TValue) const { return buffer < -err; }
};

// Host-side handle over one attached algorithm.
struct Handle {
  virtual ~Handle() = default;
  virtual void start() = 0;
  virtual void values(void *out) = 0;
  virtual void parents(uint32_t *out) = 0;
  virtual sgs::app::Stats stats() = 0;
};
template <class App, class V, class B, class W>
struct HandleOf : Handle {
  sgs::app::Query<App, V, B, W> q;
  HandleOf(sgs_engine *e, const App &a) : q(e, a) {}
  void start() override { q.start(); }
  void values(void *out) override {
    const std::vector<V> v = q.values();
    memcpy(out, v.data(), sizeof(V) * v.size());
  }
  void parents(uint32_t *out) override {
    const std::vector<V> p = q.parents();
    for (size_t i = 0; i < p.size(); ++i) out[i] = (uint32_t)p[i];
  }
  sgs::app::Stats stats() override { return q.stats(); }
};

template <class F>
int guarded(F &&f) {
  try {
    f();
    return SGS_OK;
  } catch (const sgs::Error &e) {
    sgs_set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    sgs_set_last_error(e.what());
    return SGS_ERR_CUDA;
  }
}

}  // namespace samples

extern "C" {

#define SGS_SAMPLE_BFS 0
#define SGS_SAMPLE_SSSP 1
#define SGS_SAMPLE_CC 2
#define SGS_SAMPLE_PR 3
#define SGS_SAMPLE_WIDEST 4

// Attaches a sample algorithm to an engine with a loaded graph (nothing runs
// until sgs_sample_app_start).  err and alpha are PageRank's.
__attribute__((visibility("default"))) int sgs_sample_app_create(sgs_engine *e, int kind, uint32_t source,
                                                                 double err, double alpha, void **out) {
  using namespace samples;
  if (!e || !out) {
    sgs_set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  return guarded([&] {
    Handle *h = nullptr;
    switch (kind) {
      case SGS_SAMPLE_BFS:
        h = new HandleOf<Bfs<uint32_t, uint32_t, uint32_t>, uint32_t, uint32_t, uint32_t>(
            e, Bfs<uint32_t, uint32_t, uint32_t>(source));
        break;
      case SGS_SAMPLE_SSSP:
        h = new HandleOf<Sssp<uint32_t, uint32_t, uint32_t>, uint32_t, uint32_t, uint32_t>(
            e, Sssp<uint32_t, uint32_t, uint32_t>(source));
        break;
      case SGS_SAMPLE_CC:
        h = new HandleOf<Cc<uint32_t, uint32_t, uint32_t>, uint32_t, uint32_t, uint32_t>(
            e, Cc<uint32_t, uint32_t, uint32_t>());
        break;
      case SGS_SAMPLE_PR:
        h = new HandleOf<PageRank<double, double, double>, double, double, double>(
            e, PageRank<double, double, double>(err, alpha));
        break;
      case SGS_SAMPLE_WIDEST:
        h = new HandleOf<Widest<uint32_t, uint32_t, uint32_t>, uint32_t, uint32_t, uint32_t>(
            e, Widest<uint32_t, uint32_t, uint32_t>(source));
        break;
      default:
        throw sgs::Error(SGS_ERR_INVALID, "unknown sample algorithm");
    }
    *out = h;
  });
}
__attribute__((visibility("default"))) int sgs_sample_app_start(void *h) {
  return samples::guarded([&] { static_cast<samples::Handle *>(h)->start(); });
}
// nv values: u32, or f64 for PageRank
__attribute__((visibility("default"))) int sgs_sample_app_values(void *h, void *out) {
  return samples::guarded([&] { static_cast<samples::Handle *>(h)->values(out); });
}
__attribute__((visibility("default"))) int sgs_sample_app_parents(void *h, uint32_t *out) {
  return samples::guarded([&] { static_cast<samples::Handle *>(h)->parents(out); });
}
__attribute__((visibility("default"))) int sgs_sample_app_stats(void *h, uint64_t *edges, uint64_t *resets,
                                                                uint32_t *rounds, double *ms) {
  return samples::guarded([&] {
    const sgs::app::Stats s = static_cast<samples::Handle *>(h)->stats();
    *edges = s.edges_traversed;
    *resets = s.resets;
    *rounds = s.rounds;
    *ms = s.ms;
  });
}
__attribute__((visibility("default"))) int sgs_sample_app_destroy(void *h) {
  delete static_cast<samples::Handle *>(h);
  return SGS_OK;
}

}  // extern "C"
