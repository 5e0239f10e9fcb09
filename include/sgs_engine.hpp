// sgs_engine.hpp -- header-only C++ facade over the C ABI (sgs.h) that keeps
// the call sequence and method names of the reference's sample drivers, so a
// driver written against sepgraph::engine::Engine ports line for line.
//
// Reference driver (samples/hybrid_sssp/hybrid_sssp.cu:204-296):
//     engine.LoadGraph(); engine.InitGraph(source); engine.Start();
//     engine.compute_hot_vertices_sssp(); engine.confirm_candidate_batch();
//     engine.LoadCache(); engine.get_update_file();
//     for (k = 0; k < snapshots; ++k) {
//       engine.del_edge(local_begin, k); engine.add_edge(local_begin, k);
//       engine.compute_hot_vertices_sssp(); ...; engine.LoadCache();
//     }
//     engine.GatherValue(); ... GetGraphDatum().host_value
// PageRank uses Cancelation / Compensate instead of del_edge / add_edge
// (samples/hybrid_pr/hybrid_pr.cu:154-200).
//
// Here a snapshot is applied by the second call of the pair (add_edge or
// Compensate), which hands inserts and deletes to sgs_apply_batch together:
// the reference's own order within a snapshot (inserts, then deletes,
// framework.cuh:1011-1012) is kept by the engine.  Of the cache-lifecycle
// calls, LoadCache runs the edge-cache admission (sgs_cache_refresh); the
// hotness and candidate calls are folded into it.  Every snapshot also admits
// by itself inside sgs_apply_batch.  Errors throw
// sgs::Error (the reference exits through GROUTE_CUDA_CHECK instead).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "sgs.h"

namespace sgs {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != SGS_OK) throw Error(rc, sgs_last_error());
}

// Per-vertex results, as GraphDatum exposes them after Gather*.
struct GraphDatum {
  uint32_t nnodes = 0;
  std::vector<uint32_t> host_value, host_parent, host_buffer;  // BFS/SSSP/CC
  std::vector<double> host_rank, host_delta;                   // PageRank
};

// Graph, update stream and snapshot driving shared by the engines below: the
// reference's Engine methods that do not depend on the algorithm.
class EngineBase {
 public:
  explicit EngineBase(const sgs_config *cfg = nullptr) {
    sgs_config c;
    sgs_config_default(&c);
    if (cfg) c = *cfg;
    check(sgs_create(&c, &h_));
  }
  virtual ~EngineBase() {
    if (h_) sgs_destroy(h_);
  }
  EngineBase(const EngineBase &) = delete;
  EngineBase &operator=(const EngineBase &) = delete;

  sgs_engine *handle() const { return h_; }

  // Engine::LoadGraph: graph file in market_big format (src dst [w] lines).
  void LoadGraph(const std::string &graphfile) {
    uint32_t nv = 0;
    uint64_t ne = 0;
    uint32_t *s = nullptr, *d = nullptr, *w = nullptr;
    check(sgs_read_edge_list(graphfile.c_str(), &nv, &ne, &s, &d, &w));
    const int rc = sgs_load_edge_list(h_, nv, ne, s, d, w, SGS_MEM_HOST);
    sgs_free(s);
    sgs_free(d);
    sgs_free(w);
    check(rc);
    datum_.nnodes = nv;
  }
  void LoadGraph(uint32_t nv, const uint64_t *row, const uint32_t *col, const uint32_t *w) {
    check(sgs_load_csr(h_, nv, row, col, w, SGS_MEM_HOST));
    datum_.nnodes = nv;
  }
  // Synthetic R-MAT graph generated on the device (sgs_load_rmat).
  void LoadRmat(uint32_t scale, uint32_t edge_factor = 16, uint64_t seed = 1, uint64_t wseed = 1) {
    check(sgs_load_rmat(h_, scale, edge_factor, seed, 0.57, 0.19, 0.19, wseed));
    datum_.nnodes = 1u << scale;
  }

  // Engine::get_update_file(): -update_size and -updatefile.
  void get_update_file(const std::string &update_size, const std::string &updatefile) {
    uint32_t n = 0;
    uint64_t *a = nullptr, *d = nullptr;
    check(sgs_read_stream_sizes(update_size.c_str(), &n, &a, &d));
    adds_.assign(a, a + n);
    dels_.assign(d, d + n);
    sgs_free(a);
    sgs_free(d);
    uint64_t na = 0, nd = 0;
    uint32_t *au, *av, *aw, *du, *dv, *dw;
    check(sgs_read_update_file(updatefile.c_str(), &na, &au, &av, &aw, &nd, &du, &dv, &dw));
    au_.assign(au, au + na);
    av_.assign(av, av + na);
    aw_.assign(aw, aw + na);
    du_.assign(du, du + nd);
    dv_.assign(dv, dv + nd);
    for (void *p : {(void *)au, (void *)av, (void *)aw, (void *)du, (void *)dv, (void *)dw}) sgs_free(p);
  }
  uint32_t NumSnapshots() const { return (uint32_t)adds_.size(); }

  // Snapshot k: del_edge records the deletes, add_edge applies the snapshot.
  // local_begin = (insert offset, delete offset), advanced like the reference.
  //
  // The whole snapshot -- inserts first, then deletes, the reference's order
  // within a snapshot (framework.cuh:1011-1012) -- is applied by add_edge (or
  // Compensate) in one sgs_apply_batch, which also updates every registered
  // query and attached user algorithm.  del_edge (Cancelation) changes
  // nothing yet: results gathered between del_edge and add_edge are those of
  // the previous snapshot.  (The reference's del_edge leaves the parent tree
  // half invalidated on the old graph at that point, a state no caller can
  // use; applying the deletes alone here would reverse the reference's order
  // for an edge both inserted and deleted in one snapshot.)
  void del_edge(std::pair<uint32_t, uint32_t> &, uint32_t k) { pending_ = k; }
  void add_edge(std::pair<uint32_t, uint32_t> &local_begin, uint32_t k) {
    if (k >= adds_.size()) throw Error(SGS_ERR_INVALID, "snapshot index beyond the stream-size file");
    const uint64_t ia = local_begin.first, id = local_begin.second;
    const uint64_t na = adds_[k], nd = dels_[k];
    if (ia + na > au_.size() || id + nd > du_.size())
      throw Error(SGS_ERR_INVALID, "update file holds fewer updates than the stream sizes list");
    check(sgs_apply_batch(h_, au_.data() + ia, av_.data() + ia, aw_.data() + ia, na,
                          du_.data() + id, dv_.data() + id, nd, SGS_MEM_HOST));
    local_begin.first += (uint32_t)na;
    local_begin.second += (uint32_t)nd;
    (void)pending_;
  }
  void Cancelation(std::pair<uint32_t, uint32_t> &lb, uint32_t k) { del_edge(lb, k); }
  void Compensate(std::pair<uint32_t, uint32_t> &lb, uint32_t k) { add_edge(lb, k); }
  // One snapshot from caller arrays (host memory).
  void ApplyBatch(const uint32_t *ins_src, const uint32_t *ins_dst, const uint32_t *ins_w, uint64_t n_ins,
                  const uint32_t *del_src, const uint32_t *del_dst, uint64_t n_del) {
    check(sgs_apply_batch(h_, ins_src, ins_dst, ins_w, n_ins, del_src, del_dst, n_del, SGS_MEM_HOST));
  }

  // Cache lifecycle of the reference (framework.cuh:149-308, 1304-1385):
  // hotness scoring, candidate choice, eviction and compaction are one
  // admission pass of the engine's line cache, run by LoadCache (and by every
  // snapshot); the other calls have nothing left to do.
  void compute_hot_vertices_pr() {}
  void compute_hot_vertices_sssp() {}
  void confirm_candidate_batch() {}
  void evication_cache() {}
  void compact_cache() {}
  void LoadCache() { check(sgs_cache_refresh(h_)); }

  uint32_t GetNodeNum() const { return datum_.nnodes; }

 protected:
  sgs_engine *h_ = nullptr;
  GraphDatum datum_;
  uint32_t pending_ = 0;
  std::vector<uint64_t> adds_, dels_;
  std::vector<uint32_t> au_, av_, aw_, du_, dv_;
};

// The engine for the four built-in algorithms of the samples.
class Engine : public EngineBase {
 public:
  // algo: SGS_BFS, SGS_SSSP, SGS_CC or SGS_PR
  explicit Engine(int algo, const sgs_config *cfg = nullptr) : EngineBase(cfg), algo_(algo) {}

  // Engine::InitGraph(args...): the source for BFS/SSSP (clamped to
  // [0, nnodes-1] as the samples do); PageRank's error tolerance is taken
  // from the configuration, CC takes no argument.
  void InitGraph(uint32_t source = 0) { source_ = source; }
  // Engine::Start: static convergence.
  void Start() { check(sgs_query_add(h_, algo_, source_, &qid_)); }

  void GatherValue() { gather(SGS_FIELD_VALUE); }
  void GatherParent() { gather(SGS_FIELD_PARENT); }
  void GatherBuffer() { gather(SGS_FIELD_BUFFER); }
  const GraphDatum &GetGraphDatum() const { return datum_; }

  sgs_query_stats Stats() const {
    sgs_query_stats s{};
    check(sgs_get_query_stats(h_, qid_, &s));
    return s;
  }

 private:
  void gather(int field) {
    const uint32_t n = datum_.nnodes;
    if (algo_ == SGS_PR) {
      std::vector<double> &dst = field == SGS_FIELD_VALUE ? datum_.host_rank : datum_.host_delta;
      dst.resize(n);
      check(sgs_gather(h_, qid_, field, dst.data(), SGS_MEM_HOST));
      return;
    }
    std::vector<uint32_t> &dst = field == SGS_FIELD_VALUE    ? datum_.host_value
                                 : field == SGS_FIELD_PARENT ? datum_.host_parent
                                                             : datum_.host_buffer;
    dst.resize(n);
    check(sgs_gather(h_, qid_, field, dst.data(), SGS_MEM_HOST));
  }

  int algo_;
  int qid_ = -1;
  uint32_t source_ = 0;
};

}  // namespace sgs
