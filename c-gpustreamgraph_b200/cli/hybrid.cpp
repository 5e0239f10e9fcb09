// hybrid.cpp -- drop-in command line drivers hybrid_pr / hybrid_sssp /
// hybrid_bfs / hybrid_cc (one source, SGS_APP selects the algorithm).
//
// Accepts the reference's flags (include/utils/app_skeleton.h:42-100 and the
// per-app flags of samples/*/main.c*, e.g. README.md:50,53):
//   -graphfile F -format market_big -SEGMENT N -n_stream N -block_size N
//   -cache GB -hybrid N -weight_num N -weight B -update_size F -updatefile F
//   -source_node N (sssp/bfs) -error E (pr) -max_iteration N ...
// plus: -hbm_budget GB, -weights synth|file|unit, -snapshots N (default: all
// snapshots of the stream-size file), -output F (id value [parent] lines),
// -device N.  Spellings -flag V, -flag=V, --flag V and --flag=V are accepted;
// -updatesize is accepted for -update_size (README.md:40 spells it so).
// Flags of the reference's other code paths (interactive sessions, priority
// variants, load-balancing switches) are accepted and ignored, as documented.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "sgs_engine.hpp"

#ifndef SGS_APP
#define SGS_APP SGS_SSSP
#endif

namespace {

const char *app_name() {
  switch (SGS_APP) {
    case SGS_PR: return "hybrid_pr";
    case SGS_SSSP: return "hybrid_sssp";
    case SGS_BFS: return "hybrid_bfs";
    default: return "hybrid_cc";
  }
}

struct Flags {
  std::map<std::string, std::string> v;
  std::string get(const std::string &k, const std::string &d = "") const {
    auto it = v.find(k);
    return it == v.end() ? d : it->second;
  }
  double num(const std::string &k, double d) const {
    auto it = v.find(k);
    return it == v.end() ? d : std::atof(it->second.c_str());
  }
};

// Known flags: name -> takes a value (false = boolean switch).
const std::map<std::string, bool> &known() {
  static const std::map<std::string, bool> k = {
      {"graphfile", true}, {"format", true}, {"SEGMENT", true}, {"n_stream", true},
      {"block_size", true}, {"grid_size", true}, {"cache", true}, {"hybrid", true},
      {"weight_num", true}, {"weight", true}, {"update_size", true}, {"updatesize", true},
      {"updatefile", true}, {"source_node", true}, {"error", true}, {"max_iteration", true},
      {"output", true}, {"check", false}, {"verbose", false}, {"trace", false},
      {"lb_push", true}, {"lb_pull", true}, {"json", true}, {"stats", false},
      {"undirected", false}, {"interactive", false}, {"cmdfile", true}, {"priority", false},
      {"prio_delta", true}, {"edge_factor", true}, {"alpha", true}, {"beta", true},
      {"wl_alloc_factor", true}, {"wl_sort", false}, {"wl_unique", false}, {"priority_a", true},
      {"residence", true}, {"sparse", false}, {"non_atomic", false}, {"cut_threshold", true},
      {"top_ranks", true}, {"print_ranks", false}, {"norm", false},
      {"hbm_budget", true}, {"weights", true}, {"snapshots", true}, {"device", true},
      {"pull", true}, {"repair", true},
  };
  return k;
}

bool parse(int argc, char **argv, Flags &f, std::string &err) {
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.size() < 2 || a[0] != '-') { err = "unexpected argument " + a; return false; }
    a = a.substr(a[1] == '-' ? 2 : 1);
    std::string val;
    bool has_val = false;
    const size_t eq = a.find('=');
    if (eq != std::string::npos) {
      val = a.substr(eq + 1);
      a = a.substr(0, eq);
      has_val = true;
    }
    auto it = known().find(a);
    if (it == known().end()) { err = "unknown command line flag '" + a + "'"; return false; }
    if (it->second) {
      if (!has_val) {
        if (i + 1 >= argc) { err = "flag '" + a + "' is missing its value"; return false; }
        val = argv[++i];
      }
    } else if (!has_val) {
      val = "true";
    }
    f.v[a == "updatesize" ? "update_size" : a] = val;
  }
  return true;
}

}  // namespace

int main(int argc, char **argv) {
  Flags f;
  std::string err;
  if (!parse(argc, argv, f, err)) {
    std::fprintf(stderr, "%s: %s\n", app_name(), err.c_str());
    return 1;
  }
  const std::string graphfile = f.get("graphfile");
  if (graphfile.empty()) {
    std::fprintf(stderr, "%s: -graphfile must be provided\n", app_name());
    return 1;
  }
  const std::string format = f.get("format", "market_big");
  if (format != "market_big" && format != "market") {
    std::fprintf(stderr, "%s: unsupported graph format %s (market_big)\n", app_name(), format.c_str());
    return 1;
  }
  sgs_config c;
  sgs_config_default(&c);
  c.device = (int)f.num("device", 0);
  c.segments = (uint32_t)f.num("SEGMENT", c.segments);
  c.n_stream = (uint32_t)f.num("n_stream", c.n_stream);
  c.block_size = (uint32_t)f.num("block_size", c.block_size);
  c.cache_gb = f.num("cache", 0);
  c.hbm_budget_gb = f.num("hbm_budget", 0);
  const std::string wmode = f.get("weights", "synth");
  c.weight_mode = wmode == "file" ? SGS_W_EXPLICIT : wmode == "unit" ? SGS_W_UNIT : SGS_W_SYNTH;
  if (SGS_APP == SGS_PR) c.pr_tol = f.num("error", 1e-6) * (1.0 - c.pr_alpha);
  // -pull: bit 0 PageRank pull sweeps, bit 1 direction-optimizing BFS starts
  c.pull = (uint32_t)f.num("pull", SGS_APP == SGS_BFS ? 3 : 1);
  // -hybrid: 0 zero-copy, 1 explicit copy of the host tier for every repair,
  // 2 explicit copy for dense repairs (hybrid_policy.h:241-279)
  c.host_policy = (uint32_t)f.num("hybrid", 0);
  // -repair 1: repair after deletions by pulling into the reset vertices
  c.repair = (uint32_t)f.num("repair", 0);
  try {
    using clk = std::chrono::steady_clock;
    sgs::Engine engine(SGS_APP, &c);
    auto t0 = clk::now();
    engine.LoadGraph(graphfile);
    const uint32_t nv = engine.GetNodeNum();
    std::printf("%s: %u vertices loaded from %s in %.1f ms\n", app_name(), nv, graphfile.c_str(),
                std::chrono::duration<double, std::milli>(clk::now() - t0).count());
    engine.InitGraph((uint32_t)f.num("source_node", 0));
    engine.Start();
    sgs_query_stats st = engine.Stats();
    std::printf("static: %u rounds, %llu edges, %.3f ms\n", st.rounds,
                (unsigned long long)st.edges_traversed, st.ms);
    // the reference warms its edge cache here (compute_hot_vertices_*,
    // confirm_candidate_batch, LoadCache; hybrid_sssp.cu:252-254)
    engine.compute_hot_vertices_sssp();
    engine.confirm_candidate_batch();
    engine.LoadCache();
    const std::string us = f.get("update_size"), uf = f.get("updatefile");
    if (!us.empty() && !uf.empty()) {
      engine.get_update_file(us, uf);
      uint32_t n = engine.NumSnapshots();
      if (f.v.count("snapshots")) n = std::min<uint32_t>(n, (uint32_t)f.num("snapshots", n));
      std::pair<uint32_t, uint32_t> local_begin(0, 0);
      for (uint32_t k = 0; k < n; ++k) {
        if (SGS_APP == SGS_PR) {
          engine.Cancelation(local_begin, k);
          engine.Compensate(local_begin, k);
        } else {
          engine.del_edge(local_begin, k);
          engine.add_edge(local_begin, k);
        }
        st = engine.Stats();
        std::printf("batch number %u: %u rounds, %llu edges, %.3f ms, %.2f GTEPS\n", k, st.rounds,
                    (unsigned long long)st.edges_traversed, st.ms,
                    st.ms > 0 ? st.edges_traversed / (st.ms * 1e6) : 0.0);
      }
    }
    engine.GatherValue();
    const auto &gd = engine.GetGraphDatum();
    FILE *out = nullptr;
    const std::string of = f.get("output");
    if (!of.empty()) out = std::fopen(of.c_str(), "w");
    if (SGS_APP == SGS_PR) {
      engine.GatherBuffer();
      for (uint32_t i = 0; i < std::min<uint32_t>(20, nv); ++i)
        std::printf("v %u data %f delta %e\n", i, gd.host_rank[i], gd.host_delta[i]);
      if (out)
        for (uint32_t i = 0; i < nv; ++i) std::fprintf(out, "%u %.12e\n", i, gd.host_rank[i]);
    } else {
      engine.GatherParent();
      uint64_t reached = 0;
      for (uint32_t i = 0; i < nv; ++i) reached += gd.host_value[i] != 0xFFFFFFFFu;
      std::printf("reached %llu of %u vertices\n", (unsigned long long)reached, nv);
      if (out)
        for (uint32_t i = 0; i < nv; ++i) {
          if (gd.host_value[i] == 0xFFFFFFFFu)
            std::fprintf(out, "%u INF\n", i);
          else
            std::fprintf(out, "%u %u %u\n", i, gd.host_value[i], gd.host_parent[i]);
        }
    }
    if (out) std::fclose(out);
  } catch (const sgs::Error &e) {
    std::fprintf(stderr, "%s: error %d: %s\n", app_name(), e.code, e.what());
    return 2;
  }
  std::printf("Overall: Test passed\n");
  return 0;
}
