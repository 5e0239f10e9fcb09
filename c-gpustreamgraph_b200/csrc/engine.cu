// engine.cu -- host side of the B200 streaming-graph engine and the C ABI
// declared in include/sgs.h.
//
// One engine = one dynamic graph in HBM (optionally part of it in pinned host
// memory under an HBM budget) plus registered queries (BFS, SSSP, CC, PR),
// all kept up to date snapshot by snapshot.  Everything runs on one CUDA
// stream; the host only reads a handful of counters per convergence (a
// batch of rounds is queued back to back and their frontier counters are read
// once), instead of the reference's blocking count read per segment per round
// (groute/device/queue.cuh:315-321 called from algo_variants.cuh:628 and
// framework.cuh:1460).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <array>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sgs.h"
#include "sgs_cache.cuh"
#include "sgs_group.cuh"
#include "sgs_pull.cuh"
#include "sgs_kernels.cuh"
#include "sgs_wide.cuh"

using namespace sgs;

namespace {

thread_local std::string g_last_error;

struct SgsError {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg) { throw SgsError{code, msg}; }

}  // namespace

// Shared with the other translation units of the library (not exported).
namespace sgs {
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace sgs

namespace {

void ck(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  fail(e == cudaErrorMemoryAllocation ? SGS_ERR_OOM : SGS_ERR_CUDA,
       std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(x) ck((x), #x)

template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  void ensure(size_t want) {
    if (want <= n && p) return;
    release();
    size_t bytes = std::max<size_t>(want, 1) * sizeof(T);
    CK(cudaMalloc((void **)&p, bytes));
    n = std::max<size_t>(want, 1);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { release(); }
};

// Capacity for a batch-sized buffer of n items: the next power of two (at
// least 4096), so buffers that follow the batch size grow a few times at
// most instead of at every larger batch (each growth frees and allocates).
static inline size_t batch_cap(uint64_t n) {
  if (n == 0) return 0;
  size_t c = 4096;
  while (c < n) c <<= 1;
  return c;
}

template <class T>
struct HBuf {  // pinned, mapped host memory
  T *p = nullptr;
  size_t n = 0;
  void ensure(size_t want) {
    if (want <= n && p) return;
    release();
    CK(cudaHostAlloc((void **)&p, std::max<size_t>(want, 1) * sizeof(T),
                     cudaHostAllocMapped | cudaHostAllocPortable));
    n = std::max<size_t>(want, 1);
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  ~HBuf() { release(); }
};

struct Frontier {
  DBuf<uint32_t> vtx;
  DBuf<uint32_t> len;
  DBuf<uint64_t> ebase;
  DBuf<uint32_t> ustart;
};

// A group: integer queries sharing one edge stream.  Narrow groups (width
// GMAX = 4, sgs_group.cuh) keep a vertex's lanes in one 32-B sector and the
// lanes of a slot in a thread's registers; wide groups (width 64,
// sgs_wide.cuh) keep a vertex's lanes in one 512-B row with a warp's threads
// covering them.
struct Group {
  int width = GMAX;             // GMAX or WLANES
  DBuf<unsigned long long> st;  // [nv * width] packed (value, parent)
  DBuf<uint32_t> val;           // [nv * width] value mirror (read-side filter)
  uint64_t used = 0;            // lanes in use
  uint32_t algo_packed = 0;     // narrow: 8 bits per lane
  uint64_t sssp = 0, cc = 0;    // lanes per algorithm (both widths)
  uint64_t inval[WLANES] = {};  // resets per lane in the last deletion phase
  DBuf<uint32_t> ibits;         // narrow: bitmap of vertices reset in the last deletion phase
  DBuf<unsigned long long> wreset;  // wide: per vertex, the lanes reset in the last deletion phase
  // per-lane device counters of the last snapshot: [0,64) resets, [64,128)
  // edges of the invalidation, [128,192) edges of the repair; read once at
  // the end of the snapshot
  DBuf<unsigned long long> dstat;
  bool wide() const { return width == WLANES; }
  LaneAlgo algo() const { return LaneAlgo::of(algo_packed); }
  WideAlgo walgo() const { return WideAlgo{sssp, cc}; }
  bool any_sssp(uint64_t lanes) const { return (lanes & sssp) != 0; }
  void set_lane(int l, int a) {
    if (!wide()) algo_packed = (algo_packed & ~(0xFFu << (8 * l))) | ((uint32_t)a << (8 * l));
    const uint64_t b = 1ull << l;
    sssp = a == A_SSSP ? sssp | b : sssp & ~b;
    cc = a == A_CC ? cc | b : cc & ~b;
  }
};

struct Query {
  int id = 0;
  int algo = 0;
  uint32_t source = 0;
  Group *grp = nullptr;  // BFS / SSSP / CC: group and lane
  int lane = -1;
  DBuf<double> x, r, pv;  // PageRank
  sgs_query_stats stats{};
};

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  void init() {
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
  }
  ~Events() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// NVTX range for the lifetime of a scope (phases show up in Nsight tools and
// let an ncu capture select kernels by phase).
struct Range {
  explicit Range(const char *name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
};

inline uint32_t blocks_for(uint64_t n, uint32_t cap) {
  uint64_t b = (n + 255) / 256;
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b, cap));
}

}  // namespace

struct sgs_engine {
  sgs_config cfg{};
  int dev = 0;
  int nsm = 148;
  cudaStream_t s = nullptr;
  bool loaded = false;

  // graph
  uint32_t nv = 0;
  uint64_t ne = 0;  // live edges (host mirror)
  uint64_t slots_total = 0;  // used slots (host mirror)
  DBuf<uint64_t> off;
  DBuf<uint32_t> slots, live, cap;
  DBuf<uint32_t> adj_d, wgt_d;
  HBuf<uint32_t> adj_h, wgt_h;
  uint64_t arena_cap[2] = {0, 0};
  DBuf<unsigned long long> arena_top;  // [2]
  uint32_t split = 0;                   // vertices [0,split) start in HBM
  uint64_t repacks = 0;

  // frontier scratch
  Frontier fb[3];                          // rotating frontier buffers
  DBuf<uint32_t> gm[3];                    // rotating group lane masks
  DBuf<unsigned long long> wm[3];          // the same for wide groups (u64)
  uint32_t ucap = 0;
  static constexpr uint32_t kSpecial = 8;  // extra counter slots at the end
  DBuf<unsigned long long> cnt;            // [max_rounds + 2 + kSpecial]
  unsigned long long *h_cnt = nullptr;     // pinned mirror
  DBuf<uint32_t> emark;                    // engine-level marks (touched sets)
  uint32_t estamp = 1;
  DBuf<double> l1;                         // PR per-round L1
  DBuf<unsigned long long> rstat;          // per-round instance-edge counts
  DBuf<unsigned long long> hstat;          // per-round host-tier slots
  DBuf<unsigned long long> b_lane;         // [WLANES] per-lane edge counts
  DBuf<unsigned long long> b_inval;        // [WLANES] per-lane resets
  DBuf<uint32_t> b_seed;                   // sources and lanes of new wide lanes

  // batch scratch
  DBuf<uint32_t> b_isrc, b_idst, b_iw, b_dsrc, b_ddst;
  DBuf<uint64_t> b_ikeys, b_ikeys_s, b_ikept, b_dkeys, b_dkeys_s;
  DBuf<uint32_t> b_iw_s, b_iw_kept, b_gstart;
  DBuf<unsigned char> b_flag;
  DBuf<uint32_t> b_nkept;
  DBuf<unsigned int> b_err;
  DBuf<unsigned long long> b_stat;  // [0] demand d, [1] demand h, [2] tombs, [3] inval
  DBuf<unsigned long long> b_reclaim;  // slots reclaimed by block compaction: [0] out-, [1] in-store
  DBuf<uint32_t> big_list, big_n;      // large blocks to compact (k_compact_large) and their count
  uint64_t reclaimed_total = 0;
  DBuf<uint64_t> wbase;
  DBuf<uint32_t> rl_vtx, rl_len;
  DBuf<uint64_t> rl_from, rl_to;
  DBuf<unsigned long long> rl_count;
  DBuf<unsigned char> cub_tmp;

  // per-kernel-class timing
  bool ktiming = false;
  std::vector<cudaEvent_t> kev;  // 2 per queued launch
  std::vector<cudaEvent_t> gev;  // 4 per group per snapshot
  std::vector<unsigned long long> h_gstat;
  sgs_kernel_stats kst[SGS_K_COUNT]{};
  uint64_t n_launch = 0;  // this engine's own kernel launches (library sorts/scans excluded)

  std::vector<std::unique_ptr<Query>> queries;
  std::vector<std::unique_ptr<Group>> groups;
  // user algorithms (AppBase functors compiled in the caller's translation
  // unit, include/sgs_app.cuh) updated by every snapshot through their hooks
  struct AppHook {
    int id;
    sgs_app_hooks h;
  };
  std::vector<AppHook> apps;
  int next_app = 1;
  // serving: one group kept in flight; queries join free lanes at round
  // boundaries and leave once no frontier entry carries their lane
  Group *fg = nullptr;
  uint32_t fr = 0;                   // next round; its input is buffer fr % 3 / cnt[fr]
  uint64_t frun = 0;                 // lanes with work in flight
  uint64_t fsusp = 0;                // lanes suspended while an update applies
  uint32_t fadmit[WLANES] = {};      // round at which each lane joined
  DBuf<unsigned long long> flc;      // per-lane entry counts of the next frontier
  int next_qid = 1;
  sgs_engine_stats est{};
  Events ev_batch, ev_apply, ev_q;

  // device edge cache of the host tier (sgs_cache.cuh): lines of CLINE
  // slots admitted per snapshot by hotness, copied on a side stream
  bool cache_on = false;
  uint64_t c_lines = 0;                // capacity (lines)
  uint64_t h_lines = 0;                // lines of the host arena (cmap entries)
  uint64_t cbase = 0;                  // cached lines: adj_d/wgt_d slots [cbase, cbase + c_lines*CLINE)
  DBuf<uint32_t> cmap, cown;           // host line -> cache line, cache line -> host line
  DBuf<uint32_t> cscore, chist, c_new, c_free;
  DBuf<uint2> c_pend;                  // (host line, cache line) of the last admission
  DBuf<unsigned long long> c_cc;       // counters (CC_*)
  DBuf<uint32_t> hot;                  // per vertex: four u8 activation counters
  uint32_t hot_k = 0;                  // the byte the current snapshot fills
  cudaStream_t s2 = nullptr;           // side stream of the line copies
  cudaEvent_t ev_cadmit = nullptr, ev_ccopy = nullptr;
  bool c_pending = false;              // copies issued, lines not yet published
  uint64_t c_admissions = 0;

  // in-edge store (sgs_pull.cuh), HBM only, source ids only: built by the
  // first pull sweep, then updated by every snapshot
  bool in_built = false, in_failed = false;
  DBuf<uint64_t> in_off;
  DBuf<uint32_t> in_slots, in_live, in_cap, in_adj;
  DBuf<uint32_t> in_wgt;               // weights too, for the pull repair of SSSP lanes
  DBuf<unsigned long long> in_top;     // [2]; tier 1 unused
  uint64_t in_capslots = 0;
  uint64_t in_builds = 0;
  DBuf<uint64_t> t_dkeys, t_ikeys, t_tmp;  // the batch's keys transposed
  DBuf<uint32_t> t_iw;                     // and the kept inserts' weights

  // explicit-copy host policy (cfg.host_policy): the used host arena copied
  // to HBM by the copy engine for a snapshot's repair, readers pointed at it
  DBuf<uint32_t> stage_adj, stage_wgt;
  bool staged = false;
  uint64_t stage_bytes_last = 0, stagings = 0;

  // the value vector of the last removed PageRank query: the next PageRank
  // start continues from it (its residual on the current graph is computed
  // first), so a query after a few updates needs few rounds
  DBuf<double> pr_warm;
  uint64_t pr_warm_starts = 0;

  // staged batches (sgs_stage_batch): two slots of device copies of a batch's
  // arrays, filled on a copy stream while the engine's stream computes
  struct Staged {
    DBuf<uint32_t> a[5];  // ins src, dst, w; del src, dst
    uint64_t ni = 0, nd = 0;
    bool w = false;
    bool full = false;
    cudaEvent_t copied = nullptr, consumed = nullptr;
  } stg[2];
  uint32_t stg_head = 0, stg_count = 0;  // oldest full slot, full slots
  cudaStream_t sc = nullptr;             // copy stream

  ~sgs_engine() {
    if (sc) {
      cudaStreamSynchronize(sc);
      cudaStreamDestroy(sc);
    }
    for (auto &t : stg) {
      if (t.copied) cudaEventDestroy(t.copied);
      if (t.consumed) cudaEventDestroy(t.consumed);
    }
    if (s2) {
      cudaStreamSynchronize(s2);
      cudaStreamDestroy(s2);
    }
    if (ev_cadmit) cudaEventDestroy(ev_cadmit);
    if (ev_ccopy) cudaEventDestroy(ev_ccopy);
    for (auto ev : kev) cudaEventDestroy(ev);
    for (auto ev : gev) cudaEventDestroy(ev);
    if (h_cnt) cudaFreeHost(h_cnt);
    if (s) cudaStreamDestroy(s);
  }

  GraphView view() {
    GraphView g{};
    g.nv = nv;
    g.off = off.p;
    g.slots = slots.p;
    g.live = live.p;
    g.cap = cap.p;
    g.adj_d = adj_d.p;
    g.wgt_d = wgt_d.p;
    g.adj_h = staged ? stage_adj.p : adj_h.p;
    g.wgt_h = staged ? stage_wgt.p : wgt_h.p;
    g.wmode = cfg.weight_mode;
    if (cache_on && h_lines) {
      g.cmap = cmap.p;
      g.adj_c = adj_d.p + cbase;
      g.wgt_c = wgt_d.p ? wgt_d.p + cbase : nullptr;
      g.cbase = cbase;
      g.hot = hot.p;
      g.hot_sh = 8 * hot_k;
      g.cstat = c_cc.p;
    }
    return g;
  }
  // the in-edge store keeps weights when the pull repair may need them
  bool in_w() const { return (cfg.repair & 1u) && cfg.weight_mode == SGS_W_EXPLICIT; }
  GraphView in_view() {
    GraphView g{};
    g.nv = nv;
    g.off = in_off.p;
    g.slots = in_slots.p;
    g.live = in_live.p;
    g.cap = in_cap.p;
    g.adj_d = in_adj.p;
    g.wgt_d = in_w() ? in_wgt.p : nullptr;
    g.wmode = in_w() ? SGS_W_EXPLICIT : SGS_W_UNIT;
    return g;
  }
  FrontierView fview(uint32_t buf, unsigned long long *counter) {
    FrontierView f;
    f.vtx = fb[buf % 3].vtx.p;
    f.len = fb[buf % 3].len.p;
    f.ebase = fb[buf % 3].ebase.p;
    f.ustart = fb[buf % 3].ustart.p;
    f.counter = (uint64_t *)counter;
    f.ucap = ucap;
    return f;
  }
  unsigned long long *special(uint32_t k) { return cnt.p + cfg.max_rounds + 2 + k; }
  uint32_t map_cps = 32;  // CTAs per SM of the load-balanced maps (sgs_autotune)
  uint32_t grid_map() const { return (uint32_t)nsm * map_cps; }
  uint32_t grid_elem(uint64_t n) const { return blocks_for(n, (uint32_t)nsm * 8); }
  size_t wbytes() const { return cfg.weight_mode == SGS_W_EXPLICIT ? 8 : 4; }
  // some blocks live in the pinned-host tier (the maps then compile in the
  // host-tier logic: hotness, cache lookups, link accounting)
  bool host_tier() const { return split < nv; }

  void cub_ensure(size_t bytes) { cub_tmp.ensure(batch_cap(bytes)); }

  void sync() { CK(cudaStreamSynchronize(s)); }

  // ------------------------------------------------------------------ setup
  void init(const sgs_config &c) {
    cfg = c;
    if (cfg.max_rounds == 0) cfg.max_rounds = 1000;
    if (cfg.pr_alpha <= 0 || cfg.pr_alpha >= 1) fail(SGS_ERR_INVALID, "pr_alpha must be in (0,1)");
    if (cfg.weight_mode < 0 || cfg.weight_mode > 2) fail(SGS_ERR_INVALID, "bad weight_mode");
    dev = cfg.device;
    CK(cudaSetDevice(dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cnt.ensure(cfg.max_rounds + 2 + kSpecial);
    CK(cudaHostAlloc((void **)&h_cnt, (cfg.max_rounds + 2 + kSpecial) * sizeof(unsigned long long),
                     cudaHostAllocDefault));
    arena_top.ensure(2);
    b_err.ensure(1);
    b_stat.ensure(8);
    b_reclaim.ensure(2);
    b_nkept.ensure(1);
    rl_count.ensure(1);
    l1.ensure(cfg.max_rounds + 2);
    rstat.ensure(cfg.max_rounds + 2);
    hstat.ensure(cfg.max_rounds + 2);
    b_lane.ensure(WLANES);
    b_inval.ensure(WLANES);
    if (cfg.group_size < 1 || cfg.group_size > WLANES) cfg.group_size = GMAX;
    ev_batch.init();
    ev_apply.init();
    ev_q.init();
    cache_init();
  }

  // ------------------------------------------------------------ edge cache
  // On when both an HBM budget and a cache size are given: the cache is
  // carved out of the budget (the static HBM tier gets the rest).
  void cache_init() {
    if (!(cfg.cache_gb > 0 && cfg.hbm_budget_gb > 0)) return;
    c_lines = (uint64_t)(cfg.cache_gb * 1e9 / (double)(CLINE * wbytes()));
    if (c_lines == 0) return;
    if (c_lines >= NO_LINE) fail(SGS_ERR_INVALID, "cache_gb too large");
    cache_on = true;
    cown.ensure(c_lines);
    c_new.ensure(c_lines);
    c_free.ensure(c_lines);
    c_pend.ensure(c_lines);
    chist.ensure(HOT_BINS);
    c_cc.ensure(CC_N);
    CK(cudaMemsetAsync(cown.p, 0xFF, sizeof(uint32_t) * c_lines, s));
    CK(cudaMemsetAsync(c_cc.p, 0, sizeof(unsigned long long) * CC_N, s));
    CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ev_cadmit, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_ccopy, cudaEventDisableTiming));
  }
  double static_budget_gb() const {
    return cache_on ? std::max(0.0, cfg.hbm_budget_gb - cfg.cache_gb) : cfg.hbm_budget_gb;
  }
  // Waits for copies in flight (before arenas are reallocated).
  void cache_quiesce() {
    if (!cache_on) return;
    CK(cudaStreamSynchronize(s2));
    c_pending = false;
  }
  // A new host arena of cap_h slots: every line dropped; a new graph also
  // starts a new hotness window.
  void cache_layout(uint64_t cap_h) {
    if (!cache_on) return;
    cache_quiesce();
    h_lines = (cap_h + CLINE - 1) / CLINE;
    cmap.ensure(std::max<uint64_t>(h_lines, 1));
    cscore.ensure(std::max<uint64_t>(h_lines, 1));
    if (h_lines) CK(cudaMemsetAsync(cmap.p, 0xFF, sizeof(uint32_t) * h_lines, s));
    CK(cudaMemsetAsync(cown.p, 0xFF, sizeof(uint32_t) * c_lines, s));
    if (!loaded) {
      hot.ensure(nv);
      CK(cudaMemsetAsync(hot.p, 0, sizeof(uint32_t) * nv, s));
      hot_k = 0;
      CK(cudaMemsetAsync(c_cc.p, 0, sizeof(unsigned long long) * CC_N, s));
    }
  }
  // Makes the lines of the last admission visible once their copy is done
  // (the main stream waits for the side stream).
  void cache_publish() {
    if (!c_pending) return;
    CK(cudaStreamWaitEvent(s, ev_ccopy, 0));
    { ++n_launch; k_cache_publish<<<grid_elem(c_lines), 256, 0, s>>>(c_pend.p, c_cc.p, cmap.p); }
    CK(cudaGetLastError());
    c_pending = false;
  }
  // Admission from the hotness window (advanced by one snapshot when
  // `rotate`): evictions, new lines paired with free cache lines, and their
  // copies on the side stream, which overlap whatever the main stream runs
  // next.  The lines become visible at the next cache_publish.
  void cache_admit(bool rotate) {
    if (!cache_on || !h_lines) return;
    cache_publish();  // every owned cache line mapped before the keep pass
    const uint32_t next = (hot_k + 1) & 3u;
    CK(cudaMemsetAsync(cscore.p, 0, sizeof(uint32_t) * h_lines, s));
    CK(cudaMemsetAsync(chist.p, 0, sizeof(uint32_t) * HOT_BINS, s));
    CK(cudaMemsetAsync(c_cc.p + CC_TICK, 0, sizeof(unsigned long long) * (CC_N - CC_TICK), s));
    const GraphView g = view();
    { ++n_launch; k_cache_score<<<grid_elem(nv), 256, 0, s>>>(g, rotate ? 8 * next : 32u, cscore.p, h_lines); }
    if (rotate) hot_k = next;
    { ++n_launch; k_cache_hist<<<grid_elem(h_lines), 256, 0, s>>>(cscore.p, h_lines, chist.p); }
    { ++n_launch; k_cache_threshold<<<1, 1024, 0, s>>>(chist.p, c_lines, c_cc.p); }
    { ++n_launch; k_cache_keep<<<grid_elem(c_lines), 256, 0, s>>>(cmap.p, cown.p, cscore.p, c_lines, c_cc.p); }
    { ++n_launch; k_cache_pick<<<grid_elem(h_lines), 256, 0, s>>>(cmap.p, cscore.p, h_lines, c_lines, c_new.p,
                                                      c_cc.p); }
    { ++n_launch; k_cache_free<<<grid_elem(c_lines), 256, 0, s>>>(cown.p, c_lines, c_free.p, c_cc.p); }
    { ++n_launch; k_cache_pair<<<grid_elem(c_lines), 256, 0, s>>>(c_new.p, c_free.p, c_lines, cown.p, c_pend.p,
                                                      c_cc.p); }
    CK(cudaEventRecord(ev_cadmit, s));
    CK(cudaStreamWaitEvent(s2, ev_cadmit, 0));
    { ++n_launch; k_cache_copy<<<(uint32_t)nsm * 4, 256, 0, s2>>>(
        c_pend.p, c_cc.p, adj_h.p, cfg.weight_mode == SGS_W_EXPLICIT ? wgt_h.p : nullptr,
        adj_d.p + cbase, cfg.weight_mode == SGS_W_EXPLICIT ? wgt_d.p + cbase : nullptr); }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ev_ccopy, s2));
    c_pending = true;
    ++c_admissions;
  }

  // ------------------------------------------------ explicit host policy
  // The reference's -hybrid policies (framework/hybrid_policy.h:241-279,
  // framework.cuh:2012-2180) read a segment either zero-copy or after an
  // explicit copy of its edges into device buffers (edge_dst_exp,
  // csr_graph.cuh:1877-1884), the explicit form chosen for every segment
  // (-hybrid 1) or for segments whose active share exceeds alpha (-hybrid 2).
  // Here: policy 1 copies the used host arena to HBM with the copy engine
  // (cudaMemcpyAsync, chunks of 1 GiB) before every snapshot's repair;
  // policy 2 only when the repair's first frontier covers more than half of
  // the graph's slots (the dense re-push after deletions).  Relaxation rounds
  // only read blocks, and the snapshot's writes happened before, so the
  // copy stays exact for the whole repair.
  bool stage_wanted() {
    if (!cfg.host_policy || !host_tier() || staged) return false;
    if (cfg.host_policy == 1) return true;
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, cnt.p, sizeof(c), cudaMemcpyDeviceToHost, s));
    sync();
    return (double)(c & EDGE_MASK) > 0.5 * (double)slots_total;
  }
  void stage_host() {
    unsigned long long tops[2];
    CK(cudaMemcpyAsync(tops, arena_top.p, sizeof(tops), cudaMemcpyDeviceToHost, s));
    sync();
    const uint64_t n = std::min<uint64_t>(tops[1], arena_cap[1]);
    if (!n) return;
    const bool ew = cfg.weight_mode == SGS_W_EXPLICIT;
    stage_adj.ensure(n);
    if (ew) stage_wgt.ensure(n);
    const uint64_t chunk = (1ull << 30) / sizeof(uint32_t);
    for (uint64_t o = 0; o < n; o += chunk) {
      const uint64_t k = std::min(chunk, n - o);
      CK(cudaMemcpyAsync(stage_adj.p + o, adj_h.p + o, k * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
      if (ew)
        CK(cudaMemcpyAsync(stage_wgt.p + o, wgt_h.p + o, k * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    }
    staged = true;
    stage_bytes_last = n * (ew ? 8 : 4);
    ++stagings;
  }

  // -------------------------------------------------------- in-edge store
  // Transposes the out-store: in-degrees, capacities with the same slack,
  // offsets by a scan, then every live out-slot (u -> d) places u in d's
  // in-block through a per-destination cursor.  Uses frontier buffers 0 and
  // 1 and counters special(0..1): callers build it before they seed a
  // frontier (or after the last one they use).
  void in_build(FrontierView f0, FrontierView f1) {
    const GraphView g = view();
    in_slots.ensure(nv);
    in_live.ensure(nv);
    in_cap.ensure(nv);
    in_off.ensure((size_t)nv + 1);
    in_top.ensure(2);
    CK(cudaMemsetAsync(in_slots.p, 0, sizeof(uint32_t) * nv, s));
    CK(cudaMemsetAsync(f0.counter, 0, sizeof(unsigned long long), s));
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(g, f0); }
    { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(f0, f1, InCountOp{g, in_slots.p}, nullptr); }
    { ++n_launch; k_layout_caps<<<grid_elem(nv), 256, 0, s>>>(in_slots.p, nv, cfg.slack_div, in_cap.p); }
    { ++n_launch; k_u32_to_u64<<<grid_elem(nv), 256, 0, s>>>(in_cap.p, nv, in_off.p); }
    CK(cudaMemsetAsync(in_off.p + nv, 0, sizeof(uint64_t), s));
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, in_off.p, in_off.p, (int)(nv + 1), s));
    cub_ensure(tb);
    CK(cub::DeviceScan::ExclusiveSum(cub_tmp.p, tb, in_off.p, in_off.p, (int)(nv + 1), s));
    uint64_t total = 0;
    CK(cudaMemcpyAsync(&total, in_off.p + nv, sizeof(total), cudaMemcpyDeviceToHost, s));
    sync();
    in_capslots = total + (uint64_t)(total * std::max(0.0, cfg.arena_headroom)) + 4096;
    in_adj.ensure(in_capslots);
    if (in_w()) in_wgt.ensure(in_capslots);
    unsigned long long tops[2] = {total, 0};
    CK(cudaMemcpyAsync(in_top.p, tops, sizeof(tops), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(in_live.p, 0, sizeof(uint32_t) * nv, s));  // the fill cursors
    { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(
        f0, f1, InFillOp{g, in_off.p, in_live.p, in_adj.p, in_w() ? in_wgt.p : nullptr}, nullptr); }
    CK(cudaMemcpyAsync(in_live.p, in_slots.p, sizeof(uint32_t) * nv, cudaMemcpyDeviceToDevice, s));
    CK(cudaGetLastError());
    sync();
    in_built = true;
    ++in_builds;
  }
  void in_release() {
    in_off.release();
    in_slots.release();
    in_live.release();
    in_cap.release();
    in_adj.release();
    in_wgt.release();
    in_built = false;
  }
  // True when the in-store is there (built now if needed).  If it cannot be
  // allocated the engine keeps to push sweeps (both run on the GPU).
  bool ensure_in() { return ensure_in(fview(0, special(0)), fview(1, special(1))); }
  bool ensure_in(FrontierView f0, FrontierView f1) {
    if (!cfg.pull || in_failed) return false;
    if (in_built) return true;
    try {
      in_build(f0, f1);
    } catch (const SgsError &f) {
      if (f.code != SGS_ERR_OOM) throw;
      in_release();
      in_failed = true;
      return false;
    }
    return true;
  }
  // The snapshot's deletes and kept inserts applied to the in-store, keys
  // transposed and sorted; when relocations would not fit, the store is
  // rebuilt from the (already updated) out-store instead.
  void in_apply(uint64_t ni, uint64_t nd, uint32_t nkept) {
    if (!in_built) return;
    const GraphView gi = in_view();
    const int eb = sort_bits();
    size_t tb = 0;
    if (nd) {
      t_dkeys.ensure(batch_cap(nd));
      t_tmp.ensure(batch_cap(std::max<uint64_t>(nd, nkept)));
      { ++n_launch; k_transpose_keys<<<grid_elem(nd), 256, 0, s>>>(b_dkeys_s.p, (uint32_t)nd, nullptr, t_tmp.p); }
      CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, t_tmp.p, t_dkeys.p, (int)nd, 0, eb, s));
      cub_ensure(tb);
      CK(cub::DeviceRadixSort::SortKeys(cub_tmp.p, tb, t_tmp.p, t_dkeys.p, (int)nd, 0, eb, s));
      CK(cudaMemsetAsync(special(4), 0, sizeof(unsigned long long) * 2, s));
      b_gstart.ensure((size_t)nv + 1);
      { ++n_launch; k_group_heads<<<grid_elem(nd), 256, 0, s>>>(gi, t_dkeys.p, nullptr, (uint32_t)nd, b_gstart.p,
                                                  nullptr, 0, fview(0, special(4))); }
      TombOp op{gi, t_dkeys.p, b_gstart.p, (uint32_t)nd};
      { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fview(0, special(4)), fview(1, special(5)), op,
                                                   nullptr); }
      compact_blocks(gi, nd, b_reclaim.p + 1);
      CK(cudaGetLastError());
    }
    if (!ni || !nkept) return;
    t_ikeys.ensure(batch_cap(nkept));
    t_tmp.ensure(batch_cap(nkept));
    { ++n_launch; k_transpose_keys<<<grid_elem(nkept), 256, 0, s>>>(b_ikept.p, nkept, nullptr, t_tmp.p); }
    tb = 0;
    if (in_w()) {  // the kept inserts' weights travel with their transposed keys
      t_iw.ensure(batch_cap(nkept));
      CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, t_tmp.p, t_ikeys.p, b_iw_kept.p, t_iw.p, (int)nkept, 0, eb,
                                         s));
      cub_ensure(tb);
      CK(cub::DeviceRadixSort::SortPairs(cub_tmp.p, tb, t_tmp.p, t_ikeys.p, b_iw_kept.p, t_iw.p, (int)nkept, 0,
                                         eb, s));
    } else {
      CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, t_tmp.p, t_ikeys.p, (int)nkept, 0, eb, s));
      cub_ensure(tb);
      CK(cub::DeviceRadixSort::SortKeys(cub_tmp.p, tb, t_tmp.p, t_ikeys.p, (int)nkept, 0, eb, s));
    }
    InsertCtx c{};
    c.arena_top = in_top.p;
    c.arena_cap[0] = in_capslots;
    c.arena_cap[1] = 0;
    c.err = b_err.p;
    c.wbase = wbase.p;
    CK(cudaMemsetAsync(b_stat.p, 0, sizeof(unsigned long long) * 2, s));
    { ++n_launch; k_insert_plan<<<grid_elem(nkept), 256, 0, s>>>(gi, t_ikeys.p, b_nkept.p, c, 1, b_stat.p); }
    unsigned long long h[2], tops[2];
    CK(cudaMemcpyAsync(h, b_stat.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(tops, in_top.p, sizeof(tops), cudaMemcpyDeviceToHost, s));
    sync();
    if (tops[0] + h[0] > in_capslots) {  // no room for the relocations: transpose again
      in_build(fview(0, special(0)), fview(1, special(1)));
      return;
    }
    rl_vtx.ensure(batch_cap(nkept + 1));
    rl_len.ensure(batch_cap(nkept + 1));
    rl_from.ensure(batch_cap(nkept + 1));
    rl_to.ensure(batch_cap(nkept + 1));
    c.rl_vtx = rl_vtx.p;
    c.rl_from = rl_from.p;
    c.rl_to = rl_to.p;
    c.rl_len = rl_len.p;
    c.rl_count64 = rl_count.p;
    CK(cudaMemsetAsync(rl_count.p, 0, sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(b_err.p, 0, sizeof(unsigned int), s));
    { ++n_launch; k_insert_plan<<<grid_elem(nkept), 256, 0, s>>>(gi, t_ikeys.p, b_nkept.p, c, 0, nullptr); }
    { ++n_launch; k_insert_write<<<grid_elem(nkept), 256, 0, s>>>(gi, t_ikeys.p, in_w() ? t_iw.p : nullptr,
                                                      b_nkept.p, wbase.p); }
    CK(cudaMemsetAsync(special(6), 0, sizeof(unsigned long long) * 2, s));
    { ++n_launch; k_reloc_frontier<<<grid_elem(nkept), 256, 0, s>>>(rl_count.p, rl_len.p, fview(0, special(6))); }
    { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fview(0, special(6)), fview(1, special(7)),
                                                 RelocCopyOp{gi, rl_from.p, rl_to.p}, nullptr); }
    CK(cudaGetLastError());
    unsigned int herr = 0;
    CK(cudaMemcpyAsync(&herr, b_err.p, sizeof(herr), cudaMemcpyDeviceToHost, s));
    sync();
    if (herr) fail(SGS_ERR_OOM, "in-edge arena exhausted while inserting");
  }

  // ------------------------------------------------------------- graph load
  // Lays the graph out in arenas from a device CSR: per-vertex capacity with
  // slack, offsets by an exclusive scan, the first `split` vertices in HBM
  // (as many whole segments as the HBM budget allows), the rest pinned host.
  void load_device_csr(uint32_t n, const uint64_t *d_row, const uint32_t *d_col,
                       const uint32_t *d_w) {
    if (n == 0) fail(SGS_ERR_INVALID, "empty graph");
    if (n >= (1u << 27)) fail(SGS_ERR_INVALID, "more than 2^27-1 vertices is not supported");
    queries.clear();
    groups.clear();
    apps.clear();  // user algorithms belong to the old graph
    fg = nullptr;
    frun = fsusp = 0;
    loaded = false;
    in_release();
    in_failed = false;
    pr_warm.release();
    if (sc) CK(cudaStreamSynchronize(sc));
    stg_head = stg_count = 0;  // staged batches belonged to the old graph
    est = sgs_engine_stats{};
    nv = n;
    uint64_t ne_in = 0;
    CK(cudaMemcpyAsync(&ne_in, d_row + nv, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    sync();
    if (ne_in >= (1ull << CNT_SHIFT)) fail(SGS_ERR_INVALID, "too many edges");
    if (cfg.weight_mode == SGS_W_EXPLICIT && ne_in && !d_w)
      fail(SGS_ERR_INVALID, "explicit weight mode needs weights");
    {
      CK(cudaMemsetAsync(b_err.p, 0, sizeof(unsigned int), s));
      { ++n_launch; k_validate_csr<<<grid_elem(std::max<uint64_t>(ne_in, nv)), 256, 0, s>>>(
          d_row, d_col, cfg.weight_mode == SGS_W_EXPLICIT ? d_w : nullptr, n, ne_in, b_err.p); }
      CK(cudaGetLastError());
      unsigned int herr = 0;
      CK(cudaMemcpyAsync(&herr, b_err.p, sizeof(herr), cudaMemcpyDeviceToHost, s));
      sync();
      if (herr & 4u) fail(SGS_ERR_INVALID, "row offsets must start at 0 and not decrease");
      if (herr & 1u) fail(SGS_ERR_INVALID, "edge destination out of range");
      if (herr & 2u) fail(SGS_ERR_INVALID, "edge weight 0 (weights must be >= 1)");
    }
    off.ensure(nv);
    slots.ensure(nv);
    live.ensure(nv);
    cap.ensure(nv);
    { ++n_launch; k_row_degrees<<<grid_elem(nv), 256, 0, s>>>(d_row, nv, slots.p); }
    CK(cudaGetLastError());
    layout_from(slots.p, /*extra=*/0);
    CK(cudaMemcpyAsync(live.p, slots.p, sizeof(uint32_t) * nv, cudaMemcpyDeviceToDevice, s));
    // copy lists
    reset_counters(1);
    FrontierView f0 = fview(0, special(0));
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(view(), f0); }
    LoadCsrOp op{view(), d_row, d_col, cfg.weight_mode == SGS_W_EXPLICIT ? d_w : nullptr};
    { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(f0, fview(1, special(1)), op, nullptr); }
    CK(cudaGetLastError());
    sync();
    ne = ne_in;
    slots_total = ne_in;
    loaded = true;
  }

  // New arena layout for blocks whose sizes are in `sz` (slots): capacities
  // with slack, offsets, tier split, arena allocation.  Leaves off/cap set and
  // the arenas allocated but empty; returns nothing (fills members).
  void layout_from(const uint32_t *sz, uint64_t extra) {
    cache_quiesce();
    DBuf<uint64_t> scan;
    scan.ensure((size_t)nv + 1);
    { ++n_launch; k_layout_caps<<<grid_elem(nv), 256, 0, s>>>(sz, nv, cfg.slack_div, cap.p); }
    { ++n_launch; k_u32_to_u64<<<grid_elem(nv), 256, 0, s>>>(cap.p, nv, scan.p); }
    CK(cudaMemsetAsync(scan.p + nv, 0, sizeof(uint64_t), s));
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, scan.p, scan.p, (int)(nv + 1), s));
    cub_ensure(tb);
    CK(cub::DeviceScan::ExclusiveSum(cub_tmp.p, tb, scan.p, scan.p, (int)(nv + 1), s));
    std::vector<uint64_t> hs((size_t)nv + 1);
    CK(cudaMemcpyAsync(hs.data(), scan.p, sizeof(uint64_t) * (nv + 1), cudaMemcpyDeviceToHost, s));
    sync();
    const uint64_t total = hs[nv];
    // tier split on segment boundaries
    uint32_t sp = nv;
    if (cfg.hbm_budget_gb > 0) {
      const double budget_slots = static_budget_gb() * 1e9 / (double)wbytes();
      const double usable = budget_slots / (1.0 + std::max(0.0, cfg.arena_headroom));
      const uint32_t nseg = std::max<uint32_t>(1, cfg.segments);
      // segment s = vertices [b_s, b_{s+1}) with ~total/nseg slots each
      sp = 0;
      for (uint32_t sg = 1; sg <= nseg; ++sg) {
        // segment boundaries by slot count; the last one ends at nv so that
        // trailing empty vertices stay with the resident segments
        uint64_t target = (uint64_t)((double)total * sg / nseg);
        uint32_t b = sg == nseg ? nv
                                : (uint32_t)(std::lower_bound(hs.begin(), hs.end(), target) - hs.begin());
        b = std::min(b, nv);
        // the resident blocks plus the room asked for relocations must fit
        if ((double)hs[b] + (double)extra <= usable) sp = b;
        else break;
      }
    }
    split = sp;
    const double hr = std::max(0.0, cfg.arena_headroom);
    uint64_t need_d = hs[sp], need_h = total - hs[sp];
    uint64_t cap_d = need_d + (uint64_t)(need_d * hr) + 4096 + (sp > 0 ? extra : 0);
    uint64_t cap_h = need_h ? need_h + (uint64_t)(need_h * hr) + 4096 + extra : 0;
    if (cfg.hbm_budget_gb > 0) {
      const uint64_t budget_slots = (uint64_t)(static_budget_gb() * 1e9 / (double)wbytes());
      cap_d = std::min(cap_d, std::max(budget_slots, need_d));
      if (sp < nv && cap_h < need_h + extra) cap_h = need_h + extra + 4096;
    }
    cap_h = (cap_h + CLINE - 1) / CLINE * CLINE;  // whole cache lines
    // the HBM arena, then (with the edge cache) the cache lines after it, so
    // a block held in one cached line reads like an HBM block; the lines
    // start on a line boundary (cap_d itself need not be a multiple of 4,
    // and the quads read from a line are 16-B loads)
    cbase = (cap_d + CLINE - 1) / CLINE * CLINE;
    const uint64_t cache_slots = cache_on ? c_lines * CLINE : 0;
    adj_d.ensure(cbase + cache_slots);
    if (cfg.weight_mode == SGS_W_EXPLICIT) wgt_d.ensure(cbase + cache_slots);
    if (cap_h) {
      adj_h.ensure(cap_h);
      if (cfg.weight_mode == SGS_W_EXPLICIT) wgt_h.ensure(cap_h);
    }
    arena_cap[0] = cap_d;
    arena_cap[1] = cap_h;
    cache_layout(cap_h);
    { ++n_launch; k_assign_off<<<grid_elem(nv), 256, 0, s>>>(scan.p, nv, sp, hs[sp], off.p); }
    unsigned long long tops[2] = {need_d, need_h};
    CK(cudaMemcpyAsync(arena_top.p, tops, sizeof(tops), cudaMemcpyHostToDevice, s));
    ensure_frontier(cap_d + cap_h);
    est.arena_bytes_hbm = cap_d * wbytes();
    est.arena_bytes_host = cap_h * wbytes();
    est.hbm_resident_vertices = sp;
    sync();
  }

  void ensure_frontier(uint64_t max_slots) {
    // padded ranges: at most 3 extra positions per vertex
    const uint64_t max_pos = max_slots + 3ull * nv;
    const uint32_t need_u = (uint32_t)std::min<uint64_t>(max_pos / UNIT + 2, 0xFFFFFFF0ull);
    for (int i = 0; i < 3; ++i) {
      gm[i].ensure(nv);
      CK(cudaMemsetAsync(gm[i].p, 0, sizeof(uint32_t) * nv, s));
      if (wm[i].p) {
        wm[i].ensure(nv);
        CK(cudaMemsetAsync(wm[i].p, 0, sizeof(unsigned long long) * nv, s));
      }
      fb[i].vtx.ensure((size_t)nv + 1);
      fb[i].len.ensure((size_t)nv + 1);
      fb[i].ebase.ensure((size_t)nv + 1);
      if (need_u > ucap) fb[i].ustart.ensure(need_u);
    }
    if (need_u > ucap) ucap = need_u;
    emark.ensure(nv);
    CK(cudaMemsetAsync(emark.p, 0, sizeof(uint32_t) * nv, s));
    estamp = 1;
  }

  // Repack: fresh arenas sized from the current slot counts (+extra room),
  // every block copied (tombstones included).
  void repack(uint64_t extra) {
    cache_quiesce();  // no line copy may read the old host arena
    DBuf<uint64_t> old_off;
    old_off.ensure(nv);
    CK(cudaMemcpyAsync(old_off.p, off.p, sizeof(uint64_t) * nv, cudaMemcpyDeviceToDevice, s));
    DBuf<uint32_t> od, ow;
    HBuf<uint32_t> oh, ohw;
    std::swap(od.p, adj_d.p); std::swap(od.n, adj_d.n);
    std::swap(ow.p, wgt_d.p); std::swap(ow.n, wgt_d.n);
    std::swap(oh.p, adj_h.p); std::swap(oh.n, adj_h.n);
    std::swap(ohw.p, wgt_h.p); std::swap(ohw.n, wgt_h.n);
    layout_from(slots.p, extra);
    reset_counters(1);
    FrontierView f0 = fview(0, special(0));
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(view(), f0); }
    CopyBlockOp op{view(), old_off.p, off.p, od.p, ow.p, oh.p, ohw.p};
    { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(f0, fview(1, special(1)), op, nullptr); }
    CK(cudaGetLastError());
    sync();
    ++repacks;
  }

  void reset_counters(uint32_t) {
    CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2 + kSpecial), s));
  }

  // ----------------------------------------------------------- convergence
  // Runs relaxation rounds from the frontier in buffer 0 / cnt[0] until a
  // round produces an empty frontier.  Rounds are queued in batches; the
  // host reads the batch's counters once.
  void ensure_gev(size_t n) {
    while (gev.size() < n) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      gev.push_back(e);
    }
  }
  void ensure_kev(size_t n) {
    while (kev.size() < n) {
      cudaEvent_t ev;
      CK(cudaEventCreate(&ev));
      kev.push_back(ev);
    }
  }

  // Accounts one timed launch: in = packed input counter of the launch,
  // inst = (instance, edge) pairs it relaxed, per_slot / per_inst = bytes.
  void account(int kind, unsigned long long in, unsigned long long inst, double per_slot,
               double per_inst, cudaEvent_t a, cudaEvent_t b, unsigned long long host = 0) {
    const uint64_t n = in >> CNT_SHIFT, T = in & EDGE_MASK;
    if (!n) return;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    account_n(kind, n, T, inst, per_slot, per_inst, ms, host);
  }
  // The same with the entry and slot counts given apart (a launch that ran
  // several rounds over one frontier) and its time in ms.
  void account_n(int kind, uint64_t n, uint64_t T, unsigned long long inst, double per_slot,
                 double per_inst, double ms, unsigned long long host = 0) {
    sgs_kernel_stats &k = kst[kind];
    const double bytes = per_slot * (double)T + per_inst * (double)inst + 20.0 * (double)n;
    k.launches += 1;
    k.slots += T;
    k.entries += n;
    k.bytes_alg += bytes;
    k.ms += ms;
    k.host_slots += host;
    if (T > k.max_slots) {
      k.max_slots = T;
      k.max_entries = n;
      k.max_bytes_alg = bytes;
      k.max_ms = ms;
      k.max_host_slots = host;
    }
  }

  // Rounds of a group op from the frontier in buffer 0 / cnt[0] (lane masks in
  // gm[0]) until a round appends nothing.  Rounds are queued in batches and
  // the host reads the batch's counters once.  Masks of the last non-empty
  // frontier are cleared at the end, so all mask buffers are zero again.
  template <class MakeOp>
  uint32_t run_group_rounds(MakeOp make_op, bool &converged, int kind, double per_slot,
                            const char *round0 = nullptr,
                            const std::function<void()> *after0 = nullptr) {
    return run_rounds(
        [&](uint32_t rr) { launch_group(rr, make_op(rr, gm[rr % 3].p, gm[(rr + 1) % 3].p)); },
        false, converged, kind, per_slot, round0, after0);
  }

  // The same for a wide group op (wide_map, u64 masks in wm); `op0` for
  // round 0, `op` for the others.
  template <class Op0, class Op>
  uint32_t run_wide_rounds(const Op0 &op0, const Op &op, bool &converged, int kind, double per_slot,
                           unsigned long long *lane_changes, const char *round0 = nullptr,
                           const std::function<void()> *after0 = nullptr) {
    return run_rounds(
        [&](uint32_t rr) {
          if (rr == 0) launch_wide(rr, op0, lane_changes);
          else launch_wide(rr, op, lane_changes);
        },
        true, converged, kind, per_slot, round0, after0);
  }

  template <class Op>
  void launch_wide(uint32_t rr, const Op &op, unsigned long long *lane_changes) {
    const bool hp = rr >= 1;
    auto k = host_tier() ? wide_map<Op, true> : wide_map<Op, false>;
    { ++n_launch; k<<<grid_map(), RELAX_THREADS, 0, s>>>(
        view(), fview(rr, cnt.p + rr), fview(rr + 1, cnt.p + rr + 1), op, wm[rr % 3].p,
        wm[(rr + 1) % 3].p, hp ? fb[(rr - 1) % 3].vtx.p : nullptr,
        hp ? cnt.p + rr - 1 : nullptr, hp ? wm[(rr - 1) % 3].p : nullptr, b_lane.p,
        lane_changes, rstat.p + rr); }
  }

  template <class Op>
  void launch_group(uint32_t rr, const Op &op) {
    const bool hp = rr >= 1;
    auto k = host_tier() ? group_map<Op, true> : group_map<Op, false>;
    { ++n_launch; k<<<grid_map(), RELAX_THREADS, 0, s>>>(
        fview(rr, cnt.p + rr), fview(rr + 1, cnt.p + rr + 1), op,
        hp ? fb[(rr - 1) % 3].vtx.p : nullptr, hp ? cnt.p + rr - 1 : nullptr,
        hp ? gm[(rr - 1) % 3].p : nullptr, b_lane.p, rstat.p + rr, hstat.p + rr); }
  }

  // BFS rounds of the lanes `lanes` (all BFS) of a narrow group, each round
  // top-down (group_map) or bottom-up over the in-edge store
  // (k_bfs_pull_round), chosen on the host from the frontier's size with
  // Beamer's rule: bottom-up once the frontier's out-edges exceed 1/14 of the
  // edges not yet explored, back to top-down when the frontier holds fewer
  // than 1/24 of the vertices.  One counter read per round.
  uint64_t bfs_bottom_up_total = 0;
  uint32_t run_bfs_diropt(Group &G, uint32_t lanes, bool &converged) {
    const GraphView g = view(), gi = in_view();
    const uint32_t maxr = cfg.max_rounds;
    converged = false;
    CK(cudaMemsetAsync(rstat.p, 0, sizeof(unsigned long long) * (maxr + 2), s));
    CK(cudaMemsetAsync(hstat.p, 0, sizeof(unsigned long long) * (maxr + 2), s));
    bool bu = false;
    uint64_t explored = 0;
    for (uint32_t r = 0; r < maxr; ++r) {
      unsigned long long c = 0;
      CK(cudaMemcpyAsync(&c, cnt.p + r, sizeof(c), cudaMemcpyDeviceToHost, s));
      sync();
      const uint64_t nf = c >> CNT_SHIFT, mf = c & EDGE_MASK;
      if (nf == 0) {
        if (r >= 1) clear_masks(false, r - 1);
        CK(cudaGetLastError());
        converged = true;
        return r;
      }
      const uint64_t mu = ne > explored ? ne - explored : 0;
      if (!bu && mf * 14 > mu) bu = true;
      else if (bu && nf * 24 < nv) bu = false;
      explored += mf;
      if (!bu) {
        launch_group(r, GroupRelaxOp<GMAX>{g, G.st.p, G.val.p, gm[r % 3].p, gm[(r + 1) % 3].p, G.algo(), 0});
      } else {
        const bool hp = r >= 1;
        { ++n_launch; k_bfs_pull_round<GMAX><<<grid_elem(nv), RELAX_THREADS, 0, s>>>(
            g, gi, G.st.p, G.val.p, lanes, gm[r % 3].p, gm[(r + 1) % 3].p, fview(r, cnt.p + r),
            hp ? fb[(r - 1) % 3].vtx.p : nullptr, hp ? cnt.p + r - 1 : nullptr,
            hp ? gm[(r - 1) % 3].p : nullptr, fview(r + 1, cnt.p + r + 1), b_lane.p); }
        ++bfs_bottom_up_total;
      }
      CK(cudaGetLastError());
    }
    for (uint32_t f = maxr >= 1 ? maxr - 1 : 0; f <= maxr; ++f) clear_masks(false, f);
    return maxr;
  }

  // Round loop shared by both group widths: `launch(rr)` queues round rr.
  template <class Launch>
  uint32_t run_rounds(Launch launch, bool wide, bool &converged, int kind, double per_slot,
                      const char *round0, const std::function<void()> *after0 = nullptr) {
    // no host read before the first batch: an empty start costs a few
    // launches that exit at once, a host round trip costs more
    const uint32_t maxr = cfg.max_rounds;
    uint32_t r = 0, rb = 4;
    converged = false;
    CK(cudaMemsetAsync(rstat.p, 0, sizeof(unsigned long long) * (maxr + 2), s));
    CK(cudaMemsetAsync(hstat.p, 0, sizeof(unsigned long long) * (maxr + 2), s));
    std::vector<unsigned long long> hr(18), hh(18);
    while (r < maxr) {
      const uint32_t nb = std::min(rb, maxr - r);
      if (ktiming) ensure_kev(2 * nb);
      for (uint32_t k = 0; k < nb; ++k) {
        const uint32_t rr = r + k;
        if (ktiming) CK(cudaEventRecord(kev[2 * k], s));
        if (rr == 0 && round0) nvtxRangePushA(round0);
        launch(rr);
        if (rr == 0 && round0) nvtxRangePop();
        if (rr == 0 && after0) (*after0)();
        if (ktiming) CK(cudaEventRecord(kev[2 * k + 1], s));
      }
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(h_cnt, cnt.p + r, sizeof(unsigned long long) * (nb + 1),
                         cudaMemcpyDeviceToHost, s));
      if (ktiming) {
        CK(cudaMemcpyAsync(hr.data(), rstat.p + r, sizeof(unsigned long long) * nb,
                           cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(hh.data(), hstat.p + r, sizeof(unsigned long long) * nb,
                           cudaMemcpyDeviceToHost, s));
      }
      sync();
      if (ktiming)
        for (uint32_t k = 0; k < nb; ++k)
          account(kind, h_cnt[k], hr[k], per_slot, 8.0, kev[2 * k], kev[2 * k + 1], hh[k]);
      for (uint32_t k = 0; k < nb; ++k)
        if (h_cnt[k + 1] == 0) {
          const uint32_t z = r + k + 1;  // first empty frontier
          clear_masks(wide, z - 1);
          CK(cudaGetLastError());
          converged = true;
          return z;
        }
      r += nb;
      rb = std::min<uint32_t>(rb * 2, 16);
    }
    // not converged: leave the masks clean for the next call
    for (uint32_t f = (r >= 1 ? r - 1 : 0); f <= r; ++f) clear_masks(wide, f);
    CK(cudaGetLastError());
    return r;
  }

  // ------------------------------------------------- persistent round loops
  std::map<const void *, int> coop_cache;
  DBuf<uint32_t> d_rounds;
  // One wave of co-resident CTAs for a cooperative launch.
  int coop_grid(const void *f) {
    auto it = coop_cache.find(f);
    if (it != coop_cache.end()) return it->second;
    int b = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, RELAX_THREADS, 0));
    if (b < 1) fail(SGS_ERR_CUDA, "persistent round kernel cannot be resident");
    const int g = nsm * b;
    coop_cache[f] = g;
    return g;
  }
  template <class M>
  RoundBufs<M> round_bufs(DBuf<M> (&masks)[3]) {
    RoundBufs<M> rb;
    for (int i = 0; i < 3; ++i) {
      rb.vtx[i] = fb[i].vtx.p;
      rb.len[i] = fb[i].len.p;
      rb.ebase[i] = fb[i].ebase.p;
      rb.ustart[i] = fb[i].ustart.p;
      rb.mask[i] = masks[i].p;
    }
    rb.cnt = cnt.p;
    rb.ucap = ucap;
    return rb;
  }
  // After a persistent launch: its round count (one host read) and, with
  // kernel timing, the whole launch accounted as one.
  uint32_t finish_persistent(uint32_t r0, bool &converged, int kind, double per_slot,
                             cudaEvent_t a, cudaEvent_t b) {
    uint32_t rounds = 0;
    CK(cudaMemcpyAsync(&rounds, d_rounds.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    std::vector<unsigned long long> hc, hr, hh;
    if (ktiming) {
      const size_t m = cfg.max_rounds + 2;
      hc.resize(m);
      hr.resize(m);
      hh.resize(m);
      CK(cudaMemcpyAsync(hc.data(), cnt.p, sizeof(unsigned long long) * m, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(hr.data(), rstat.p, sizeof(unsigned long long) * m, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(hh.data(), hstat.p, sizeof(unsigned long long) * m, cudaMemcpyDeviceToHost, s));
    }
    sync();
    converged = rounds < cfg.max_rounds;
    if (ktiming) {
      unsigned long long n = 0, T = 0, inst = 0, host = 0;
      for (uint32_t r = r0; r < rounds && r < cfg.max_rounds; ++r) {
        n += hc[r] >> CNT_SHIFT;
        T += hc[r] & EDGE_MASK;
        inst += hr[r];
        host += hh[r];
      }
      if (n) account(kind, (n << CNT_SHIFT) | T, inst, per_slot, 8.0, a, b, host);
    }
    return rounds;
  }
  template <class Op>
  uint32_t run_group_persistent(const Op &op, uint32_t r0, bool &converged, int kind, double per_slot) {
    d_rounds.ensure(1);
    if (r0 == 0) {
      CK(cudaMemsetAsync(rstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
      CK(cudaMemsetAsync(hstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
    }
    RoundBufs<uint32_t> rb = round_bufs(gm);
    uint32_t maxr = cfg.max_rounds;
    unsigned long long *le = b_lane.p, *rs = rstat.p, *hs = hstat.p;
    uint32_t *ro = d_rounds.p;
    Op o = op;
    void *args[] = {&rb, &o, &r0, &maxr, &le, &rs, &hs, &ro};
    const void *f = host_tier() ? (const void *)group_rounds<Op, true> : (const void *)group_rounds<Op, false>;
    if (ktiming) { ensure_kev(2); CK(cudaEventRecord(kev[0], s)); }
    ++n_launch;
    CK(cudaLaunchCooperativeKernel(f, coop_grid(f), RELAX_THREADS, args, 0, s));
    if (ktiming) CK(cudaEventRecord(kev[1], s));
    return finish_persistent(r0, converged, kind, per_slot, ktiming ? kev[0] : nullptr,
                             ktiming ? kev[1] : nullptr);
  }
  template <class Op>
  uint32_t run_wide_persistent(const Op &op, uint32_t r0, bool &converged, int kind, double per_slot,
                               unsigned long long *lane_changes) {
    d_rounds.ensure(1);
    if (r0 == 0) CK(cudaMemsetAsync(rstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
    CK(cudaMemsetAsync(hstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
    GraphView g = view();
    RoundBufs<unsigned long long> rb = round_bufs(wm);
    uint32_t maxr = cfg.max_rounds;
    unsigned long long *le = b_lane.p, *lc = lane_changes, *rs = rstat.p;
    uint32_t *ro = d_rounds.p;
    Op o = op;
    void *args[] = {&g, &rb, &o, &r0, &maxr, &le, &lc, &rs, &ro};
    const void *f = host_tier() ? (const void *)wide_rounds<Op, true> : (const void *)wide_rounds<Op, false>;
    if (ktiming) { ensure_kev(2); CK(cudaEventRecord(kev[0], s)); }
    ++n_launch;
    CK(cudaLaunchCooperativeKernel(f, coop_grid(f), RELAX_THREADS, args, 0, s));
    if (ktiming) CK(cudaEventRecord(kev[1], s));
    return finish_persistent(r0, converged, kind, per_slot, ktiming ? kev[0] : nullptr,
                             ktiming ? kev[1] : nullptr);
  }

  // Masks of the frontier of round f (buffer f % 3, counter cnt[f]).
  void clear_masks(bool wide, uint32_t f) {
    if (wide)
      { ++n_launch; k_clear_masks64<<<grid_elem(nv), 256, 0, s>>>(fb[f % 3].vtx.p, cnt.p + f, wm[f % 3].p); }
    else
      { ++n_launch; k_clear_masks<<<grid_elem(nv), 256, 0, s>>>(fb[f % 3].vtx.p, cnt.p + f, gm[f % 3].p); }
  }

  void ensure_wide_masks() {
    for (int i = 0; i < 3; ++i)
      if (!wm[i].p || wm[i].n < nv) {
        wm[i].ensure(nv);
        CK(cudaMemsetAsync(wm[i].p, 0, sizeof(unsigned long long) * nv, s));
      }
  }

  // Relaxation rounds for the lanes whose frontier is in buffer 0.  With
  // `only0` (wide groups: per vertex the lanes reset there), round 0 relaxes
  // an edge only in the lanes its destination had reset, i.e. only edges into
  // bitmap; `after0` runs right after round 0 (it may append to frontier 1).
  uint32_t group_relax(Group &G, bool &conv, const char *round0 = nullptr,
                       const unsigned long long *only0 = nullptr,
                       const std::function<void()> *after0 = nullptr) {
    GraphView g = view();
    if (G.wide()) {
      const bool anyw = G.sssp && cfg.weight_mode == SGS_W_EXPLICIT;
      WideRelaxOp<> op{G.st.p, G.val.p, G.walgo()};
      WideRelaxOp<true> op0{G.st.p, G.val.p, G.walgo()};
      op0.only = only0;
      if (cfg.persistent & 1u) {  // (bit 2 is for narrow groups: the wide
                                  // cooperative grid is capped at 3 CTAs/SM,
                                  // too few for their heavier later rounds)
        if (!only0 && !after0) return run_wide_persistent(op, 0, conv, SGS_K_WIDE, anyw ? 8.0 : 4.0, nullptr);
        // round 0 (restricted) and its hook as plain launches, then one launch
        CK(cudaMemsetAsync(rstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
        if (round0) nvtxRangePushA(round0);
        if (only0) launch_wide(0, op0, nullptr);
        else launch_wide(0, op, nullptr);
        if (round0) nvtxRangePop();
        if (after0) (*after0)();
        return run_wide_persistent(op, 1, conv, SGS_K_WIDE, anyw ? 8.0 : 4.0, nullptr);
      }
      if (only0)
        return run_wide_rounds(op0, op, conv, SGS_K_WIDE, anyw ? 8.0 : 4.0, nullptr, round0, after0);
      return run_wide_rounds(op, op, conv, SGS_K_WIDE, anyw ? 8.0 : 4.0, nullptr, round0, after0);
    }
    const uint32_t anyw = G.any_sssp(G.used | 0xF) && cfg.weight_mode == SGS_W_EXPLICIT;
    if ((cfg.persistent & 4u) && !(cfg.persistent & 1u) && !after0) {
      // round 0 (a snapshot's sweep, or a start's first round) as a plain
      // launch on the large grid, the rest of the phase as one cooperative
      // launch: the sweep wants the grid, the small later rounds want no
      // host round trips
      CK(cudaMemsetAsync(rstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
      CK(cudaMemsetAsync(hstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
      if (round0) nvtxRangePushA(round0);
      if (ktiming) { ensure_kev(2); CK(cudaEventRecord(kev[0], s)); }
      launch_group(0, GroupRelaxOp<GMAX>{g, G.st.p, G.val.p, gm[0].p, gm[1].p, G.algo(), anyw});
      if (ktiming) {
        CK(cudaEventRecord(kev[1], s));
        unsigned long long c0 = 0, r0s = 0, h0 = 0;
        CK(cudaMemcpyAsync(&c0, cnt.p, sizeof(c0), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&r0s, rstat.p, sizeof(r0s), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&h0, hstat.p, sizeof(h0), cudaMemcpyDeviceToHost, s));
        sync();
        account(SGS_K_GROUP_SWEEP, c0, r0s, anyw ? 8.0 : 4.0, 8.0, kev[0], kev[1], h0);
      }
      if (round0) nvtxRangePop();
      return run_group_persistent(GroupRelaxOp<GMAX>{g, G.st.p, G.val.p, nullptr, nullptr, G.algo(), anyw}, 1,
                                  conv, SGS_K_GROUP, anyw ? 8.0 : 4.0);
    }
    if ((cfg.persistent & 1u) && !after0) {
      if (round0) nvtxRangePushA(round0);
      const uint32_t r = run_group_persistent(
          GroupRelaxOp<GMAX>{g, G.st.p, G.val.p, nullptr, nullptr, G.algo(), anyw}, 0, conv, SGS_K_GROUP,
          anyw ? 8.0 : 4.0);
      if (round0) nvtxRangePop();
      return r;
    }
    return run_rounds(
        [&](uint32_t rr) {
          uint32_t *mi = gm[rr % 3].p, *mo = gm[(rr + 1) % 3].p;
          launch_group(rr, GroupRelaxOp<GMAX>{g, G.st.p, G.val.p, mi, mo, G.algo(), anyw});
        },
        false, conv, SGS_K_GROUP, anyw ? 8.0 : 4.0, round0, after0);
  }

  // PageRank rounds over the static frontier of all non-empty blocks:
  // absorb (value += residual) then push alpha*res/outdeg; stop after the
  // first round whose absorbed residual L1 is below pr_tol.
  // Rounds of the PageRank sweep over all vertices: absorb (value +=
  // residual, push value = alpha * residual / outdeg), then the residual of
  // every vertex from its in-neighbours' push values -- a pull over the
  // in-edge store when it is there (cfg.pull), else a push over the
  // out-blocks with FP64 atomics.
  uint32_t pr_rounds(Query &q, unsigned long long *edge_stat, bool &conv, double &last_l1) {
    const bool pull = (cfg.pull & 1u) && ensure_in();
    const GraphView gi = pull ? in_view() : view();
    reset_counters(0);
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(gi, fview(0, cnt.p)); }
    const uint32_t maxr = cfg.max_rounds;
    CK(cudaMemsetAsync(l1.p, 0, sizeof(double) * (maxr + 2), s));
    unsigned long long pr_in = 0;
    CK(cudaMemcpyAsync(&pr_in, cnt.p, sizeof(pr_in), cudaMemcpyDeviceToHost, s));
    sync();
    return pr_steps(q, fview(0, cnt.p), fview(1, cnt.p + 1), pull, l1.p, 0, maxr, edge_stat, pr_in, conv,
                    last_l1);
  }

  // Rounds r0, r0+1, ... (at most `limit`) over a prebuilt dense frontier
  // `fin` of the store the sweep reads (in-edge store when `pull`); per-round
  // absorbed L1 in l1buf[r].  Returns the rounds run; conv when a round's L1
  // falls below pr_tol.
  uint32_t pr_steps(Query &q, FrontierView fin, FrontierView fout, bool pull, double *l1buf, uint32_t r0,
                    uint32_t limit, unsigned long long *edge_stat, unsigned long long pr_in, bool &conv,
                    double &last_l1) {
    const GraphView g = view();
    const GraphView gi = pull ? in_view() : g;
    std::vector<double> hl(34);
    uint32_t r = 0, rb = 8;
    conv = false;
    last_l1 = 0;
    PrPushOp op{g, q.pv.p, q.r.p};
    const unsigned long long pr_inst = (pr_in & EDGE_MASK);
    // all rounds in one cooperative launch (k_pr_rounds, one host read) when
    // the sweep's units fit one wave of it -- a graph small enough that the
    // launches and host reads of the round loop, not the sweeps, set the
    // time; a larger one keeps the multi-wave launches, which balance better
    const void *fn = (const void *)k_pr_rounds;
    const uint64_t units = ((pr_in & EDGE_MASK) + UNIT - 1) / UNIT;
    if (pull && (cfg.persistent & 8u) && limit && units <= (uint64_t)coop_grid(fn)) {
      d_rounds.ensure(1);
      GraphView ga = g, gb = gi;
      FrontierView f = fin;
      double *x = q.x.p, *rp = q.r.p, *pv = q.pv.p, *l1b = l1buf;
      double alpha = cfg.pr_alpha, tol = cfg.pr_tol;
      uint32_t r0a = r0, lim = limit;
      unsigned long long *es = edge_stat;
      uint32_t *ro = d_rounds.p;
      void *args[] = {&ga, &f, &gb, &x, &rp, &pv, &alpha, &tol, &l1b, &r0a, &lim, &es, &ro};
      // no more CTAs than units (idle CTAs only lengthen the grid barriers)
      const int grid = (int)std::max<uint64_t>(std::min<uint64_t>(units, (uint64_t)coop_grid(fn)), nsm);
      if (ktiming) {
        ensure_kev(2);
        CK(cudaEventRecord(kev[0], s));
      }
      ++n_launch;
      CK(cudaLaunchCooperativeKernel(fn, grid, RELAX_THREADS, args, 0, s));
      if (ktiming) CK(cudaEventRecord(kev[1], s));
      uint32_t ran = 0;
      hl.resize(limit);
      CK(cudaMemcpyAsync(&ran, d_rounds.p, sizeof(ran), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(hl.data(), l1buf + r0, sizeof(double) * limit, cudaMemcpyDeviceToHost, s));
      sync();
      if (ran > limit) fail(SGS_ERR_CUDA, "PageRank round kernel returned a bad round count");
      if (ran) {
        last_l1 = hl[ran - 1];
        conv = last_l1 < cfg.pr_tol;
      }
      if (ktiming && ran) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, kev[0], kev[1]));
        account_n(SGS_K_PR_PULL, (pr_in >> CNT_SHIFT) * ran, pr_inst * ran, pr_inst * ran, 4.0, 16.0, ms);
      }
      return ran;
    }
    while (r < limit) {
      const uint32_t nb = std::min(rb, limit - r);
      if (ktiming) ensure_kev(2 * nb);
      for (uint32_t k = 0; k < nb; ++k) {
        { ++n_launch; k_pr_absorb<<<grid_elem(nv), RELAX_THREADS, 0, s>>>(g, q.x.p, q.r.p, q.pv.p, cfg.pr_alpha,
                                                           l1buf + r0 + r + k); }
        if (ktiming) CK(cudaEventRecord(kev[2 * k], s));
        if (pull)
          { ++n_launch; k_pull_pr<<<grid_map(), RELAX_THREADS, 0, s>>>(fin, gi, q.pv.p, q.r.p, edge_stat); }
        else
          { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fin, fout, op, edge_stat); }
        if (ktiming) CK(cudaEventRecord(kev[2 * k + 1], s));
      }
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(hl.data(), l1buf + r0 + r, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
      sync();
      if (ktiming)
        for (uint32_t k = 0; k < nb; ++k)
          account(pull ? SGS_K_PR_PULL : SGS_K_PR_PUSH, pr_in, pr_inst, 4.0, 16.0, kev[2 * k],
                  kev[2 * k + 1]);
      for (uint32_t k = 0; k < nb; ++k) {
        last_l1 = hl[k];
        if (hl[k] < cfg.pr_tol) { conv = true; return r + k + 1; }
      }
      r += nb;
      rb = std::min<uint32_t>(rb * 2, 32);
    }
    return r;
  }

  // ------------------------------------------------------- PageRank jobs
  // A PageRank computation the served loop advances a few rounds at a time
  // between the steps of its query flight.  It has its own frontier buffers
  // and counters, so its rounds do not disturb the flight's.
  struct PrJob {
    Query *q = nullptr;
    bool pull = false;
    uint32_t r = 0;
    Frontier f;
    uint32_t ucap = 0;
    DBuf<unsigned long long> c;  // [0] frontier counter, [1] output counter, [2] edge count
    DBuf<double> l1;
    unsigned long long pr_in = 0;
    float ms = 0;
    // a snapshot was applied while the job ran: its residual was amended
    // like any PageRank query's, and its dense frontier (block sizes of the
    // old graph) is rebuilt before the next sweep
    bool stale = false;
  } job;
  FrontierView job_view(uint32_t k) {
    FrontierView f;
    f.vtx = job.f.vtx.p;
    f.len = job.f.len.p;
    f.ebase = job.f.ebase.p;
    f.ustart = job.f.ustart.p;
    f.counter = (uint64_t *)(job.c.p + k);
    f.ucap = job.ucap;
    return f;
  }
  // The job's dense frontier over the store its sweeps read, for the current
  // graph (buffers sized for a dense frontier of either store).
  void job_frontier() {
    const uint64_t max_pos = std::max<uint64_t>(slots_total, in_capslots) + 3ull * nv;
    job.ucap = (uint32_t)std::min<uint64_t>(max_pos / UNIT + 2, 0xFFFFFFF0ull);
    job.f.ustart.ensure(job.ucap);
    CK(cudaMemsetAsync(job.c.p, 0, sizeof(unsigned long long) * 2, s));
    const GraphView gi = job.pull ? in_view() : view();
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(gi, job_view(0)); }
    CK(cudaMemcpyAsync(&job.pr_in, job.c.p, sizeof(job.pr_in), cudaMemcpyDeviceToHost, s));
    sync();
  }
  int pr_job_start() {
    if (job.q) fail(SGS_ERR_STATE, "a PageRank job is already running");
    // frontier buffers of the job, sized for a dense frontier of either store
    const uint64_t max_pos = slots_total + 3ull * nv;
    job.ucap = (uint32_t)std::min<uint64_t>(max_pos / UNIT + 2, 0xFFFFFFF0ull);
    job.f.vtx.ensure((size_t)nv + 1);
    job.f.len.ensure((size_t)nv + 1);
    job.f.ebase.ensure((size_t)nv + 1);
    job.f.ustart.ensure(job.ucap);
    job.c.ensure(3);
    job.l1.ensure(cfg.max_rounds + 2);
    job.stale = false;
    job.pull = (cfg.pull & 1u) && ensure_in(job_view(0), job_view(1));
    auto q = std::make_unique<Query>();
    q->id = next_qid++;
    q->algo = SGS_PR;
    q->x.ensure(nv);
    q->r.ensure(nv);
    q->pv.ensure(nv);
    CK(cudaEventRecord(ev_q.a, s));
    pr_init(*q, job_view(0), job_view(1));
    CK(cudaMemsetAsync(job.c.p, 0, sizeof(unsigned long long) * 3, s));
    const GraphView gi = job.pull ? in_view() : view();
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(gi, job_view(0)); }
    CK(cudaMemsetAsync(job.l1.p, 0, sizeof(double) * (cfg.max_rounds + 2), s));
    CK(cudaMemcpyAsync(&job.pr_in, job.c.p, sizeof(job.pr_in), cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(ev_q.b, s));
    sync();
    CK(cudaEventElapsedTime(&job.ms, ev_q.a, ev_q.b));
    job.r = 0;
    job.q = q.get();
    q->stats = sgs_query_stats{};
    const int id = q->id;
    queries.push_back(std::move(q));
    return id;
  }
  // Up to `rounds` more rounds; true when the job has finished (converged or
  // at the round limit; its query then holds the result and its stats).
  bool pr_job_advance(uint32_t rounds) {
    if (!job.q) fail(SGS_ERR_STATE, "no PageRank job");
    if (job.stale) {
      job_frontier();
      job.stale = false;
    }
    Query &q = *job.q;
    const uint32_t lim = std::min(rounds, cfg.max_rounds - job.r);
    bool conv = false;
    double l1v = 0;
    CK(cudaEventRecord(ev_q.a, s));
    const uint32_t ran = pr_steps(q, job_view(0), job_view(1), job.pull, job.l1.p, job.r, lim, job.c.p + 2,
                                  job.pr_in, conv, l1v);
    CK(cudaEventRecord(ev_q.b, s));
    sync();
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev_q.a, ev_q.b));
    job.ms += ms;
    job.r += ran;
    q.stats.pr_residual_l1 = l1v;
    if (!conv && job.r < cfg.max_rounds) return false;
    unsigned long long e = 0;
    CK(cudaMemcpyAsync(&e, job.c.p + 2, sizeof(e), cudaMemcpyDeviceToHost, s));
    sync();
    q.stats.edges_traversed = e;
    q.stats.edges_total += e;
    q.stats.rounds = job.r;
    q.stats.converged = conv ? 1 : 0;
    q.stats.ms = job.ms;
    job.q = nullptr;
    return true;
  }

  // ---------------------------------------------------------------- queries
  Query &find(int qid) {
    for (auto &q : queries)
      if (q->id == qid) return *q;
    fail(SGS_ERR_INVALID, "unknown query id");
  }

  // One all-vertex sweep r[v] = sum over in-edges of pv[u] (pull over the
  // in-edge store when it is there, else a push over the out-blocks), with
  // the frontier buffers f0 (input, counter zeroed here) and f1.
  void pr_sweep_once(Query &q, FrontierView f0, FrontierView f1) {
    const GraphView g = view();
    const bool pull = (cfg.pull & 1u) && ensure_in(f0, f1);
    const GraphView gi = pull ? in_view() : g;
    CK(cudaMemsetAsync(f0.counter, 0, sizeof(unsigned long long), s));
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(gi, f0); }
    if (pull)
      { ++n_launch; k_pull_pr<<<grid_map(), RELAX_THREADS, 0, s>>>(f0, gi, q.pv.p, q.r.p, nullptr); }
    else
      { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(f0, f1, PrPushOp{g, q.pv.p, q.r.p}, nullptr); }
    CK(cudaGetLastError());
  }

  // Initial state of a PageRank query: the reference's value 0, residual
  // 1 - alpha, or a warm start from the kept vector of a removed query.
  void pr_init(Query &q, FrontierView f0, FrontierView f1) {
    if (pr_warm.p && pr_warm.n >= nv) {
      // warm start: take over the kept vector, residual of it on this graph
      std::swap(q.x.p, pr_warm.p);
      std::swap(q.x.n, pr_warm.n);
      pr_warm.release();
      const GraphView g = view();
      { ++n_launch; k_pr_warm_pv<<<grid_elem(nv), 256, 0, s>>>(g, q.x.p, q.pv.p, q.r.p, cfg.pr_alpha); }
      pr_sweep_once(q, f0, f1);
      { ++n_launch; k_pr_warm_res<<<grid_elem(nv), 256, 0, s>>>(q.x.p, q.r.p, nv, 1.0 - cfg.pr_alpha); }
      CK(cudaGetLastError());
      ++pr_warm_starts;
    } else {
      { ++n_launch; k_pr_init<<<grid_elem(nv), 256, 0, s>>>(q.x.p, q.r.p, nv, 1.0 - cfg.pr_alpha); }
    }
  }

  void start_pr(Query &q) {
    CK(cudaEventRecord(ev_q.a, s));
    CK(cudaMemsetAsync(b_stat.p, 0, sizeof(unsigned long long) * 8, s));
    bool conv = false;
    double l1v = 0;
    CK(cudaMemsetAsync(special(0), 0, sizeof(unsigned long long) * 2, s));
    pr_init(q, fview(0, special(0)), fview(1, special(1)));
    const uint32_t rounds = pr_rounds(q, b_stat.p + 4, conv, l1v);
    CK(cudaEventRecord(ev_q.b, s));
    unsigned long long e = 0;
    CK(cudaMemcpyAsync(&e, b_stat.p + 4, sizeof(e), cudaMemcpyDeviceToHost, s));
    sync();
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev_q.a, ev_q.b));
    q.stats.edges_traversed = e;
    q.stats.edges_total += e;
    q.stats.rounds = rounds;
    q.stats.converged = conv ? 1 : 0;
    q.stats.ms = ms;
    q.stats.pr_residual_l1 = l1v;
    q.stats.invalidated = 0;
  }

  // Static convergence of the new lanes `fresh` of a group, all together
  // (InitGraph + Start for each of those queries): CC lanes start from a
  // dense frontier, BFS/SSSP lanes from their sources, then one round loop.
  void start_lanes(Group &G, uint64_t fresh, const std::vector<Query *> &qs) {
    // a narrow group whose new lanes are all BFS: direction-optimizing
    // rounds (the in-edge store is built here, before the frontier buffers
    // are seeded, since building it uses them)
    bool all_bfs = !G.wide() && fresh != 0;
    for (int q = 0; q < G.width; ++q)
      if ((fresh >> q & 1ull) && (G.algo_packed >> (8 * q) & 0xFFu) != (uint32_t)A_BFS) all_bfs = false;
    const bool diropt = all_bfs && (cfg.pull & 2u) && ensure_in();
    GraphView g = view();
    CK(cudaEventRecord(ev_q.a, s));
    CK(cudaMemsetAsync(b_lane.p, 0, sizeof(unsigned long long) * WLANES, s));
    reset_counters(0);
    const uint64_t fresh_cc = fresh & G.cc;
    if (G.wide()) {
      ensure_wide_masks();
      { ++n_launch; k_wide_init_lanes<<<grid_elem((uint64_t)nv * 32), 256, 0, s>>>(G.st.p, G.val.p, nv, fresh, G.cc); }
      if (fresh_cc)
        { ++n_launch; k_wide_dense<<<grid_elem(nv), RELAX_THREADS, 0, s>>>(g, G.val.p, fresh_cc, G.cc, wm[0].p,
                                                               fview(0, cnt.p)); }
      std::vector<uint32_t> src, lane;
      for (Query *q : qs)
        if (q->algo != SGS_CC) {
          src.push_back(q->source);
          lane.push_back((uint32_t)q->lane);
        }
      if (!src.empty()) {
        b_seed.ensure(2 * src.size());
        CK(cudaMemcpyAsync(b_seed.p, src.data(), sizeof(uint32_t) * src.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(b_seed.p + src.size(), lane.data(), sizeof(uint32_t) * lane.size(),
                           cudaMemcpyHostToDevice, s));
        { ++n_launch; k_wide_seed_sources<<<grid_elem(src.size()), 256, 0, s>>>(
            g, G.st.p, G.val.p, b_seed.p, b_seed.p + src.size(), (uint32_t)src.size(), wm[0].p,
            fview(0, cnt.p)); }
      }
    } else {
      for (Query *q : qs)
        { ++n_launch; k_group_init_lane<GMAX><<<grid_elem(nv), 256, 0, s>>>(G.st.p, G.val.p, nv, q->lane, q->algo,
                                                                q->source); }
      if (fresh_cc)
        { ++n_launch; k_group_dense<GMAX><<<grid_elem(nv), 256, 0, s>>>(g, G.val.p, (uint32_t)fresh_cc, G.algo(),
                                                            gm[0].p, fview(0, cnt.p)); }
      for (Query *q : qs)
        if (q->algo != SGS_CC)
          { ++n_launch; k_group_seed_one<<<1, 32, 0, s>>>(g, q->source, 1u << q->lane, gm[0].p, fview(0, cnt.p)); }
    }
    CK(cudaGetLastError());
    bool conv = false;
    const uint32_t rounds = diropt ? run_bfs_diropt(G, (uint32_t)fresh, conv) : group_relax(G, conv);
    CK(cudaEventRecord(ev_q.b, s));
    sync();
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ev_q.a, ev_q.b));
    unsigned long long le[WLANES];
    CK(cudaMemcpyAsync(le, b_lane.p, sizeof(unsigned long long) * G.width, cudaMemcpyDeviceToHost, s));
    sync();
    for (Query *q : qs) {
      const int l = q->lane;
      q->stats.edges_traversed = le[l];
      q->stats.edges_total += le[l];
      q->stats.rounds = rounds;
      q->stats.converged = conv ? 1 : 0;
      q->stats.ms = ms;
      q->stats.invalidated = 0;
    }
    if (!conv) fail(SGS_ERR_NOCONV, "round limit reached before convergence");
  }

  int add_query(int algo, uint32_t source) {
    int id = 0;
    add_queries(1, &algo, &source, &id);
    return id;
  }

  // Registers n queries and brings them to their static fixed points; the
  // BFS/SSSP/CC ones fill free lanes of groups of cfg.group_size lanes
  // (narrow groups up to 4 lanes, wide groups above) and every group that
  // received lanes converges them in one pass.
  void add_queries(uint32_t n, const int *algos, const uint32_t *sources, int *ids) {
    if (!loaded) fail(SGS_ERR_STATE, "no graph loaded");
    for (uint32_t i = 0; i < n; ++i)
      if (algos[i] < 0 || algos[i] > 3) fail(SGS_ERR_INVALID, "unknown algorithm");
    const bool wide = cfg.group_size > (uint32_t)GMAX;
    const uint64_t full = cfg.group_size >= 64 ? ~0ull : (1ull << cfg.group_size) - 1ull;
    std::vector<Query *> added;
    std::vector<std::pair<Group *, uint64_t>> touched;
    for (uint32_t i = 0; i < n; ++i) {
      auto q = std::make_unique<Query>();
      q->id = next_qid++;
      q->algo = algos[i];
      q->source = std::min(sources[i], nv - 1);
      if (q->algo == SGS_PR) {
        q->x.ensure(nv);
        q->r.ensure(nv);
        q->pv.ensure(nv);
      } else {
        Group *G = nullptr;
        for (auto &gp : groups) {
          if (gp->wide() != wide || gp.get() == fg) continue;
          uint64_t pend = 0;
          for (auto &t : touched)
            if (t.first == gp.get()) pend = t.second;
          if (((gp->used | pend) & full) != full) { G = gp.get(); break; }
        }
        if (!G) {
          auto ng = std::make_unique<Group>();
          ng->width = wide ? WLANES : GMAX;
          for (int attempt = 0;; ++attempt) {
            try {
              ng->st.ensure((size_t)nv * ng->width);
              ng->val.ensure((size_t)nv * ng->width);
              break;
            } catch (const SgsError &f) {
              // out of memory: drop pooled empty groups (not pending here) once
              bool freed = false;
              if (f.code == SGS_ERR_OOM && attempt == 0)
                for (size_t j = groups.size(); j-- > 0;) {
                  bool pend = false;
                  for (auto &t : touched) pend |= t.first == groups[j].get();
                  if (groups[j]->used == 0 && !pend && !(groups[j].get() == fg && (frun || fsusp))) {
                    if (groups[j].get() == fg) fg = nullptr;
                    groups.erase(groups.begin() + j);
                    freed = true;
                  }
                }
              if (!freed) throw;
            }
          }
          G = ng.get();
          groups.push_back(std::move(ng));
        }
        uint64_t pend = 0;
        size_t ti = touched.size();
        for (size_t k = 0; k < touched.size(); ++k)
          if (touched[k].first == G) { pend = touched[k].second; ti = k; }
        if (ti == touched.size()) touched.push_back({G, 0});
        int l = 0;
        while ((G->used | pend) >> l & 1ull) ++l;
        G->set_lane(l, q->algo);
        touched[ti].second |= 1ull << l;
        q->grp = G;
        q->lane = l;
      }
      ids[i] = q->id;
      added.push_back(q.get());
      queries.push_back(std::move(q));
    }
    for (Query *q : added)
      if (q->algo == SGS_PR) start_pr(*q);
    for (auto &t : touched) {
      std::vector<Query *> qs;
      for (Query *q : added)
        if (q->grp == t.first) qs.push_back(q);
      start_lanes(*t.first, t.second, qs);
      t.first->used |= t.second;
    }
  }

  // ------------------------------------------------------------ serving
  Group &flight_group() {
    if (!fg) {
      auto ng = std::make_unique<Group>();
      ng->width = cfg.group_size > (uint32_t)GMAX ? WLANES : GMAX;
      ng->st.ensure((size_t)nv * ng->width);
      ng->val.ensure((size_t)nv * ng->width);
      if (ng->wide()) ensure_wide_masks();
      fg = ng.get();
      groups.push_back(std::move(ng));
    }
    flc.ensure(WLANES);
    return *fg;
  }
  uint32_t flight_lanes() const {
    const uint32_t w = cfg.group_size > (uint32_t)GMAX ? WLANES : GMAX;
    return std::min<uint32_t>(w, std::max<uint32_t>(cfg.group_size, 1));
  }
  uint32_t flight_free() {
    Group &G = flight_group();
    uint32_t f = 0;
    for (uint32_t l = 0; l < flight_lanes(); ++l) f += !(G.used >> l & 1ull);
    return f;
  }

  // Joins BFS/SSSP/CC queries to the flight: lanes initialised, sources (CC:
  // every vertex) seeded into the next round's frontier.
  void flight_admit(uint32_t n, const int *algos, const uint32_t *sources, int *ids) {
    if (!loaded) fail(SGS_ERR_STATE, "no graph loaded");
    Group &G = flight_group();
    for (uint32_t i = 0; i < n; ++i)
      if (algos[i] < 0 || algos[i] > 2) fail(SGS_ERR_INVALID, "flight lanes take BFS, SSSP or CC");
    if (n > flight_free()) fail(SGS_ERR_STATE, "no free lane in the flight");
    if (!frun) {  // a new flight: counters from round 0, masks are clean
      reset_counters(0);
      fr = 0;
    }
    uint64_t fresh = 0, cc = 0;
    std::vector<Query *> qs;
    for (uint32_t i = 0; i < n; ++i) {
      int l = 0;
      while (G.used >> l & 1ull) ++l;
      auto q = std::make_unique<Query>();
      q->id = next_qid++;
      q->algo = algos[i];
      q->source = std::min(sources[i], nv - 1);
      q->grp = &G;
      q->lane = l;
      G.set_lane(l, q->algo);
      G.used |= 1ull << l;
      fresh |= 1ull << l;
      if (q->algo == SGS_CC) cc |= 1ull << l;
      fadmit[l] = fr;
      ids[i] = q->id;
      qs.push_back(q.get());
      queries.push_back(std::move(q));
      CK(cudaMemsetAsync(b_lane.p + l, 0, sizeof(unsigned long long), s));
    }
    seed_flight_lanes(G, qs, fresh, cc);
    frun |= fresh;
  }

  // Lane state of the flight's queries `qs` (lanes `fresh`, the CC ones in
  // `cc`) initialised, and their sources (CC: every vertex) seeded into
  // frontier fr.
  void seed_flight_lanes(Group &G, const std::vector<Query *> &qs, uint64_t fresh, uint64_t cc) {
    GraphView g = view();
    const uint32_t b = fr % 3;
    if (G.wide()) {
      { ++n_launch; k_wide_init_lanes<<<grid_elem((uint64_t)nv * 32), 256, 0, s>>>(G.st.p, G.val.p, nv, fresh, G.cc); }
      if (cc)
        { ++n_launch; k_seed_all_or<unsigned long long><<<grid_elem(nv), RELAX_THREADS, 0, s>>>(
            g, (unsigned long long)cc, wm[b].p, fview(fr, cnt.p + fr)); }
      std::vector<uint32_t> src, lane;
      for (Query *q : qs)
        if (q->algo != SGS_CC) {
          src.push_back(q->source);
          lane.push_back((uint32_t)q->lane);
        }
      if (!src.empty()) {
        b_seed.ensure(2 * src.size());
        CK(cudaMemcpyAsync(b_seed.p, src.data(), sizeof(uint32_t) * src.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(b_seed.p + src.size(), lane.data(), sizeof(uint32_t) * lane.size(),
                           cudaMemcpyHostToDevice, s));
        { ++n_launch; k_wide_seed_sources<<<grid_elem(src.size()), 256, 0, s>>>(
            g, G.st.p, G.val.p, b_seed.p, b_seed.p + src.size(), (uint32_t)src.size(), wm[b].p,
            fview(fr, cnt.p + fr)); }
      }
    } else {
      for (Query *q : qs)
        { ++n_launch; k_group_init_lane<GMAX><<<grid_elem(nv), 256, 0, s>>>(G.st.p, G.val.p, nv, q->lane, q->algo,
                                                                q->source); }
      if (cc)
        { ++n_launch; k_seed_all_or<uint32_t><<<grid_elem(nv), RELAX_THREADS, 0, s>>>(
            g, (uint32_t)cc, gm[b].p, fview(fr, cnt.p + fr)); }
      for (Query *q : qs)
        if (q->algo != SGS_CC)
          { ++n_launch; k_group_seed_one<<<1, 32, 0, s>>>(g, q->source, 1u << q->lane, gm[b].p, fview(fr, cnt.p + fr)); }
    }
    CK(cudaGetLastError());
  }

  // An update preempts the flight (served loop): the lanes in flight stop at
  // this round boundary, their live frontiers (fr - 1 and fr) lose their
  // masks, and the lanes leave the group's used set, so the snapshot neither
  // invalidates nor repairs their partial state.  flight_resume restarts
  // them on the updated graph.
  void flight_suspend() {
    if (!frun || !fg) return;
    Group &G = *fg;
    if (fr >= 1) clear_masks(G.wide(), fr - 1);
    clear_masks(G.wide(), fr);
    CK(cudaGetLastError());
    G.used &= ~frun;
    fsusp = frun;
    frun = 0;
  }

  // Restarts the suspended lanes from their sources on the current graph as
  // a new flight (round 0, counters and per-lane edge counts cleared): their
  // results are those of the snapshot they restart on.
  void flight_resume() {
    if (!fsusp || !fg) {
      fsusp = 0;
      return;
    }
    Group &G = *fg;
    reset_counters(0);
    fr = 0;
    std::vector<Query *> qs;
    uint64_t cc = 0;
    for (auto &q : queries) {
      if (q->grp != &G || !(fsusp >> q->lane & 1ull)) continue;
      qs.push_back(q.get());
      if (q->algo == SGS_CC) cc |= 1ull << q->lane;
      fadmit[q->lane] = 0;
      CK(cudaMemsetAsync(b_lane.p + q->lane, 0, sizeof(unsigned long long), s));
    }
    G.used |= fsusp;
    const uint64_t lanes = fsusp;
    fsusp = 0;
    seed_flight_lanes(G, qs, lanes, cc);
    frun = lanes;
  }

  // Runs up to `rounds` relaxation rounds of the flight and returns the
  // queries whose lanes no longer appear in the frontier (their results are
  // final; they stay registered until removed).
  void flight_advance(uint32_t rounds, std::vector<int> &done) {
    done.clear();
    if (!frun || !fg) return;
    Group &G = *fg;
    const uint32_t maxr = cfg.max_rounds;
    rounds = std::max<uint32_t>(1, std::min<uint32_t>(rounds, 16));
    if (fr + rounds + 3 >= maxr) {
      // rebase the round index (same buffers: keep fr mod 3)
      const uint32_t nb = 3 + fr % 3;
      CK(cudaMemcpyAsync(cnt.p + nb - 1, cnt.p + fr - 1, 2 * sizeof(unsigned long long),
                         cudaMemcpyDeviceToDevice, s));
      CK(cudaMemsetAsync(cnt.p + nb + 1, 0, sizeof(unsigned long long) * (maxr + 1 - nb), s));
      fr = nb;
    }
    GraphView g = view();
    const bool anyw = G.sssp && cfg.weight_mode == SGS_W_EXPLICIT;
    for (uint32_t k = 0; k < rounds; ++k) {
      const uint32_t rr = fr + k;
      if (G.wide())
        launch_wide(rr, WideRelaxOp<>{G.st.p, G.val.p, G.walgo()}, nullptr);
      else
        launch_group(rr, GroupRelaxOp<GMAX>{g, G.st.p, G.val.p, gm[rr % 3].p, gm[(rr + 1) % 3].p,
                                            G.algo(), anyw});
    }
    const uint32_t nf = fr + rounds;  // the next input frontier
    CK(cudaMemsetAsync(flc.p, 0, sizeof(unsigned long long) * WLANES, s));
    if (G.wide())
      { ++n_launch; k_lane_counts<unsigned long long><<<grid_elem(nv), 256, 0, s>>>(
          fb[nf % 3].vtx.p, cnt.p + nf, wm[nf % 3].p, flc.p); }
    else
      { ++n_launch; k_lane_counts<uint32_t><<<grid_elem(nv), 256, 0, s>>>(fb[nf % 3].vtx.p, cnt.p + nf,
                                                                      gm[nf % 3].p, flc.p); }
    CK(cudaGetLastError());
    unsigned long long lc[WLANES], le[WLANES];
    CK(cudaMemcpyAsync(h_cnt, cnt.p + fr, sizeof(unsigned long long) * (rounds + 1),
                       cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(lc, flc.p, sizeof(lc), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(le, b_lane.p, sizeof(le), cudaMemcpyDeviceToHost, s));
    sync();
    uint32_t z = 0;  // first empty frontier of the batch, if any
    for (uint32_t k = 1; k <= rounds && !z; ++k)
      if ((h_cnt[k] >> CNT_SHIFT) == 0) z = fr + k;
    uint64_t fin = 0;
    if (z) {
      clear_masks(G.wide(), z - 1);
      fin = frun;
    } else {
      for (int l = 0; l < G.width; ++l)
        if ((frun >> l & 1ull) && lc[l] == 0) fin |= 1ull << l;
    }
    const uint32_t end = z ? z : nf;
    for (auto &q : queries) {
      if (q->grp != &G || !(fin >> q->lane & 1ull)) continue;
      q->stats.edges_traversed = le[q->lane];
      q->stats.edges_total += le[q->lane];
      q->stats.rounds = end - fadmit[q->lane];
      q->stats.converged = 1;
      q->stats.invalidated = 0;
      done.push_back(q->id);
    }
    frun &= ~fin;
    fr = end;
  }

  // ------------------------------------------------------------- autotune
  // Times a probe -- the static convergence of SSSP, BFS and CC from vertex
  // 0 in one group, device time from the engine's events -- for every pair
  // of (CTAs per SM of the relaxation map, launch mode) and keeps the
  // fastest.  Results do not depend on either choice.
  void autotune(sgs_tune *out) {
    if (!loaded) fail(SGS_ERR_STATE, "no graph loaded");
    static const uint32_t cps[] = {4, 8, 16, 32};
    const uint32_t keep_cps = map_cps, keep_pers = cfg.persistent;
    double best = 1e300;
    uint32_t bc = keep_cps, bp = keep_pers, tried = 0;
    const int algos[3] = {SGS_SSSP, SGS_BFS, SGS_CC};
    const uint32_t srcs[3] = {0, 0, 0};
    for (uint32_t pers = 0; pers < 2; ++pers)
      for (uint32_t c : cps) {
        map_cps = c;
        cfg.persistent = (keep_pers & ~1u) | pers;
        double t = 1e300;
        for (int rep = 0; rep < 2; ++rep) {  // the first run also warms up
          int ids[3];
          add_queries(3, algos, srcs, ids);
          t = std::min(t, find(ids[0]).stats.ms);
          for (int id : ids) remove_query(id);
        }
        ++tried;
        if (t < best) {
          best = t;
          bc = c;
          bp = pers;
        }
      }
    map_cps = bc;
    cfg.persistent = (keep_pers & ~1u) | bp;
    (void)keep_cps;
    (void)keep_pers;
    out->ctas_per_sm = bc;
    out->persistent = cfg.persistent;
    out->best_ms = best;
    out->tried = tried;
  }

  // Frees the state of groups without lanes in use; true if any was freed.
  bool release_empty_groups() {
    bool any = false;
    for (size_t j = groups.size(); j-- > 0;)
      if (groups[j]->used == 0) {
        if (groups[j].get() == fg) {
          if (frun || fsusp) continue;
          fg = nullptr;
        }
        groups.erase(groups.begin() + j);
        any = true;
      }
    return any;
  }

  void remove_query(int qid) {
    for (size_t i = 0; i < queries.size(); ++i)
      if (queries[i]->id == qid) {
        sync();
        Query &q = *queries[i];
        if (q.grp) q.grp->used &= ~(1ull << q.lane);
        if (job.q == &q) job.q = nullptr;
        if (q.algo == SGS_PR && cfg.pr_warm) {  // keep its vector for the next start
          std::swap(pr_warm.p, q.x.p);
          std::swap(pr_warm.n, q.x.n);
        }
        queries.erase(queries.begin() + i);
        // an empty group keeps its state arrays for the next queries (a
        // serving loop admits and retires queries all the time); they are
        // released when an allocation would fail (release_empty_groups)
        return;
      }
    fail(SGS_ERR_INVALID, "unknown query id");
  }

  // ------------------------------------------------------------ snapshots
  // Copies a batch into the next staging slot on the copy stream (from
  // pinned host or device memory) and returns at once; apply_staged applies
  // the oldest staged batch.  A slot is refilled only after the snapshot
  // that consumed it has copied it out.
  void stage_batch(const uint32_t *is, const uint32_t *id, const uint32_t *iw, uint64_t ni,
                   const uint32_t *ds, const uint32_t *dd, uint64_t nd, int mem) {
    if (stg_count >= 2) fail(SGS_ERR_STATE, "two batches are staged already");
    if (ni >= (1ull << 31) || nd >= (1ull << 31)) fail(SGS_ERR_INVALID, "batch too large");
    if ((ni && (!is || !id)) || (nd && (!ds || !dd))) fail(SGS_ERR_INVALID, "null batch array");
    const bool ew = cfg.weight_mode == SGS_W_EXPLICIT;
    if (ni && ew && !iw) fail(SGS_ERR_INVALID, "explicit weight mode needs insert weights");
    if (!sc) CK(cudaStreamCreateWithFlags(&sc, cudaStreamNonBlocking));
    Staged &t = stg[(stg_head + stg_count) % 2];
    if (!t.copied) {
      CK(cudaEventCreateWithFlags(&t.copied, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&t.consumed, cudaEventDisableTiming));
      CK(cudaEventRecord(t.consumed, s));
    }
    CK(cudaStreamWaitEvent(sc, t.consumed, 0));  // its previous batch was copied out
    const uint32_t *src[5] = {is, id, ew ? iw : nullptr, ds, dd};
    const uint64_t cnt[5] = {ni, ni, ew ? ni : 0, nd, nd};
    const cudaMemcpyKind kind = mem == SGS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    for (int k = 0; k < 5; ++k) {
      if (!cnt[k]) continue;
      t.a[k].ensure(cnt[k]);
      CK(cudaMemcpyAsync(t.a[k].p, src[k], cnt[k] * sizeof(uint32_t), kind, sc));
    }
    // the other slot grows with it (an allocation later, while copies and
    // snapshots are in flight, would stall the pipeline)
    Staged &o = stg[(stg_head + stg_count + 1) % 2];
    if (!o.copied) {
      CK(cudaEventCreateWithFlags(&o.copied, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&o.consumed, cudaEventDisableTiming));
      CK(cudaEventRecord(o.consumed, s));
    }
    for (int k = 0; k < 5; ++k)
      if (cnt[k] && o.a[k].n < cnt[k] && !o.full) o.a[k].ensure(cnt[k]);
    CK(cudaEventRecord(t.copied, sc));
    t.ni = ni;
    t.nd = nd;
    t.w = ew;
    t.full = true;
    ++stg_count;
  }
  void apply_staged() {
    if (!stg_count) fail(SGS_ERR_STATE, "no staged batch");
    Staged &t = stg[stg_head];
    CK(cudaStreamWaitEvent(s, t.copied, 0));
    stg_head = (stg_head + 1) % 2;
    --stg_count;
    t.full = false;
    staged_in = &t;
    try {
      apply_batch(t.a[0].p, t.a[1].p, t.w ? t.a[2].p : nullptr, t.ni, t.a[3].p, t.a[4].p, t.nd, SGS_MEM_DEVICE);
    } catch (...) {
      staged_in = nullptr;
      CK(cudaEventRecord(t.consumed, s));
      throw;
    }
    staged_in = nullptr;
  }
  Staged *staged_in = nullptr;  // the staged batch apply_batch is reading

  // Batch-sized buffers (and the sort's temporary storage) for batches of up
  // to ni inserts and nd deletes, at the capacities apply_batch grows them
  // to, so that a later batch of at most that size allocates nothing (a
  // growth frees and allocates, and a free waits for the whole device).
  void reserve_batch(uint64_t ni, uint64_t nd) {
    const size_t ci = batch_cap(ni), cd = batch_cap(nd), cm = batch_cap(std::max(ni, nd));
    for (DBuf<uint32_t> *b : {&b_isrc, &b_idst, &b_iw, &b_iw_s, &b_iw_kept, &t_iw}) b->ensure(ci);
    for (DBuf<uint32_t> *b : {&b_dsrc, &b_ddst}) b->ensure(cd);
    for (DBuf<uint64_t> *b : {&b_ikeys, &b_ikeys_s, &b_ikept, &t_ikeys}) b->ensure(ci);
    for (DBuf<uint64_t> *b : {&b_dkeys, &b_dkeys_s, &t_dkeys}) b->ensure(cd);
    t_tmp.ensure(cm);
    b_flag.ensure(ci);
    big_list.ensure(batch_cap(nd + 1));
    const size_t cr = batch_cap(ni + 1);
    rl_vtx.ensure(cr);
    rl_len.ensure(cr);
    rl_from.ensure(cr);
    rl_to.ensure(cr);
    // the sorts and the selection of apply_batch and of the in-edge store's
    // update, at the largest sizes
    const int eb = sort_bits();
    size_t tb = 0, t2 = 0, t3 = 0, t4 = 0;
    if (nd || ni)
      CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, b_dkeys.p, b_dkeys_s.p, (int)std::max(ni, nd), 0, eb, s));
    if (ni) {
      CK(cub::DeviceRadixSort::SortPairs(nullptr, t2, b_ikeys.p, b_ikeys_s.p, b_iw.p, b_iw_s.p, (int)ni, 0,
                                         eb, s));
      CK(cub::DeviceSelect::Flagged(nullptr, t3, b_ikeys_s.p, b_flag.p, b_ikept.p, b_nkept.p, (int)ni, s));
      CK(cub::DeviceRadixSort::SortPairs(nullptr, t4, t_tmp.p, t_ikeys.p, b_iw_kept.p, t_iw.p, (int)ni, 0,
                                         eb, s));
    }
    cub_ensure(std::max(std::max(tb, t2), std::max(t3, t4)));
  }

  // Tombstone reclamation of the blocks touched by this snapshot's nd
  // deletes (the frontier in buffer 0 / special(4)): small blocks a warp
  // each, the large ones listed by that pass a CTA each.
  void compact_blocks(const GraphView &gv, uint64_t nd, unsigned long long *reclaimed) {
    big_list.ensure(batch_cap(nd + 1));  // at most one entry per delete group
    big_n.ensure(1);
    CK(cudaMemsetAsync(big_n.p, 0, sizeof(uint32_t), s));
    { ++n_launch; k_compact_blocks<<<(uint32_t)nsm * 8, 256, 0, s>>>(gv, fview(0, special(4)), reclaimed,
                                                                     big_list.p, big_n.p); }
    { ++n_launch; k_compact_large<<<(uint32_t)nsm * 2, COMPACT_THREADS, 0, s>>>(gv, big_list.p, big_n.p,
                                                                               reclaimed); }
  }

  void upload(DBuf<uint32_t> &dst, const uint32_t *src, uint64_t n, int mem) {
    dst.ensure(batch_cap(n));
    if (n)
      CK(cudaMemcpyAsync(dst.p, src, n * sizeof(uint32_t),
                         mem == SGS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
  }

  // Repair of a narrow group by pull (cfg.repair bit 0): round 0 pulls over
  // the in-edges of the vertices the invalidation reset (GroupPullOp), the
  // kept inserted edges are relaxed into round 1's frontier, and the later
  // rounds push from the vertices that improved (one cooperative launch).
  // Returns the rounds run; fails on the round limit.
  uint32_t pull_repair(Group &G, bool had_deletes, uint64_t ni, bool explicit_w) {
    const GraphView g = view(), gi = in_view();
    const uint32_t anyw = G.any_sssp(G.used | 0xF) && cfg.weight_mode == SGS_W_EXPLICIT;
    CK(cudaMemsetAsync(rstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
    CK(cudaMemsetAsync(hstat.p, 0, sizeof(unsigned long long) * (cfg.max_rounds + 2), s));
    if (had_deletes)
      { ++n_launch; k_bits_frontier<<<grid_elem(nv), 256, 0, s>>>(G.ibits.p, gi, (uint32_t)G.used, gm[0].p,
                                                       fview(0, cnt.p)); }
    launch_group(0, GroupPullOp<GMAX>{gi, slots.p, G.st.p, G.val.p, gm[0].p, gm[1].p, G.algo(), cfg.weight_mode});
    if (ni)
      { ++n_launch; k_group_relax_inserted<GMAX><<<grid_elem(ni), 256, 0, s>>>(
          g, G.st.p, G.val.p, (uint32_t)G.used, G.algo(), b_ikept.p, explicit_w ? b_iw_kept.p : nullptr,
          b_nkept.p, gm[1].p, fview(1, cnt.p + 1), b_lane.p, nullptr); }
    CK(cudaGetLastError());
    // explicit host policy (-hybrid 1/2): the push rounds after round 0 read
    // the out-blocks, so they read an HBM copy of the host tier when the
    // policy asks for one (policy 2 judges by round 0's frontier)
    if (stage_wanted()) stage_host();
    const GraphView gs = view();
    bool conv = false;
    const uint32_t r = run_group_persistent(GroupRelaxOp<GMAX>{gs, G.st.p, G.val.p, nullptr, nullptr, G.algo(),
                                                               anyw},
                                            1, conv, SGS_K_GROUP, anyw ? 8.0 : 4.0);
    if (!conv) fail(SGS_ERR_NOCONV, "round limit reached before convergence");
    return r;
  }

  int sort_bits() const {
    int b = 1;
    while (b < 32 && (1ull << b) < nv) ++b;
    return 32 + b;
  }

  // The current layout as user algorithms see it (sgs_graph_view).
  sgs_graph_view graph_view() {
    const GraphView g = view();
    sgs_graph_view v{};
    v.nv = nv;
    v.weight_mode = cfg.weight_mode;
    v.ne = ne;
    v.slots_total = slots_total;
    v.off = g.off;
    v.slots = g.slots;
    v.live = g.live;
    v.cap = g.cap;
    v.adj_d = g.adj_d;
    v.wgt_d = g.wgt_d;
    v.adj_h = g.adj_h;
    v.wgt_h = g.wgt_h;
    v.cmap = g.cmap;
    v.adj_c = g.adj_c;
    v.wgt_c = g.wgt_c;
    v.cbase = g.cbase;
    v.stream = (void *)s;
    v.device = dev;
    return v;
  }
  // Runs every attached user algorithm's phase (before or after the graph
  // update) on the engine's stream, with the snapshot's sorted device keys.
  void run_app_hooks(bool after, uint64_t ni, uint64_t nd) {
    if (apps.empty()) return;
    const sgs_graph_view gv = graph_view();
    sgs_update_view u{};
    u.del_keys = nd ? b_dkeys_s.p : nullptr;
    u.n_del = nd;
    u.ins_keys = ni ? b_ikept.p : nullptr;
    u.ins_w = ni && cfg.weight_mode == SGS_W_EXPLICIT ? b_iw_kept.p : nullptr;
    u.n_ins = b_nkept.p;
    u.n_ins_max = ni;
    for (const AppHook &a : apps) {
      sgs_app_phase_fn f = after ? a.h.after_update : a.h.before_update;
      if (!f) continue;
      g_last_error.clear();
      const int rc = f(a.h.ctx, &gv, &u);
      if (rc != SGS_OK)
        fail(rc, g_last_error.empty() ? std::string("user algorithm phase failed") : g_last_error);
    }
  }

  void apply_batch(const uint32_t *is, const uint32_t *id, const uint32_t *iw, uint64_t ni,
                   const uint32_t *ds, const uint32_t *dd, uint64_t nd, int mem) {
    if (!loaded) fail(SGS_ERR_STATE, "no graph loaded");
    if (ni >= (1ull << 31) || nd >= (1ull << 31)) fail(SGS_ERR_INVALID, "batch too large");
    if ((ni && (!is || !id)) || (nd && (!ds || !dd))) fail(SGS_ERR_INVALID, "null batch array");
    const bool explicit_w = cfg.weight_mode == SGS_W_EXPLICIT;
    if (ni && explicit_w && !iw) fail(SGS_ERR_INVALID, "explicit weight mode needs insert weights");
    staged = false;  // the host arena itself is what the update writes
    GraphView g = view();
    Range snap("sgs:snapshot");
    CK(cudaEventRecord(ev_batch.a, s));
    // ---- upload + keys + sort
    upload(b_isrc, is, ni, mem);
    upload(b_idst, id, ni, mem);
    if (explicit_w) upload(b_iw, iw, ni, mem);
    upload(b_dsrc, ds, nd, mem);
    upload(b_ddst, dd, nd, mem);
    if (staged_in) CK(cudaEventRecord(staged_in->consumed, s));  // its slot may be refilled
    const size_t ci = batch_cap(ni), cd = batch_cap(nd);
    b_ikeys.ensure(ci); b_ikeys_s.ensure(ci); b_ikept.ensure(ci);
    b_iw_s.ensure(ci); b_iw_kept.ensure(ci); b_flag.ensure(ci);
    b_dkeys.ensure(cd); b_dkeys_s.ensure(cd);
    CK(cudaMemsetAsync(b_err.p, 0, sizeof(unsigned int), s));
    CK(cudaMemsetAsync(b_stat.p, 0, sizeof(unsigned long long) * 8, s));
    if (ni)
      { ++n_launch; k_make_keys<<<grid_elem(ni), 256, 0, s>>>(b_isrc.p, b_idst.p, ni, nv, b_ikeys.p,
                                                explicit_w ? b_iw.p : nullptr, explicit_w, b_err.p); }
    if (nd)
      { ++n_launch; k_make_keys<<<grid_elem(nd), 256, 0, s>>>(b_dsrc.p, b_ddst.p, nd, nv, b_dkeys.p, nullptr, 0,
                                                b_err.p); }
    const int eb = sort_bits();
    size_t tb = 0, t2 = 0, t3 = 0;
    if (nd) CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, b_dkeys.p, b_dkeys_s.p, (int)nd, 0, eb, s));
    if (ni) {
      CK(cub::DeviceRadixSort::SortPairs(nullptr, t2, b_ikeys.p, b_ikeys_s.p,
                                         explicit_w ? b_iw.p : b_isrc.p, b_iw_s.p, (int)ni, 0, eb, s));
      CK(cub::DeviceSelect::Flagged(nullptr, t3, b_ikeys_s.p, b_flag.p, b_ikept.p, b_nkept.p, (int)ni, s));
    }
    cub_ensure(std::max(tb, std::max(t2, t3)));
    if (nd) CK(cub::DeviceRadixSort::SortKeys(cub_tmp.p, tb, b_dkeys.p, b_dkeys_s.p, (int)nd, 0, eb, s));
    CK(cudaMemsetAsync(b_nkept.p, 0, sizeof(uint32_t), s));
    if (ni) {
      CK(cub::DeviceRadixSort::SortPairs(cub_tmp.p, t2, b_ikeys.p, b_ikeys_s.p,
                                         explicit_w ? b_iw.p : b_isrc.p, b_iw_s.p, (int)ni, 0, eb, s));
      { ++n_launch; k_filter_inserts<<<grid_elem(ni), 256, 0, s>>>(b_ikeys_s.p, (uint32_t)ni, b_dkeys_s.p,
                                                     (uint32_t)nd, b_flag.p); }
      CK(cub::DeviceSelect::Flagged(cub_tmp.p, t3, b_ikeys_s.p, b_flag.p, b_ikept.p, b_nkept.p,
                                    (int)ni, s));
      if (explicit_w)
        CK(cub::DeviceSelect::Flagged(cub_tmp.p, t3, b_iw_s.p, b_flag.p, b_iw_kept.p, b_nkept.p,
                                      (int)ni, s));
    }
    CK(cudaGetLastError());
    unsigned int herr = 0;
    CK(cudaMemcpyAsync(&herr, b_err.p, sizeof(herr), cudaMemcpyDeviceToHost, s));
    sync();
    if (herr & 1u) fail(SGS_ERR_INVALID, "batch vertex id out of range");
    if (herr & 2u) fail(SGS_ERR_INVALID, "insert weight 0 (weights must be >= 1)");

    bool any_pr = false;
    for (auto &q : queries) any_pr |= q->algo == SGS_PR;
    const size_t ng = groups.size();
    // per group: events around its invalidation [4i, 4i+1] and repair
    // [4i+2, 4i+3]; counters in G.dstat; all read after the last sync
    ensure_gev(4 * ng);
    std::vector<uint32_t> grounds(ng, 0);
    std::vector<char> gdel(ng, 0);
    for (size_t i = 0; i < ng; ++i) {
      Group &G = *groups[i];
      if (!G.used) continue;
      G.dstat.ensure(3 * WLANES);
      CK(cudaMemsetAsync(G.dstat.p, 0, sizeof(unsigned long long) * 3 * WLANES, s));
    }

    // pull repair of narrow groups (cfg.repair): the in-edge store is built
    // here if needed, before any frontier of this snapshot is seeded
    bool any_narrow = false;
    for (size_t i = 0; i < ng; ++i) any_narrow |= groups[i]->used && !groups[i]->wide();
    const bool prep = (cfg.repair & 1u) && any_narrow && nd && ensure_in();

    // ---- PR cancel over the old out-lists of touched sources
    if (any_pr) {
      build_touched(g, ni, nd);
      for (auto &qp : queries) {
        Query &q = *qp;
        if (q.algo != SGS_PR) continue;
        PrAmendOp op{g, q.x.p, q.r.p, -cfg.pr_alpha};
        { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fview(0, special(2)), fview(1, special(3)), op,
                                                     nullptr); }
      }
    }
    // ---- deletion phase: parent-tree invalidation on the old graph, all
    // lanes of a group together
    for (size_t i = 0; i < ng && nd; ++i) {
      Range rg("sgs:invalidate");
      Group &G = *groups[i];
      if (!G.used) continue;
      gdel[i] = 1;
      CK(cudaEventRecord(gev[4 * i], s));
      CK(cudaMemsetAsync(b_lane.p, 0, sizeof(unsigned long long) * WLANES, s));
      CK(cudaMemsetAsync(b_inval.p, 0, sizeof(unsigned long long) * WLANES, s));
      reset_counters(0);
      if (G.wide()) {  // the lanes this invalidation resets, per vertex
        G.wreset.ensure(nv);
        CK(cudaMemsetAsync(G.wreset.p, 0, sizeof(unsigned long long) * nv, s));
      } else if (prep) {  // bitmap of the vertices this invalidation resets
        const size_t nw = (size_t)nv / 32 + 1;
        G.ibits.ensure(nw);
        CK(cudaMemsetAsync(G.ibits.p, 0, sizeof(uint32_t) * nw, s));
      }
      uint32_t *nmark = prep ? G.ibits.p : nullptr;  // narrow groups mark only for the pull repair
      bool conv = false;
      if (G.wide()) {
        { ++n_launch; k_wide_seed_deleted<<<grid_elem(nd), 256, 0, s>>>(
            g, G.st.p, G.val.p, G.used, G.cc, b_dkeys_s.p, (uint32_t)nd, b_inval.p, G.wreset.p, wm[0].p,
            fview(0, cnt.p)); }
        CK(cudaGetLastError());
        WideInvalidateOp op{G.st.p, G.val.p, WideAlgo{0ull, G.cc}};  // no weights needed
        op.mark = G.wreset.p;
        if (cfg.persistent & 2u) run_wide_persistent(op, 0, conv, SGS_K_WIDE_INVAL, 4.0, b_inval.p);
        else run_wide_rounds(op, op, conv, SGS_K_WIDE_INVAL, 4.0, b_inval.p);
      } else {
        { ++n_launch; k_group_seed_deleted<GMAX><<<grid_elem(nd), 256, 0, s>>>(
            g, G.st.p, G.val.p, (uint32_t)G.used, G.algo(), b_dkeys_s.p, (uint32_t)nd, b_inval.p,
            nmark, gm[0].p, fview(0, cnt.p)); }
        CK(cudaGetLastError());
        if (cfg.persistent & 2u)
          run_group_persistent(GroupInvalidateOp<GMAX>{g, G.st.p, G.val.p, nullptr, nullptr, G.algo(),
                                                       b_inval.p, nmark},
                               0, conv, SGS_K_GROUP_INVAL, 4.0);
        else
          run_group_rounds(
              [&](uint32_t, uint32_t *mi, uint32_t *mo) {
                return GroupInvalidateOp<GMAX>{g, G.st.p, G.val.p, mi, mo, G.algo(), b_inval.p, nmark};
              },
              conv, SGS_K_GROUP_INVAL, 4.0);
      }
      if (!conv) fail(SGS_ERR_NOCONV, "invalidation did not converge");
      CK(cudaEventRecord(gev[4 * i + 1], s));
      CK(cudaMemcpyAsync(G.dstat.p, b_inval.p, sizeof(unsigned long long) * WLANES,
                         cudaMemcpyDeviceToDevice, s));
      CK(cudaMemcpyAsync(G.dstat.p + WLANES, b_lane.p, sizeof(unsigned long long) * WLANES,
                         cudaMemcpyDeviceToDevice, s));
    }

    // ---- user algorithms: their deletion phase on the old graph
    run_app_hooks(false, ni, nd);

    // ---- graph update
    CK(cudaEventRecord(ev_apply.a, s));
    {
      Range rg("sgs:apply_graph");
      apply_graph(ni, nd);
    }
    CK(cudaEventRecord(ev_apply.b, s));
    // ---- edge cache: admission from the hotness window; the copies run on
    // the side stream under the repair below
    cache_admit(/*rotate=*/true);
    g = view();

    // ---- PR compensate over the new out-lists, then convergence
    if (any_pr) {
      build_touched(g, ni, nd);
      for (auto &qp : queries) {
        Query &q = *qp;
        if (q.algo != SGS_PR) continue;
        PrAmendOp op{g, q.x.p, q.r.p, cfg.pr_alpha};
        { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fview(0, special(2)), fview(1, special(3)), op,
                                                     nullptr); }
      }
      for (auto &qp : queries) {
        Query &q = *qp;
        if (q.algo != SGS_PR) continue;
        if (&q == job.q) {  // a served PageRank job converges at its own pace
          job.stale = true;
          continue;
        }
        CK(cudaEventRecord(ev_q.a, s));
        CK(cudaMemsetAsync(b_stat.p + 4, 0, sizeof(unsigned long long), s));
        bool conv = false;
        double l1v = 0;
        const uint32_t rounds = pr_rounds(q, b_stat.p + 4, conv, l1v);
        CK(cudaEventRecord(ev_q.b, s));
        unsigned long long e = 0;
        CK(cudaMemcpyAsync(&e, b_stat.p + 4, sizeof(e), cudaMemcpyDeviceToHost, s));
        sync();
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev_q.a, ev_q.b));
        q.stats.edges_traversed = e;
        q.stats.edges_total += e;
        q.stats.rounds = rounds;
        q.stats.converged = conv;
        q.stats.ms = ms;
        q.stats.pr_residual_l1 = l1v;
        q.stats.invalidated = 0;
        if (!conv) fail(SGS_ERR_NOCONV, "round limit reached before convergence");
      }
    }
    // ---- add phase per group.  After an invalidation the reference re-pushes
    // from every reached vertex (SyncPushDDBAll), and so do narrow groups.
    // In a wide group that first round visits the same edges but relaxes
    // only those into vertices reset in this snapshot (bitmap G.ibits), and
    // the kept inserted edges are relaxed right after it: before the repair,
    // every other edge (u,v) already satisfies value(u) + w >= value(v) -- u
    // kept a value that was valid on the old graph, v kept its own, and the
    // edge existed -- so these two sets hold every violated edge.  Later
    // rounds are unrestricted, so the fixed point is the same.  (For a narrow
    // group the 16-B state row costs no more than the bitmap probe, so the
    // restriction does not pay.)  Without invalidation only the inserted
    // edges are relaxed.  Then rounds to convergence.
    for (size_t i = 0; i < ng; ++i) {
      Group &G = *groups[i];
      if (!G.used) continue;
      Range rg("sgs:repair");
      CK(cudaEventRecord(gev[4 * i + 2], s));
      CK(cudaMemsetAsync(b_lane.p, 0, sizeof(unsigned long long) * WLANES, s));
      reset_counters(0);
      if (G.wide() && !gdel[i]) {  // no deletion phase ran: no lane was reset
        G.wreset.ensure(nv);
        CK(cudaMemsetAsync(G.wreset.p, 0, sizeof(unsigned long long) * nv, s));
      }
      // the path is chosen on the device from the group's reset counts
      // (G.dstat[0, 64)): the dense frontier only if a lane was reset
      const unsigned long long *resets = G.dstat.p;
      if (!G.wide() && prep) {  // work-efficient repair: pull into the reset vertices
        bool conv = false;
        grounds[i] = pull_repair(G, gdel[i] != 0, ni, explicit_w);
        (void)conv;
        CK(cudaEventRecord(gev[4 * i + 3], s));
        CK(cudaMemcpyAsync(G.dstat.p + 2 * WLANES, b_lane.p, sizeof(unsigned long long) * WLANES,
                           cudaMemcpyDeviceToDevice, s));
        continue;
      }
      if (G.wide())
        { ++n_launch; k_wide_dense<<<grid_elem(nv), RELAX_THREADS, 0, s>>>(g, G.val.p, G.used, G.cc, wm[0].p,
                                                               fview(0, cnt.p), resets); }
      else
        { ++n_launch; k_group_dense<GMAX><<<grid_elem(nv), 256, 0, s>>>(g, G.val.p, (uint32_t)G.used, G.algo(),
                                                            gm[0].p, fview(0, cnt.p), resets); }
      if (ni && !G.wide())  // narrow, nothing reset: only the inserted edges
        { ++n_launch; k_group_relax_inserted<GMAX><<<grid_elem(ni), 256, 0, s>>>(
            g, G.st.p, G.val.p, (uint32_t)G.used, G.algo(), b_ikept.p, explicit_w ? b_iw_kept.p : nullptr,
            b_nkept.p, gm[0].p, fview(0, cnt.p), b_lane.p, resets); }
      CK(cudaGetLastError());
      if (stage_wanted()) stage_host();  // explicit host policy: repair reads an HBM copy
      // wide: the inserted edges after the restricted round 0, into its
      // output frontier (round 0 is empty when nothing was reset)
      const std::function<void()> ins_after0 = [&] {
        { ++n_launch; k_wide_relax_inserted<<<grid_elem(ni), 256, 0, s>>>(
            g, G.st.p, G.val.p, G.used, G.walgo(), b_ikept.p, explicit_w ? b_iw_kept.p : nullptr,
            b_nkept.p, wm[1].p, fview(1, cnt.p + 1), b_lane.p); }
      };
      bool conv = false;
      grounds[i] = G.wide() ? group_relax(G, conv, "sgs:sweep", G.wreset.p, ni ? &ins_after0 : nullptr)
                            : group_relax(G, conv, "sgs:sweep");
      if (!conv) fail(SGS_ERR_NOCONV, "round limit reached before convergence");
      CK(cudaEventRecord(gev[4 * i + 3], s));
      CK(cudaMemcpyAsync(G.dstat.p + 2 * WLANES, b_lane.p, sizeof(unsigned long long) * WLANES,
                         cudaMemcpyDeviceToDevice, s));
    }
    staged = false;  // back to the host arena (zero-copy) for everything else
    cache_publish();  // the snapshot ends when its line copies are visible
    // ---- user algorithms: repair and convergence on the new graph
    run_app_hooks(true, ni, nd);
    // per-lane counters of every group, one read
    h_gstat.resize(3 * WLANES * std::max<size_t>(ng, 1));
    for (size_t i = 0; i < ng; ++i)
      if (groups[i]->used)
        CK(cudaMemcpyAsync(h_gstat.data() + 3 * WLANES * i, groups[i]->dstat.p,
                           sizeof(unsigned long long) * 3 * WLANES, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(ev_batch.b, s));
    sync();
    for (size_t i = 0; i < ng; ++i) {
      Group &G = *groups[i];
      if (!G.used) continue;
      const unsigned long long *h = h_gstat.data() + 3 * WLANES * i;
      float ms = 0, m2 = 0;
      if (gdel[i]) CK(cudaEventElapsedTime(&ms, gev[4 * i], gev[4 * i + 1]));
      CK(cudaEventElapsedTime(&m2, gev[4 * i + 2], gev[4 * i + 3]));
      for (int q = 0; q < G.width; ++q) G.inval[q] = h[q];
      for (auto &qp : queries) {
        if (qp->grp != &G) continue;
        const int l = qp->lane;
        const uint64_t e = h[WLANES + l] + h[2 * WLANES + l];
        qp->stats.edges_traversed = e;
        qp->stats.edges_total += e;
        qp->stats.rounds = grounds[i];
        qp->stats.converged = 1;
        qp->stats.ms = ms + m2;
        qp->stats.pr_residual_l1 = 0;
        qp->stats.invalidated = h[l];
      }
    }
    float ams = 0, bms = 0;
    CK(cudaEventElapsedTime(&ams, ev_apply.a, ev_apply.b));
    CK(cudaEventElapsedTime(&bms, ev_batch.a, ev_batch.b));
    est.last_apply_ms = ams;
    est.last_batch_ms = bms;
    uint64_t edges = 0;
    for (auto &q : queries) edges += q->stats.edges_traversed;
    est.last_batch_edges = edges;
  }

  // Union of the distinct sources of the sorted deletes and kept inserts, with
  // their current block sizes, as a frontier in buffer 0 / special(2).
  void build_touched(const GraphView &g, uint64_t ni, uint64_t nd) {
    if (estamp >= 0xFFFFFFF0u) {
      CK(cudaMemsetAsync(emark.p, 0, sizeof(uint32_t) * nv, s));
      estamp = 1;
    }
    const uint32_t st = ++estamp;
    CK(cudaMemsetAsync(special(2), 0, sizeof(unsigned long long), s));
    if (nd)
      { ++n_launch; k_group_heads<<<grid_elem(nd), 256, 0, s>>>(g, b_dkeys_s.p, nullptr, (uint32_t)nd, nullptr,
                                                  emark.p, st, fview(0, special(2))); }
    if (ni)
      { ++n_launch; k_group_heads<<<grid_elem(ni), 256, 0, s>>>(g, b_ikept.p, b_nkept.p, 0, nullptr, emark.p, st,
                                                  fview(0, special(2))); }
    CK(cudaGetLastError());
  }

  // Deletes become tombstones; kept inserts are appended in place or their
  // block is relocated (capacity x1.5) within its tier; the arena is repacked
  // first when the relocations would not fit.
  void apply_graph(uint64_t ni, uint64_t nd) {
    cache_publish();  // no line copy may run while blocks are written (through)
    GraphView g = view();
    unsigned long long *tombs = b_stat.p + 2;
    CK(cudaMemsetAsync(tombs, 0, sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(b_reclaim.p, 0, sizeof(unsigned long long) * 2, s));
    if (nd) {
      CK(cudaMemsetAsync(special(4), 0, sizeof(unsigned long long), s));
      b_gstart.ensure((size_t)nv + 1);
      { ++n_launch; k_group_heads<<<grid_elem(nd), 256, 0, s>>>(g, b_dkeys_s.p, nullptr, (uint32_t)nd, b_gstart.p,
                                                  nullptr, 0, fview(0, special(4))); }
      TombOp op{g, b_dkeys_s.p, b_gstart.p, (uint32_t)nd};
      { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fview(0, special(4)), fview(1, special(5)), op,
                                                   tombs); }
      // the touched blocks that now hold a sixteenth or more of dead slots are
      // compacted in place before the inserts append to them
      compact_blocks(g, nd, b_reclaim.p);
      CK(cudaGetLastError());
    }
    uint32_t nkept = 0;
    uint64_t nreloc = 0;
    if (ni) {
      wbase.ensure(nv);
      InsertCtx c{};
      c.arena_top = arena_top.p;
      c.arena_cap[0] = arena_cap[0];
      c.arena_cap[1] = arena_cap[1];
      c.err = b_err.p;
      c.wbase = wbase.p;
      // dry run: relocation demand per tier
      CK(cudaMemsetAsync(b_stat.p, 0, sizeof(unsigned long long) * 2, s));
      { ++n_launch; k_insert_plan<<<grid_elem(ni), 256, 0, s>>>(g, b_ikept.p, b_nkept.p, c, 1, b_stat.p); }
      unsigned long long h[2], tops[2];
      CK(cudaMemcpyAsync(h, b_stat.p, sizeof(h), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(tops, arena_top.p, sizeof(tops), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(&nkept, b_nkept.p, sizeof(nkept), cudaMemcpyDeviceToHost, s));
      sync();
      if (tops[0] + h[0] > arena_cap[0] || tops[1] + h[1] > arena_cap[1]) {
        repack(h[0] + h[1] + 4096);
        g = view();
        c.arena_cap[0] = arena_cap[0];
        c.arena_cap[1] = arena_cap[1];
      }
      rl_vtx.ensure(batch_cap(nkept + 1));
      rl_len.ensure(batch_cap(nkept + 1));
      rl_from.ensure(batch_cap(nkept + 1));
      rl_to.ensure(batch_cap(nkept + 1));
      c.rl_vtx = rl_vtx.p;
      c.rl_from = rl_from.p;
      c.rl_to = rl_to.p;
      c.rl_len = rl_len.p;
      c.rl_count64 = rl_count.p;
      CK(cudaMemsetAsync(rl_count.p, 0, sizeof(unsigned long long), s));
      CK(cudaMemsetAsync(b_err.p, 0, sizeof(unsigned int), s));
      { ++n_launch; k_insert_plan<<<grid_elem(ni), 256, 0, s>>>(g, b_ikept.p, b_nkept.p, c, 0, nullptr); }
      { ++n_launch; k_insert_write<<<grid_elem(ni), 256, 0, s>>>(
          g, b_ikept.p, cfg.weight_mode == SGS_W_EXPLICIT ? b_iw_kept.p : nullptr, b_nkept.p, wbase.p); }
      CK(cudaMemsetAsync(special(6), 0, sizeof(unsigned long long), s));
      { ++n_launch; k_reloc_frontier<<<grid_elem(nkept), 256, 0, s>>>(rl_count.p, rl_len.p, fview(0, special(6))); }
      RelocCopyOp op{g, rl_from.p, rl_to.p};
      { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fview(0, special(6)), fview(1, special(7)), op,
                                                   nullptr); }
      CK(cudaGetLastError());
      unsigned int herr = 0;
      unsigned long long hrl = 0;
      CK(cudaMemcpyAsync(&herr, b_err.p, sizeof(herr), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(&hrl, rl_count.p, sizeof(hrl), cudaMemcpyDeviceToHost, s));
      sync();
      if (herr) fail(SGS_ERR_OOM, "edge arena exhausted while inserting");
      nreloc = hrl;
    }
    unsigned long long ht = 0, hrc = 0;
    CK(cudaMemcpyAsync(&ht, tombs, sizeof(ht), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&hrc, b_reclaim.p, sizeof(hrc), cudaMemcpyDeviceToHost, s));
    sync();
    in_apply(ni, nd, nkept);
    ne = ne + nkept - ht;
    slots_total = slots_total + nkept - hrc;
    reclaimed_total += hrc;
    est.last_inserted = nkept;
    est.last_deleted = ht;
    est.last_relocated = nreloc;
  }

  // --------------------------------------------------------------- output
  void gather(Query &q, int field, void *out, int mem) {
    const cudaMemcpyKind kind = mem == SGS_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (q.algo == SGS_PR) {
      if (field == SGS_FIELD_PARENT) fail(SGS_ERR_INVALID, "PageRank has no parent field");
      if (field != SGS_FIELD_VALUE && field != SGS_FIELD_BUFFER) fail(SGS_ERR_INVALID, "unknown field");
      const double *src = field == SGS_FIELD_VALUE ? q.x.p : q.r.p;
      CK(cudaMemcpyAsync(out, src, sizeof(double) * nv, kind, s));
      sync();
      return;
    }
    DBuf<uint32_t> tmp;
    tmp.ensure(nv);
    if (field != SGS_FIELD_PARENT && field != SGS_FIELD_VALUE && field != SGS_FIELD_BUFFER)
      fail(SGS_ERR_INVALID, "unknown field");
    uint32_t *vo = field == SGS_FIELD_PARENT ? nullptr : tmp.p;
    uint32_t *po = field == SGS_FIELD_PARENT ? tmp.p : nullptr;
    if (q.grp->wide())
      { ++n_launch; k_group_split<WLANES><<<grid_elem(nv), 256, 0, s>>>(q.grp->st.p, nv, q.lane, vo, po); }
    else
      { ++n_launch; k_group_split<GMAX><<<grid_elem(nv), 256, 0, s>>>(q.grp->st.p, nv, q.lane, vo, po); }
    CK(cudaMemcpyAsync(out, tmp.p, sizeof(uint32_t) * nv, kind, s));
    sync();
  }

  void summary(Query &q, uint64_t out[4]) {
    CK(cudaMemsetAsync(b_stat.p, 0, sizeof(unsigned long long) * 4, s));
    if (q.algo == SGS_PR) {
      { ++n_launch; k_summary_pr<<<grid_elem(nv), RELAX_THREADS, 0, s>>>(q.x.p, nv, (double *)b_stat.p + 1); }
    } else {
      if (q.grp->wide())
        { ++n_launch; k_group_summary<WLANES><<<grid_elem(nv), RELAX_THREADS, 0, s>>>(q.grp->st.p, nv, q.lane,
                                                                          b_stat.p); }
      else
        { ++n_launch; k_group_summary<GMAX><<<grid_elem(nv), RELAX_THREADS, 0, s>>>(q.grp->st.p, nv, q.lane,
                                                                        b_stat.p); }
    }
    CK(cudaGetLastError());
    unsigned long long h[4];
    CK(cudaMemcpyAsync(h, b_stat.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    sync();
    if (q.algo == SGS_PR) h[0] = nv;
    for (int i = 0; i < 4; ++i) out[i] = h[i];
  }

  // Summaries of several queries with one read-back: a narrow group's lanes
  // in one pass over its state rows, the others as in summary().
  DBuf<unsigned long long> b_sum;
  void summaries(uint32_t n, const int *qids, uint64_t *out) {
    b_sum.ensure(4ull * std::max<uint32_t>(n, 1));
    CK(cudaMemsetAsync(b_sum.p, 0, sizeof(unsigned long long) * 4 * n, s));
    std::vector<Query *> qs(n);
    for (uint32_t i = 0; i < n; ++i) qs[i] = &find(qids[i]);
    std::vector<char> done(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
      if (done[i]) continue;
      Query &q = *qs[i];
      if (q.algo == SGS_PR) {
        { ++n_launch; k_summary_pr<<<grid_elem(nv), RELAX_THREADS, 0, s>>>(q.x.p, nv,
                                                             (double *)(b_sum.p + 4 * i) + 1); }
      } else if (q.grp->wide()) {
        WideSlots ws;
        for (int l = 0; l < WLANES; ++l) ws.slot[l] = -1;
        for (uint32_t j = i; j < n; ++j)  // every requested lane of this group
          if (!done[j] && qs[j]->algo != SGS_PR && qs[j]->grp == q.grp && ws.slot[qs[j]->lane] < 0) {
            ws.slot[qs[j]->lane] = (int)j;
            done[j] = 1;
          }
        { ++n_launch; k_wide_summary_lanes<<<grid_elem((uint64_t)nv * 32), RELAX_THREADS, 0, s>>>(
            q.grp->st.p, nv, ws, b_sum.p); }
      } else {
        LaneSlots ls;
        for (int l = 0; l < GMAX; ++l) ls.slot[l] = -1;
        for (uint32_t j = i; j < n; ++j)  // every requested lane of this group
          if (!done[j] && qs[j]->algo != SGS_PR && qs[j]->grp == q.grp && ls.slot[qs[j]->lane] < 0) {
            ls.slot[qs[j]->lane] = (int)j;
            done[j] = 1;
          }
        { ++n_launch; k_group_summary_lanes<<<grid_elem(nv), RELAX_THREADS, 0, s>>>(q.grp->st.p, nv, ls,
                                                                       b_sum.p); }
      }
      done[i] = 1;
    }
    CK(cudaGetLastError());
    std::vector<unsigned long long> h(4ull * n);
    if (n) CK(cudaMemcpyAsync(h.data(), b_sum.p, sizeof(unsigned long long) * 4 * n, cudaMemcpyDeviceToHost, s));
    sync();
    for (uint32_t i = 0; i < n; ++i) {
      uint32_t src = i;
      for (uint32_t j = 0; j < i; ++j)
        if (qids[j] == qids[i]) src = j;  // repeated id: same counters
      for (int k = 0; k < 4; ++k) out[4 * i + k] = h[4 * src + k];
      if (qs[i]->algo == SGS_PR) out[4 * i] = nv;
    }
  }

  void export_graph(uint64_t *row, uint32_t *col, uint32_t *w, int mem) {
    DBuf<uint64_t> drow;
    drow.ensure((size_t)nv + 1);
    { ++n_launch; k_u32_to_u64<<<grid_elem(nv), 256, 0, s>>>(live.p, nv, drow.p); }
    CK(cudaMemsetAsync(drow.p + nv, 0, sizeof(uint64_t), s));
    size_t tb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, drow.p, drow.p, (int)(nv + 1), s));
    cub_ensure(tb);
    CK(cub::DeviceScan::ExclusiveSum(cub_tmp.p, tb, drow.p, drow.p, (int)(nv + 1), s));
    DBuf<uint32_t> dcol, dw, fill;
    dcol.ensure(ne + 1);
    if (w) dw.ensure(ne + 1);
    fill.ensure(nv);
    CK(cudaMemsetAsync(fill.p, 0, sizeof(uint32_t) * nv, s));
    reset_counters(0);
    { ++n_launch; k_dense_frontier<<<grid_elem(nv), 256, 0, s>>>(view(), fview(0, special(0))); }
    ExportOp op{view(), drow.p, dcol.p, w ? dw.p : nullptr, fill.p};
    { ++n_launch; seg_map<<<grid_map(), RELAX_THREADS, 0, s>>>(fview(0, special(0)), fview(1, special(1)), op,
                                                 nullptr); }
    CK(cudaGetLastError());
    const cudaMemcpyKind kind = mem == SGS_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    CK(cudaMemcpyAsync(row, drow.p, sizeof(uint64_t) * (nv + 1), kind, s));
    if (ne) CK(cudaMemcpyAsync(col, dcol.p, sizeof(uint32_t) * ne, kind, s));
    if (w && ne) CK(cudaMemcpyAsync(w, dw.p, sizeof(uint32_t) * ne, kind, s));
    sync();
  }

  // ------------------------------------------------------------- generator
  void load_rmat(uint32_t scale, uint32_t ef, uint64_t seed, double a, double b, double c,
                 uint64_t wseed) {
    if (scale < 1 || scale > 26) fail(SGS_ERR_INVALID, "scale must be in [1,26]");
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1) fail(SGS_ERR_INVALID, "bad R-MAT probabilities");
    const uint32_t n = 1u << scale;
    const uint64_t m = (uint64_t)n * ef;
    if (m >= (1ull << 31)) fail(SGS_ERR_INVALID, "too many edges for the generator");
    const double S = (double)(1ull << 53);
    const uint64_t tA = (uint64_t)(a * S), tAB = (uint64_t)((a + b) * S),
                   tABC = (uint64_t)((a + b + c) * S);
    const uint64_t key = fin64_host(seed ^ 0x524D4154ull);
    DBuf<uint64_t> k1, k2;
    k1.ensure(m);
    k2.ensure(m);
    { ++n_launch; k_rmat<<<grid_elem(m), 256, 0, s>>>(scale, m, key, tA, tAB, tABC, 1, k1.p); }
    size_t tb = 0, tu = 0;
    DBuf<uint32_t> nsel;
    nsel.ensure(1);
    CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, k1.p, k2.p, (int)m, 0, 64, s));
    CK(cub::DeviceSelect::Unique(nullptr, tu, k2.p, k1.p, nsel.p, (int)m, s));
    cub_ensure(std::max(tb, tu));
    CK(cub::DeviceRadixSort::SortKeys(cub_tmp.p, tb, k1.p, k2.p, (int)m, 0, 64, s));
    CK(cub::DeviceSelect::Unique(cub_tmp.p, tu, k2.p, k1.p, nsel.p, (int)m, s));
    uint32_t hn = 0;
    CK(cudaMemcpyAsync(&hn, nsel.p, sizeof(hn), cudaMemcpyDeviceToHost, s));
    sync();
    // the self-loop marker ~0 sorts last
    uint64_t lastk = 0;
    if (hn) CK(cudaMemcpyAsync(&lastk, k1.p + hn - 1, sizeof(lastk), cudaMemcpyDeviceToHost, s));
    sync();
    if (hn && lastk == ~0ull) --hn;
    CK(cudaMemcpyAsync(nsel.p, &hn, sizeof(hn), cudaMemcpyHostToDevice, s));
    k2.release();
    DBuf<uint64_t> row;
    DBuf<uint32_t> col, w;
    row.ensure((size_t)n + 1);
    col.ensure(hn + 1);
    { ++n_launch; k_row_from_sorted<<<grid_elem(n + 1), 256, 0, s>>>(k1.p, nsel.p, n, row.p); }
    { ++n_launch; k_keys_low<<<grid_elem(hn), 256, 0, s>>>(k1.p, nsel.p, col.p); }
    if (cfg.weight_mode == SGS_W_EXPLICIT) {
      w.ensure(hn + 1);
      const uint64_t wkey = fin64_host(wseed ^ 0x57454947ull);
      { ++n_launch; k_hash_weights<<<grid_elem(hn), 256, 0, s>>>(k1.p, nsel.p, wkey, w.p); }
    }
    CK(cudaGetLastError());
    k1.release();
    load_device_csr(n, row.p, col.p, cfg.weight_mode == SGS_W_EXPLICIT ? w.p : nullptr);
  }

  static uint64_t fin64_host(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
};

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
template <class F>
static int guarded(F &&f) {
  try {
    f();
    return SGS_OK;
  } catch (const SgsError &e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    g_last_error = "host allocation failed";
    return SGS_ERR_OOM;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return SGS_ERR_CUDA;
  }
}

extern "C" {

SGS_API const char *sgs_version(void) { return "sgs-b200 0.1"; }
SGS_API const char *sgs_last_error(void) { return g_last_error.c_str(); }

SGS_API void sgs_config_default(sgs_config *c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->device = 0;
  c->segments = 512;
  c->n_stream = 3;
  c->block_size = 512;
  c->cache_gb = 0;
  c->hbm_budget_gb = 0;
  c->weight_mode = SGS_W_EXPLICIT;
  c->max_rounds = 1000;
  c->pr_alpha = 0.85;
  c->pr_tol = 1e-6 * 0.15;
  c->slack_div = 8;
  c->arena_headroom = 0.30;
  c->group_size = 4;
  c->persistent = 14;  // invalidation phases persistent (many small rounds); relaxation: round 0
                      // (the snapshot's sweep) on the large grid, the rest persistent; PageRank
                      // pull rounds in one launch
  c->pull = 1;  // PageRank sweeps as pulls; bit 1 (direction-optimizing BFS) is opt-in
  c->host_policy = 0;  // zero-copy reads of the host tier
  c->pr_warm = 1;
  c->repair = 0;  // the reference's re-push from every reached vertex
  c->serve_restarts = 2;  // served loop: an update may restart a lane query twice
}

SGS_API int sgs_create(const sgs_config *cfg, sgs_engine **out) {
  if (!out) { g_last_error = "null out"; return SGS_ERR_INVALID; }
  *out = nullptr;
  return guarded([&] {
    sgs_config c;
    if (cfg) c = *cfg;
    else sgs_config_default(&c);
    auto e = std::make_unique<sgs_engine>();
    e->init(c);
    *out = e.release();
  });
}

SGS_API int sgs_destroy(sgs_engine *e) {
  if (!e) return SGS_OK;
  return guarded([&] {
    cudaSetDevice(e->dev);
    cudaStreamSynchronize(e->s);
    delete e;
  });
}

SGS_API int sgs_load_csr(sgs_engine *e, uint32_t nv, const uint64_t *row, const uint32_t *col,
                         const uint32_t *w, int mem) {
  if (!e || !row) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    if (mem == SGS_MEM_DEVICE) {
      e->load_device_csr(nv, row, col, w);
      return;
    }
    const uint64_t ne = row[nv];
    for (uint32_t v = 0; v < nv; ++v)
      if (row[v + 1] < row[v]) fail(SGS_ERR_INVALID, "row offsets must be non-decreasing");
    if (row[0] != 0) fail(SGS_ERR_INVALID, "row[0] must be 0");
    for (uint64_t i = 0; i < ne; ++i)
      if (col[i] >= nv) fail(SGS_ERR_INVALID, "edge destination out of range");
    const bool ew = e->cfg.weight_mode == SGS_W_EXPLICIT;
    if (ew && ne && !w) fail(SGS_ERR_INVALID, "explicit weight mode needs weights");
    if (ew)
      for (uint64_t i = 0; i < ne; ++i)
        if (w[i] == 0) fail(SGS_ERR_INVALID, "edge weight 0 (weights must be >= 1)");
    DBuf<uint64_t> drow;
    DBuf<uint32_t> dcol, dw;
    drow.ensure((size_t)nv + 1);
    dcol.ensure(ne + 1);
    CK(cudaMemcpyAsync(drow.p, row, sizeof(uint64_t) * (nv + 1), cudaMemcpyHostToDevice, e->s));
    if (ne) CK(cudaMemcpyAsync(dcol.p, col, sizeof(uint32_t) * ne, cudaMemcpyHostToDevice, e->s));
    if (ew) {
      dw.ensure(ne + 1);
      if (ne) CK(cudaMemcpyAsync(dw.p, w, sizeof(uint32_t) * ne, cudaMemcpyHostToDevice, e->s));
    }
    e->load_device_csr(nv, drow.p, dcol.p, ew ? dw.p : nullptr);
  });
}

SGS_API int sgs_load_edge_list(sgs_engine *e, uint32_t nv, uint64_t ne, const uint32_t *src,
                               const uint32_t *dst, const uint32_t *w, int mem) {
  if (!e || (ne && (!src || !dst))) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    std::vector<uint32_t> hs, hd, hw;
    const uint32_t *S = src, *D = dst, *W = w;
    if (mem == SGS_MEM_DEVICE) {
      hs.resize(ne); hd.resize(ne);
      if (ne) {
        CK(cudaMemcpy(hs.data(), src, ne * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hd.data(), dst, ne * 4, cudaMemcpyDeviceToHost));
      }
      S = hs.data(); D = hd.data();
      if (w) {
        hw.resize(ne);
        if (ne) CK(cudaMemcpy(hw.data(), w, ne * 4, cudaMemcpyDeviceToHost));
        W = hw.data();
      }
    }
    uint64_t mx = 0;
    for (uint64_t i = 0; i < ne; ++i) mx = std::max<uint64_t>(mx, std::max(S[i], D[i]));
    uint64_t n = nv ? nv : (ne ? mx + 1 : 0);
    if (n == 0 || n > 0xFFFFFFFFull) fail(SGS_ERR_INVALID, "bad vertex count");
    if (ne && mx >= n) fail(SGS_ERR_INVALID, "edge endpoint out of range");
    // counting sort by source, stable (file order within a source)
    std::vector<uint64_t> row(n + 1, 0);
    for (uint64_t i = 0; i < ne; ++i) row[S[i] + 1]++;
    for (uint64_t v = 0; v < n; ++v) row[v + 1] += row[v];
    std::vector<uint64_t> fill(row.begin(), row.end() - 1);
    std::vector<uint32_t> col(ne), ww(W ? ne : 0);
    for (uint64_t i = 0; i < ne; ++i) {
      const uint64_t p = fill[S[i]]++;
      col[p] = D[i];
      if (W) ww[p] = W[i];
    }
    // weights: explicit mode without weights falls back to the reference's
    // synthesized (u+v)%128+1 so that market_big files without weights load
    if (e->cfg.weight_mode == SGS_W_EXPLICIT && !W) {
      ww.resize(ne);
      for (uint32_t u = 0; u < n; ++u)
        for (uint64_t p = row[u]; p < row[u + 1]; ++p) ww[p] = (u + col[p]) % 128u + 1u;
    }
    const int rc = sgs_load_csr(e, (uint32_t)n, row.data(), col.data(),
                                ww.empty() ? nullptr : ww.data(), SGS_MEM_HOST);
    if (rc != SGS_OK) fail(rc, g_last_error);
  });
}

SGS_API int sgs_load_rmat(sgs_engine *e, uint32_t scale, uint32_t edge_factor, uint64_t seed,
                          double a, double b, double c, uint64_t wseed) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->load_rmat(scale, edge_factor, seed, a, b, c, wseed);
  });
}

SGS_API int sgs_query_add(sgs_engine *e, int algo, uint32_t source, int *qid) {
  if (!e || !qid) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    *qid = e->add_query(algo, source);
    if (!e->find(*qid).stats.converged) fail(SGS_ERR_NOCONV, "round limit reached before convergence");
  });
}

SGS_API int sgs_query_add_many(sgs_engine *e, uint32_t n, const int *algos, const uint32_t *sources,
                               int *qids) {
  if (!e || (n && (!algos || !sources || !qids))) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    if (n == 0) return;
    e->add_queries(n, algos, sources, qids);
    for (uint32_t i = 0; i < n; ++i)
      if (!e->find(qids[i]).stats.converged) fail(SGS_ERR_NOCONV, "round limit reached before convergence");
  });
}

}  // extern "C"

// Flight interface used by the served loop (serve.cpp); not exported.
namespace sgs {
int flight_free(sgs_engine *e, uint32_t *lanes) {
  return guarded([&] { *lanes = e->flight_free(); });
}
int flight_admit(sgs_engine *e, uint32_t n, const int *algos, const uint32_t *sources, int *ids) {
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->flight_admit(n, algos, sources, ids);
  });
}
int flight_advance(sgs_engine *e, uint32_t rounds, std::vector<int> &done, uint64_t *running) {
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->flight_advance(rounds, done);
    *running = e->frun;
  });
}
int flight_suspend(sgs_engine *e) {
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->flight_suspend();
  });
}
int flight_resume(sgs_engine *e) {
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->flight_resume();
  });
}
uint32_t serve_restarts(sgs_engine *e) { return e->cfg.serve_restarts; }
int reserve_batch(sgs_engine *e, uint64_t ni, uint64_t nd) {
  return guarded([&] {
    if (!e->loaded) fail(SGS_ERR_STATE, "no graph loaded");
    CK(cudaSetDevice(e->dev));
    e->reserve_batch(ni, nd);
  });
}
int pr_job_start(sgs_engine *e, int *qid) {
  return guarded([&] {
    if (!e->loaded) fail(SGS_ERR_STATE, "no graph loaded");
    CK(cudaSetDevice(e->dev));
    *qid = e->pr_job_start();
  });
}
int pr_job_advance(sgs_engine *e, uint32_t rounds, int *done) {
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    *done = e->pr_job_advance(rounds) ? 1 : 0;
  });
}
}  // namespace sgs

extern "C" {

SGS_API int sgs_query_remove(sgs_engine *e, int qid) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  return guarded([&] { e->remove_query(qid); });
}

SGS_API int sgs_apply_batch(sgs_engine *e, const uint32_t *ins_src, const uint32_t *ins_dst,
                            const uint32_t *ins_w, uint64_t n_ins, const uint32_t *del_src,
                            const uint32_t *del_dst, uint64_t n_del, int mem) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->apply_batch(ins_src, ins_dst, ins_w, n_ins, del_src, del_dst, n_del, mem);
  });
}

SGS_API int sgs_stage_batch(sgs_engine *e, const uint32_t *ins_src, const uint32_t *ins_dst,
                            const uint32_t *ins_w, uint64_t n_ins, const uint32_t *del_src,
                            const uint32_t *del_dst, uint64_t n_del, int mem) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  return guarded([&] {
    if (!e->loaded) fail(SGS_ERR_STATE, "no graph loaded");
    CK(cudaSetDevice(e->dev));
    e->stage_batch(ins_src, ins_dst, ins_w, n_ins, del_src, del_dst, n_del, mem);
  });
}

SGS_API int sgs_apply_staged(sgs_engine *e) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->apply_staged();
  });
}

SGS_API int sgs_gather(sgs_engine *e, int qid, int field, void *out, int mem) {
  if (!e || !out) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->gather(e->find(qid), field, out, mem);
  });
}

SGS_API int sgs_get_query_stats(sgs_engine *e, int qid, sgs_query_stats *out) {
  if (!e || !out) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] { *out = e->find(qid).stats; });
}

SGS_API int sgs_get_engine_stats(sgs_engine *e, sgs_engine_stats *out) {
  if (!e || !out) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    e->est.nv = e->nv;
    e->est.ne = e->ne;
    e->est.repacks = e->repacks;
    e->est.kernel_launches = e->n_launch;
    unsigned long long tops[2] = {0, 0};
    if (e->loaded) {
      CK(cudaMemcpyAsync(tops, e->arena_top.p, sizeof(tops), cudaMemcpyDeviceToHost, e->s));
      CK(cudaStreamSynchronize(e->s));
    }
    e->est.slots = e->slots_total;
    if (e->cache_on) {
      unsigned long long cc[CC_N];
      CK(cudaMemcpyAsync(cc, e->c_cc.p, sizeof(cc), cudaMemcpyDeviceToHost, e->s));
      CK(cudaStreamSynchronize(e->s));
      e->est.cache_lines = e->c_lines;
      e->est.cache_admissions = e->c_admissions;
      e->est.last_admitted = e->c_admissions ? cc[CC_ADMIT] : 0;
      e->est.last_evicted = e->c_admissions ? cc[CC_EVICT] : 0;
      e->est.cache_resident = e->c_admissions ? e->c_lines - (cc[CC_FREE] - cc[CC_ADMIT]) : 0;
      e->est.cache_hit_slots = cc[CC_WALK] - std::min(cc[CC_WALK], cc[CC_MISS]);
      e->est.cache_miss_slots = cc[CC_MISS];
    }
    e->est.in_store_bytes = e->in_built ? e->in_capslots * 4 + (uint64_t)e->nv * 20 : 0;
    e->est.in_store_builds = e->in_builds;
    e->est.bfs_bottom_up_rounds = e->bfs_bottom_up_total;
    e->est.host_stagings = e->stagings;
    e->est.pr_warm_starts = e->pr_warm_starts;
    e->est.reclaimed_slots = e->reclaimed_total;
    e->est.last_stage_bytes = e->stage_bytes_last;
    *out = e->est;
  });
}

SGS_API int sgs_cache_refresh(sgs_engine *e) {
  if (!e) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    if (!e->loaded) fail(SGS_ERR_STATE, "no graph loaded");
    CK(cudaSetDevice(e->dev));
    e->cache_admit(/*rotate=*/false);
    e->cache_publish();
    e->sync();
  });
}

SGS_API int sgs_graph_export(sgs_engine *e, uint64_t *row, uint32_t *col, uint32_t *w, int mem) {
  if (!e || !row || !col) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    if (!e->loaded) fail(SGS_ERR_STATE, "no graph loaded");
    CK(cudaSetDevice(e->dev));
    e->export_graph(row, col, w, mem);
  });
}

SGS_API int sgs_query_summaries(sgs_engine *e, uint32_t n, const int *qids, uint64_t *out) {
  if (!e || (n && (!qids || !out))) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->summaries(n, qids, out);
  });
}

SGS_API int sgs_query_summary(sgs_engine *e, int qid, uint64_t out[4]) {
  if (!e || !out) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->summary(e->find(qid), out);
  });
}

// splitmix64 output function and stream (same definitions as the device
// generator in sgs_kernels.cuh).
static inline uint64_t h_fin64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline uint64_t h_mix64(uint64_t x) { return h_fin64(x + 0x9E3779B97F4A7C15ull); }
static inline uint64_t h_stream(uint64_t key, uint64_t i) {
  return h_fin64(key + (i + 1) * 0x9E3779B97F4A7C15ull);
}

SGS_API int sgs_gen_update_stream(uint32_t nv, const uint64_t *row, const uint32_t *col,
                                  uint64_t seed, uint64_t n_ins, uint64_t n_del, uint32_t *ins_src,
                                  uint32_t *ins_dst, uint32_t *del_src, uint32_t *del_dst) {
  if (!row || (row[nv] && !col) || (n_ins && (!ins_src || !ins_dst)) ||
      (n_del && (!del_src || !del_dst))) {
    g_last_error = "null argument";
    return SGS_ERR_INVALID;
  }
  return guarded([&] {
    const uint64_t ne = row[nv];
    if (n_del > ne) fail(SGS_ERR_INVALID, "more deletes than edges");
    if (n_del) {
      std::vector<uint64_t> bits(ne / 64 + 1, 0);
      const uint64_t key = h_mix64(seed ^ 0x44454C45ull);
      uint64_t got = 0, i = 0;
      while (got < n_del) {
        const uint64_t idx =
            (uint64_t)(((unsigned __int128)h_stream(key, i++) * (unsigned __int128)ne) >> 64);
        if (bits[idx >> 6] >> (idx & 63) & 1) continue;
        bits[idx >> 6] |= 1ull << (idx & 63);
        const uint32_t u = (uint32_t)(std::upper_bound(row, row + nv + 1, idx) - row) - 1;
        del_src[got] = u;
        del_dst[got] = col[idx];
        ++got;
      }
    }
    if (n_ins) {
      if (nv < 2) fail(SGS_ERR_INVALID, "graph too small for inserts");
      uint64_t tsz = 1;
      while (tsz < 2 * n_ins + 16) tsz <<= 1;
      std::vector<uint64_t> tab(tsz, ~0ull);
      const uint64_t key = h_mix64(seed ^ 0x494E5345ull);
      uint64_t got = 0, i = 0;
      const uint64_t limit = 64 * n_ins + 1000000;
      while (got < n_ins) {
        if (i > limit) fail(SGS_ERR_INVALID, "graph too dense for the requested inserts");
        const uint64_t h = h_stream(key, i++);
        const uint32_t u = (uint32_t)(((h >> 32) * (uint64_t)nv) >> 32);
        const uint32_t v = (uint32_t)(((h & 0xFFFFFFFFull) * (uint64_t)nv) >> 32);
        if (u == v) continue;
        if (std::binary_search(col + row[u], col + row[u + 1], v)) continue;
        const uint64_t k = ((uint64_t)u << 32) | v;
        uint64_t s = h_mix64(k) & (tsz - 1);
        bool dup = false;
        while (tab[s] != ~0ull) {
          if (tab[s] == k) { dup = true; break; }
          s = (s + 1) & (tsz - 1);
        }
        if (dup) continue;
        tab[s] = k;
        ins_src[got] = u;
        ins_dst[got] = v;
        ++got;
      }
    }
  });
}

SGS_API void sgs_hash_weights(uint64_t wseed, uint64_t n, const uint32_t *src, const uint32_t *dst,
                              uint32_t *w) {
  if (!src || !dst || !w) return;
  const uint64_t key = h_mix64(wseed ^ 0x57454947ull);
  for (uint64_t i = 0; i < n; ++i)
    w[i] = 1u + (uint32_t)(h_fin64(key ^ (((uint64_t)src[i] << 32) | dst[i])) >> 58);
}

SGS_API int sgs_autotune(sgs_engine *e, sgs_tune *out) {
  if (!e || !out) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  return guarded([&] {
    CK(cudaSetDevice(e->dev));
    e->autotune(out);
  });
}

SGS_API int sgs_kernel_timing(sgs_engine *e, int enable) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  return guarded([&] {
    e->ktiming = enable != 0;
    for (auto &k : e->kst) k = sgs_kernel_stats{};
  });
}

SGS_API int sgs_get_kernel_stats(sgs_engine *e, int kind, sgs_kernel_stats *out) {
  if (!e || !out) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  if (kind < 0 || kind >= SGS_K_COUNT) { g_last_error = "bad kernel kind"; return SGS_ERR_INVALID; }
  *out = e->kst[kind];
  return SGS_OK;
}

SGS_API int sgs_get_graph_view(sgs_engine *e, sgs_graph_view *out) {
  if (!e || !out) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  if (!e->loaded) { g_last_error = "no graph loaded"; return SGS_ERR_STATE; }
  return guarded([&] { *out = e->graph_view(); });
}

SGS_API int sgs_app_attach(sgs_engine *e, const sgs_app_hooks *h, int *app_id) {
  if (!e || !h || !app_id) { g_last_error = "null argument"; return SGS_ERR_INVALID; }
  if (!e->loaded) { g_last_error = "no graph loaded"; return SGS_ERR_STATE; }
  return guarded([&] {
    e->apps.push_back({e->next_app, *h});
    *app_id = e->next_app++;
  });
}

SGS_API int sgs_app_detach(sgs_engine *e, int app_id) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  for (size_t i = 0; i < e->apps.size(); ++i)
    if (e->apps[i].id == app_id) {
      e->apps.erase(e->apps.begin() + i);
      return SGS_OK;
    }
  g_last_error = "unknown user algorithm id";
  return SGS_ERR_INVALID;
}

SGS_API void sgs_set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

SGS_API int sgs_synchronize(sgs_engine *e) {
  if (!e) { g_last_error = "null engine"; return SGS_ERR_INVALID; }
  return guarded([&] { CK(cudaStreamSynchronize(e->s)); });
}

}  // extern "C"
