// serve.cpp -- a served request loop over one engine (host code).
//
// No counterpart in the reference, whose drivers run one source through a
// fixed list of snapshots (samples/hybrid_sssp/hybrid_sssp.cu:204-296).
// Here a trace of requests -- update batches and one-shot queries, each with
// an arrival time -- is served in arrival order (FIFO) on one host thread,
// with continuous batching at the granularity of relaxation rounds:
//
//   * BFS/SSSP/CC queries join free lanes of one group kept in flight (up to
//     `slots` lanes in use), between two rounds: a query that arrives while
//     others are on the GPU starts at the next round boundary and its rounds
//     overlap theirs in the same edge passes;
//   * a query leaves as soon as no entry of the frontier carries its lane:
//     its result is read back (summary, and optionally its value/parent
//     vectors) and its lane freed for the next arrival;
//   * an update batch is one snapshot.  When it reaches the head of the
//     queue while lane queries are in flight, it preempts them: it is applied
//     at the next round boundary and the queries in flight restart from
//     their sources on the new snapshot (sgs_config.serve_restarts bounds
//     how often one query may be restarted; once a query in flight has used
//     its restarts, the update waits for the flight to drain).  A query's
//     "version" is the snapshot of its last run: at least the updates that
//     arrived before it, exactly those with serve_restarts = 0.  Queries
//     behind an update wait for it;
//   * PageRank has no lanes (and no source): PR queries share one
//     computation, a job that starts as soon as they reach the head of the
//     queue (later PR queries join it when they reach the head while it
//     runs) and runs a few sweeps per loop iteration between the flight's
//     steps, so lane queries behind it keep being admitted and served (the
//     job has its own frontier buffers; a PageRank start continues from the
//     vector of the previous one, see sgs_config.pr_warm).  Updates do not
//     wait for it: a snapshot amends the job's residual for the out-lists it
//     changes (the cancel/compensate of every PageRank query) and the job
//     continues on the new graph, so its result reflects every update applied
//     before it finished -- at least those that arrived before its requests --
//     and its completions report that version;
//
// With `realtime` the loop waits for arrival times on the wall clock, and
// latency = done_s - arrival_s includes queueing; without it every request
// is taken as soon as the loop reaches it (a closed loop, latency = done_s).
// Times are host wall-clock seconds from the start of the call.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sgs.h"

#ifndef SGS_PR_SHARE_EVERY
#define SGS_PR_SHARE_EVERY 4
#endif

namespace sgs {
void set_last_error(const std::string &msg);
// flight interface (engine.cu)
int flight_free(sgs_engine *e, uint32_t *lanes);
int flight_admit(sgs_engine *e, uint32_t n, const int *algos, const uint32_t *sources, int *ids);
int flight_advance(sgs_engine *e, uint32_t rounds, std::vector<int> &done, uint64_t *running);
int flight_suspend(sgs_engine *e);
int flight_resume(sgs_engine *e);
uint32_t serve_restarts(sgs_engine *e);
int reserve_batch(sgs_engine *e, uint64_t ni, uint64_t nd);
int pr_job_start(sgs_engine *e, int *qid);
int pr_job_advance(sgs_engine *e, uint32_t rounds, int *done);
}  // namespace sgs

namespace {

using clk = std::chrono::steady_clock;

double since(clk::time_point t0) {
  return std::chrono::duration<double>(clk::now() - t0).count();
}

// Rounds between two admission points (and points where an update may
// preempt the flight)
constexpr uint32_t kRoundsPerStep = 2;
// PageRank sweeps per loop iteration: a long job yields to the lane queries
// while any are in flight -- one sweep every kPrShareEvery iterations, so
// the short queries keep most of the GPU -- and runs in longer steps when it
// has the GPU to itself, short enough that an arriving update waits for a
// few sweeps at most
constexpr uint32_t kPrRoundsPerStep = 2;
constexpr uint32_t kPrRoundsPerStepShared = 1;
constexpr uint32_t kPrShareEvery = SGS_PR_SHARE_EVERY;

// Result of a finished query into its completion record.
void finish(sgs_engine *e, int qid, const sgs_request &r, sgs_completion &c) {
  sgs_query_stats qs;
  if (sgs_get_query_stats(e, qid, &qs) == SGS_OK) c.edges = qs.edges_traversed;
  if (c.status == SGS_OK) c.status = sgs_query_summary(e, qid, c.summary);
  if (c.status == SGS_OK && r.value_out)
    c.status = sgs_gather(e, qid, SGS_FIELD_VALUE, r.value_out, SGS_MEM_HOST);
  if (c.status == SGS_OK && r.parent_out && r.algo != SGS_PR)
    c.status = sgs_gather(e, qid, SGS_FIELD_PARENT, r.parent_out, SGS_MEM_HOST);
}

bool lane_query(const sgs_request &r) { return r.kind == SGS_REQ_QUERY && r.algo != SGS_PR; }

}  // namespace

extern "C" {

SGS_API int sgs_serve(sgs_engine *e, const sgs_request *req, uint32_t n, uint32_t slots,
                      int realtime, sgs_completion *out) {
  if (!e || (n && (!req || !out))) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  for (uint32_t i = 0; i < n; ++i) {
    const sgs_request &r = req[i];
    if (r.kind != SGS_REQ_QUERY && r.kind != SGS_REQ_UPDATE) {
      sgs::set_last_error("request " + std::to_string(i) + ": unknown kind");
      return SGS_ERR_INVALID;
    }
    if (!(r.arrival_s >= 0.0)) {
      sgs::set_last_error("request " + std::to_string(i) + ": arrival time must be >= 0");
      return SGS_ERR_INVALID;
    }
    if (r.kind == SGS_REQ_QUERY && (r.algo < 0 || r.algo > 3)) {
      sgs::set_last_error("request " + std::to_string(i) + ": unknown algorithm");
      return SGS_ERR_INVALID;
    }
  }
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return req[a].arrival_s < req[b].arrival_s; });
  for (uint32_t i = 0; i < n; ++i) std::memset(&out[i], 0, sizeof(sgs_completion));

  // batch buffers for the trace's largest update, before the clock starts
  // (if that fails, e.g. no graph is loaded, each update reports its error)
  uint64_t max_ni = 0, max_nd = 0;
  for (uint32_t i = 0; i < n; ++i)
    if (req[i].kind == SGS_REQ_UPDATE) {
      max_ni = std::max(max_ni, req[i].n_ins);
      max_nd = std::max(max_nd, req[i].n_del);
    }
  if (max_ni || max_nd) (void)sgs::reserve_batch(e, max_ni, max_nd);

  const clk::time_point t0 = clk::now();
  std::deque<uint32_t> pending;
  std::map<int, uint32_t> inflight;  // query id -> request
  uint32_t next = 0, done = 0;
  uint64_t version = 0, running = 0;
  std::vector<int> algos, qids, fin;
  std::vector<uint32_t> sources, batch;
  const uint32_t max_restarts = sgs::serve_restarts(e);
  uint32_t pr_turn = 0;  // loop iterations with lane queries in flight
  int pr_qid = 0;                 // the PageRank job, if one runs
  std::vector<uint32_t> pr_batch;  // its requests
  double pr_start = 0;
  // Applies the update at the head of the queue (one snapshot).
  auto apply_head_update = [&]() {
    const uint32_t head = pending.front();
    const sgs_request &r = req[head];
    pending.pop_front();
    sgs_completion &c = out[head];
    c.start_s = since(t0);
    c.status = sgs_apply_batch(e, r.ins_src, r.ins_dst, r.ins_w, r.n_ins, r.del_src, r.del_dst,
                               r.n_del, SGS_MEM_HOST);
    if (c.status == SGS_OK) {
      ++version;
      sgs_engine_stats st;
      if (sgs_get_engine_stats(e, &st) == SGS_OK) c.edges = st.last_batch_edges;
    }
    c.version = version;
    c.batch = 1;
    c.done_s = since(t0);
    ++done;
  };
  // Fails every lane query in flight with `rc` (the flight could not go on).
  auto fail_flight = [&](int rc) {
    for (auto &kv : inflight) {
      out[kv.second].status = rc;
      out[kv.second].done_s = since(t0);
      sgs_query_remove(e, kv.first);
      ++done;
    }
    inflight.clear();
  };
  auto update_at_head = [&]() {
    return !pending.empty() && req[pending.front()].kind == SGS_REQ_UPDATE;
  };
  auto pr_at_head = [&]() {
    return !pending.empty() && req[pending.front()].kind == SGS_REQ_QUERY &&
           req[pending.front()].algo == SGS_PR;
  };
  while (done < n) {
    const double now = since(t0);
    while (next < n && (!realtime || req[order[next]].arrival_s <= now)) pending.push_back(order[next++]);

    // 0. PageRank requests at the head join the job that runs -- its result
    // reflects every update applied before it finishes, so at least those
    // that arrived before them -- or start one
    if (pr_qid && pr_at_head()) {
      const double now_s = since(t0);
      while (pr_at_head()) {
        const uint32_t k = pending.front();
        pending.pop_front();
        pr_batch.push_back(k);
        out[k].start_s = now_s;
        out[k].status = SGS_OK;
      }
      for (uint32_t k : pr_batch) out[k].batch = (uint32_t)pr_batch.size();
    }
    if (!pr_qid && pr_at_head()) {
      pr_batch.clear();
      while (pr_at_head()) {
        pr_batch.push_back(pending.front());
        pending.pop_front();
      }
      pr_start = since(t0);
      int qid = 0;
      const int rc = sgs::pr_job_start(e, &qid);
      for (uint32_t k : pr_batch) {
        out[k].start_s = pr_start;
        out[k].version = version;
        out[k].batch = (uint32_t)pr_batch.size();
        out[k].status = rc;
      }
      if (rc == SGS_OK) {
        pr_qid = qid;
      } else {
        if (qid > 0) sgs_query_remove(e, qid);
        for (uint32_t k : pr_batch) out[k].done_s = since(t0);
        done += (uint32_t)pr_batch.size();
      }
    }

    // 1. admission: lane queries at the head of the queue into free lanes
    if (!pending.empty() && lane_query(req[pending.front()])) {
      uint32_t free = 0;
      if (sgs::flight_free(e, &free) != SGS_OK) free = 0;
      if (slots) free = std::min<uint32_t>(free, slots > inflight.size() ? slots - (uint32_t)inflight.size() : 0u);
      batch.clear();
      while (batch.size() < free && !pending.empty() && lane_query(req[pending.front()])) {
        batch.push_back(pending.front());
        pending.pop_front();
      }
      const uint32_t nb = (uint32_t)batch.size();
      if (nb) {
        algos.resize(nb);
        sources.resize(nb);
        qids.assign(nb, 0);
        for (uint32_t k = 0; k < nb; ++k) {
          algos[k] = req[batch[k]].algo;
          sources[k] = req[batch[k]].source;
        }
        const double start = since(t0);
        const int rc = sgs::flight_admit(e, nb, algos.data(), sources.data(), qids.data());
        const uint32_t lanes_now = (uint32_t)inflight.size() + nb;  // lanes in flight with it
        for (uint32_t k = 0; k < nb; ++k) {
          sgs_completion &c = out[batch[k]];
          c.start_s = start;
          c.version = version;
          c.batch = lanes_now;
          c.status = rc;
          if (rc == SGS_OK) {
            inflight[qids[k]] = batch[k];
          } else {
            if (qids[k] > 0) sgs_query_remove(e, qids[k]);
            c.done_s = since(t0);
            ++done;
          }
        }
      }
    }

    if (inflight.empty() && !pending.empty() && lane_query(req[pending.front()])) {
      // nothing in flight and still no lane for the head: the flight cannot
      // start (e.g. its state could not be allocated); fail the request
      const uint32_t head = pending.front();
      pending.pop_front();
      out[head].status = SGS_ERR_STATE;
      out[head].version = version;
      out[head].start_s = out[head].done_s = since(t0);
      ++done;
      continue;
    }

    // 1b. an update at the head preempts the lane queries in flight, unless
    // one of them has used up its restarts: the flight stops at this round
    // boundary, the snapshot is applied, and the queries restart on it
    if (!inflight.empty() && update_at_head() && max_restarts) {
      bool can = true;
      for (auto &kv : inflight) can = can && out[kv.second].restarts < max_restarts;
      if (can) {
        int rc = sgs::flight_suspend(e);
        if (rc != SGS_OK) {
          fail_flight(rc);
          continue;
        }
        apply_head_update();
        rc = sgs::flight_resume(e);
        if (rc != SGS_OK) {
          fail_flight(rc);
          continue;
        }
        for (auto &kv : inflight) {
          ++out[kv.second].restarts;
          out[kv.second].version = version;
        }
        continue;
      }
    }

    bool worked = false;
    // 2. the PageRank job: a few sweeps
    if (pr_qid && (inflight.empty() || ++pr_turn % kPrShareEvery == 0)) {
      worked = true;
      int fin_pr = 0;
      const int rc =
          sgs::pr_job_advance(e, inflight.empty() ? kPrRoundsPerStep : kPrRoundsPerStepShared, &fin_pr);
      if (rc != SGS_OK || fin_pr) {
        for (uint32_t k : pr_batch) {
          sgs_completion &c = out[k];
          c.status = rc;
          c.version = version;  // the snapshots applied while it ran included
          if (rc == SGS_OK) finish(e, pr_qid, req[k], c);
        }
        sgs_query_remove(e, pr_qid);
        const double end = since(t0);
        for (uint32_t k : pr_batch) out[k].done_s = end;
        done += (uint32_t)pr_batch.size();
        pr_qid = 0;
      }
    }

    // 3. the flight: a few rounds, then retire the lanes that finished
    if (!inflight.empty()) {
      worked = true;
      const int rc = sgs::flight_advance(e, kRoundsPerStep, fin, &running);
      if (rc != SGS_OK) {  // fail every query in flight, keep serving
        fail_flight(rc);
        continue;
      }
      for (int qid : fin) {
        auto it = inflight.find(qid);
        if (it == inflight.end()) continue;
        finish(e, qid, req[it->second], out[it->second]);
        sgs_query_remove(e, qid);
        out[it->second].done_s = since(t0);
        inflight.erase(it);
        ++done;
      }
    }
    // 4. an update at the head, once no lane query is in flight (a PageRank
    // job may be running: the snapshot amends it)
    if (inflight.empty() && update_at_head()) {
      apply_head_update();
      continue;
    }
    if (worked) continue;

    // 5. idle until the next arrival
    if (pending.empty() && next < n) {
      const double wait = req[order[next]].arrival_s - since(t0);
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
    }
  }
  (void)running;
  return SGS_OK;
}

}  // extern "C"
