// serve.cpp -- a served request loop over one engine (host code).
//
// No counterpart in the reference, whose drivers run one source through a
// fixed list of snapshots (samples/hybrid_sssp/hybrid_sssp.cu:204-296).
// Here a trace of requests -- update batches and one-shot queries, each with
// an arrival time -- is served in arrival order on one host thread:
//
//   * an update batch is one snapshot (sgs_apply_batch), applied alone and
//     in order, so every query sees exactly the updates that arrived before
//     it and none after it (its "version");
//   * consecutive queries at the head of the queue are admitted together
//     (continuous batching): up to `slots` of them go through one
//     sgs_query_add_many, so the BFS/SSSP/CC ones share group lanes and one
//     convergence, and the PageRank ones (which have no source) share one
//     computation; queries that arrive meanwhile wait for the next step;
//   * a query's result (summary, and optionally its value/parent vectors)
//     is read back and the query retired before the next step.
//
// `slots` bounds the queries in flight: the caller sizes it from the HBM
// left after the graph (a lane's state is resident while it runs).  With
// `realtime` the loop waits for arrival times on the wall clock, and
// latency = done_s - arrival_s includes queueing; without it every request
// is taken as soon as the loop reaches it (a closed loop, latency = done_s).
// Times are host wall-clock seconds from the start of the call.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sgs.h"

namespace sgs {
void set_last_error(const std::string &msg);
}

namespace {

using clk = std::chrono::steady_clock;

double since(clk::time_point t0) {
  return std::chrono::duration<double>(clk::now() - t0).count();
}

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
  }
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return req[a].arrival_s < req[b].arrival_s; });
  for (uint32_t i = 0; i < n; ++i) std::memset(&out[i], 0, sizeof(sgs_completion));

  const clk::time_point t0 = clk::now();
  std::deque<uint32_t> pending;
  uint32_t next = 0, done = 0;
  uint64_t version = 0;
  std::vector<int> algos, qids;
  std::vector<uint32_t> sources, batch, slot;
  while (done < n) {
    double now = since(t0);
    while (next < n && (!realtime || req[order[next]].arrival_s <= now)) pending.push_back(order[next++]);
    if (pending.empty()) {
      // idle until the next arrival
      const double wait = req[order[next]].arrival_s - now;
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
      continue;
    }
    const uint32_t head = pending.front();
    if (req[head].kind == SGS_REQ_UPDATE) {
      pending.pop_front();
      const sgs_request &r = req[head];
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
      continue;
    }
    // the run of queries at the head of the queue, up to `slots`
    batch.clear();
    while (!pending.empty() && req[pending.front()].kind == SGS_REQ_QUERY &&
           (slots == 0 || batch.size() < slots)) {
      batch.push_back(pending.front());
      pending.pop_front();
    }
    const uint32_t nb = (uint32_t)batch.size();
    // PageRank does not depend on the source: the batch's PR queries share
    // one computation (slot[k] = which registered query answers request k)
    algos.clear();
    sources.clear();
    slot.assign(nb, 0);
    int pr_slot = -1;
    for (uint32_t k = 0; k < nb; ++k) {
      const sgs_request &r = req[batch[k]];
      if (r.algo == SGS_PR && pr_slot >= 0) {
        slot[k] = (uint32_t)pr_slot;
        continue;
      }
      slot[k] = (uint32_t)algos.size();
      if (r.algo == SGS_PR) pr_slot = (int)algos.size();
      algos.push_back(r.algo);
      sources.push_back(r.source);
    }
    const uint32_t nq = (uint32_t)algos.size();
    qids.assign(nq, 0);
    const double start = since(t0);
    const int rc = sgs_query_add_many(e, nq, algos.data(), sources.data(), qids.data());
    for (uint32_t k = 0; k < nb; ++k) {
      const sgs_request &r = req[batch[k]];
      sgs_completion &c = out[batch[k]];
      const int qid = qids[slot[k]];
      c.start_s = start;
      c.version = version;
      c.batch = nb;
      c.status = rc;
      if (rc == SGS_OK) {
        sgs_query_stats qs;
        if (sgs_get_query_stats(e, qid, &qs) == SGS_OK) c.edges = qs.edges_traversed;
        c.status = sgs_query_summary(e, qid, c.summary);
        if (c.status == SGS_OK && r.value_out)
          c.status = sgs_gather(e, qid, SGS_FIELD_VALUE, r.value_out, SGS_MEM_HOST);
        if (c.status == SGS_OK && r.parent_out && r.algo != SGS_PR)
          c.status = sgs_gather(e, qid, SGS_FIELD_PARENT, r.parent_out, SGS_MEM_HOST);
      }
    }
    // retire the batch (a failed add may have registered some of them)
    for (uint32_t k = 0; k < nq; ++k)
      if (qids[k] > 0) sgs_query_remove(e, qids[k]);
    const double fin = since(t0);
    for (uint32_t k = 0; k < nb; ++k) out[batch[k]].done_s = fin;
    done += nb;
  }
  return SGS_OK;
}

}  // extern "C"
