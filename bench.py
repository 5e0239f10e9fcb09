#!/usr/bin/env python
"""GTEPS per snapshot of the incremental streaming-graph engine on B200.

Workload (the plain incremental SSSP/BFS/CC configuration): directed R-MAT
scale 24 (16.7M vertices, edge factor 16, a/b/c/d = 0.57/0.19/0.19/0.05,
seed 1, self-loops and duplicates removed), uint32 weights uniform in [1,64]
from the seed, HBM edge budget 4 GB, queries SSSP(0), BFS(0) and CC kept up
to date over snapshots of 1M updates (500k inserts of new edges + 500k
deletes of existing edges).  Synthetic data generated on the device.

One step = one snapshot: the batch is applied to the graph and the three
queries are brought up to date incrementally.  GTEPS = edges traversed by the
three queries (invalidation + re-push + convergence rounds) / step time.

* value: batches already resident in HBM, time from CUDA events on the
  engine's stream (summed over the K timed steps);
* e2e:   the same through the C ABI with the batch in pinned host memory
  (host->device copy inside the step) and a device->host read of each query's
  summary (reached count, value sum, max, parent sum) after every step;
  wall-clock per step.

--impl reference times the reference's own CPU code for this path on the
host cores (oracle/_ref, compiled from the reference sources) on a bounded
sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "c-gpustreamgraph_b200"))

import numpy as np  # noqa: E402

METRIC = "GTEPS per snapshot (incremental SSSP+BFS+CC, R-MAT s24, 1M updates/snapshot)"
UNIT = "GTEPS"
L2_BYTES = 126 * 2**20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--updates", type=int, default=1_000_000)
    ap.add_argument("--budget-gb", type=float, default=4.0)
    ap.add_argument("--permute", action="store_true",
                    help="relabel the R-MAT vertices by a seeded random permutation (hubs spread over "
                         "all segments); the source is vertex 0's new label")
    ap.add_argument("--cache-gb", type=float, default=0.0,
                    help="device edge cache of the host tier, carved out of --budget-gb (0: none)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--ref-seconds", type=float, default=60.0,
                    help="reference arm: traversal time budget over the timed snapshots")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations' sub-records after the headline")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip sgs_autotune (by default it picks the relaxation map's CTAs per SM "
                         "and the launch mode by timing a probe, before the timed region)")
    ap.add_argument("--persistent", type=int, default=None,
                    help="1: each relaxation phase as one cooperative launch over rounds")
    ap.add_argument("--workload", default="snapshot",
                    choices=["snapshot", "ppr", "batched", "served", "pagerank", "bfs"],
                    help="snapshot: incremental SSSP/BFS/CC (the headline); ppr: weighted "
                         "personalized PageRank forward + adjoint; batched: 256 BFS + 256 SSSP "
                         "queries kept up to date together")
    ap.add_argument("--batched-scale", type=int, default=22)
    ap.add_argument("--batched-bfs", type=int, default=256)
    ap.add_argument("--batched-sssp", type=int, default=256)
    ap.add_argument("--batched-updates", type=int, default=100_000)
    ap.add_argument("--group-size", type=int, default=64)
    ap.add_argument("--served-scale", type=int, default=26)
    ap.add_argument("--served-seconds", type=float, default=30.0)
    ap.add_argument("--served-rate", type=float, default=12.0, help="requests per second (Poisson)")
    ap.add_argument("--served-budget-gb", type=float, default=16.0)
    ap.add_argument("--slots", type=int, default=64)
    ap.add_argument("--served-group-size", type=int, default=4,
                    help="lanes of the served flight: 1-4 a narrow group (16-B state rows), 5-64 a wide one")
    ap.add_argument("--serve-restarts", type=int, default=2,
                    help="served loop: times an update may preempt (restart) one query in flight; "
                         "0: updates wait for the flight to drain")
    ap.add_argument("--served-plain", type=int, default=16,
                    help="served workload: queries of the trace timed alone on the plain engine")
    ap.add_argument("--plain-sample", type=int, default=32,
                    help="batched workload: queries of the sample run one per edge pass")
    ap.add_argument("--pull", type=int, default=None,
                    help="engine pull bits (1: PageRank pull sweeps, 2: direction-optimizing BFS); "
                         "library default otherwise")
    ap.add_argument("--host-policy", type=int, default=None,
                    help="reads of the host tier in a repair (-hybrid): 0 zero-copy, 1 explicit copy "
                         "every snapshot, 2 explicit copy for dense repairs; library default otherwise")
    ap.add_argument("--repair", type=int, default=None,
                    help="1: narrow groups repair deletions by pulling into the reset vertices (fewer edges "
                         "read and counted); library default (0: the reference's re-push) otherwise")
    ap.add_argument("--pr-scale", type=int, default=16)
    ap.add_argument("--pr-updates", type=int, default=20_000)
    ap.add_argument("--bfs-sources", type=int, default=8)
    ap.add_argument("--ppr-scale", type=int, default=22)
    ap.add_argument("--ppr-vectors", type=int, default=64)
    ap.add_argument("--ppr-seeds", type=int, default=32)
    ap.add_argument("--ppr-targets", type=int, default=1024)
    return ap.parse_args()


# ----------------------------------------------------------------- ranks
class Ranks:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.dist, self.torch, self.pg = dist, torch, True

    def _reduce(self, x, op):
        if not self.pg:
            return x
        t = self.torch.tensor([float(x)], dtype=self.torch.float64,
                              device="cuda" if self.torch.cuda.is_available() else "cpu")
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return self._reduce(x, self.dist.ReduceOp.MAX) if self.pg else x

    def sum(self, x):
        return self._reduce(x, self.dist.ReduceOp.SUM) if self.pg else x

    def barrier(self):
        if self.pg:
            self.dist.barrier()

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


# ----------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        load = [s for s in sm if s > 0.5 * (max(mx) if mx else 0)] or sm
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def pers(a):
    """Engine options for --persistent / --pull (the library defaults otherwise)."""
    o = {} if a.persistent is None else {"persistent": int(a.persistent)}
    if getattr(a, "pull", None) is not None:
        o["pull"] = int(a.pull)
    if getattr(a, "host_policy", None) is not None:
        o["host_policy"] = int(a.host_policy)
    if getattr(a, "repair", None) is not None:
        o["repair"] = int(a.repair)
    return o


def measure_h2d_gbs(dev, nbytes=1 << 30, reps=3):
    """Pinned host -> device copy bandwidth (GB/s), best of `reps`, CUDA
    events: the host-link peak for blocks kept in the pinned-host tier."""
    import torch

    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    best = 0.0
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        d.copy_(h, non_blocking=True)
        b.record()
        b.synchronize()
        best = max(best, nbytes / (a.elapsed_time(b) * 1e-3) / 1e9)
    del h, d
    return best


def profile_traffic():
    """Bytes per slot / per entry of the dominant kernel from the committed ncu
    summary (profiles/relax_traffic.json), if present."""
    path = os.path.join(REPO, "profiles", "relax_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def permute_graph(e, seed):
    """Reloads the engine's graph with vertex v relabelled p[v] (p a seeded
    random permutation, as the reference's unused GAP generator permutes,
    include/framework/generator.h:53-63); returns p[0]."""
    row, col, w = e.export(weights=True)
    nv = len(row) - 1
    p = np.random.default_rng(seed * 7919 + 17).permutation(nv).astype(np.uint32)
    src = p[np.repeat(np.arange(nv, dtype=np.uint32), np.diff(row).astype(np.int64))]
    dst = p[col]
    del row, col
    e.load_edge_list(src, dst, w, nv=nv)
    return int(p[0])


# ----------------------------------------------------------------- engine arm
def engine_arm(a, R):
    import torch

    import sgs

    dev = torch.device("cuda", R.local)
    torch.cuda.set_device(dev)
    e = sgs.Engine(device=R.local, hbm_budget_gb=a.budget_gb, cache_gb=a.cache_gb,
                   weight_mode=sgs.W_EXPLICIT, **pers(a))
    t0 = time.time()
    e.load_rmat(a.scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
    source = 0
    if a.permute:
        source = permute_graph(e, a.seed)
    t_gen = time.time() - t0
    st0 = e.engine_stats()
    nv = int(st0["nv"])
    row, col, _ = e.export()
    half = a.updates // 2
    nbatch = a.warmup + a.steps
    i_s, i_d, d_s, d_d = sgs.gen_update_stream(nv, row, col, a.seed * 1000003, nbatch * half,
                                               nbatch * half)
    i_w = sgs.hash_weights(a.seed, i_s, i_d)
    del row, col
    tune = e.autotune() if a.autotune else None
    queries = [e.add_query(sgs.SSSP, source), e.add_query(sgs.BFS, source), e.add_query(sgs.CC, 0)]
    e.cache_refresh()  # warm the edge cache after the static run (no-op without one)

    def batch(k):
        s = slice(k * half, (k + 1) * half)
        return i_s[s], i_d[s], i_w[s], d_s[s], d_d[s]

    def to_dev(arrs):
        return [torch.from_numpy(x.view(np.int32)).to(dev) for x in arrs]

    dev_batches = [to_dev(batch(k)) for k in range(a.warmup + a.steps)]

    def run_dev(b):
        isrc, idst, iw, dsrc, ddst = b
        e.apply_batch_ptr(isrc.data_ptr(), idst.data_ptr(), iw.data_ptr(), half,
                          dsrc.data_ptr(), ddst.data_ptr(), half, sgs.MEM_DEVICE)
        return sum(q.stats()["edges_traversed"] for q in queries)

    for k in range(a.warmup):
        run_dev(dev_batches[k])
    # ---------------- timed region (inputs resident in HBM)
    e.kernel_timing(True)
    clocks = Clocks(R.local)
    R.barrier()
    torch.cuda.synchronize()
    e.synchronize()
    cs0 = e.engine_stats()
    launches0 = cs0["kernel_launches"]
    clocks.start()
    w0 = time.perf_counter()
    edges = 0
    dev_ms = 0.0
    per_step = []
    for k in range(a.steps):
        ed = run_dev(dev_batches[a.warmup + k])
        ms = e.engine_stats()["last_batch_ms"]
        edges += ed
        dev_ms += ms
        per_step.append((ed, ms))
    e.synchronize()
    torch.cuda.synchronize()
    R.barrier()
    wall_ms = (time.perf_counter() - w0) * 1e3
    clk = clocks.stop()
    cs1 = e.engine_stats()
    gpu_launches = int(cs1["kernel_launches"] - launches0)
    kst = e.kernel_stats()
    e.kernel_timing(False)
    del dev_batches
    cache = None
    if cs1["cache_lines"]:
        hit = cs1["cache_hit_slots"] - cs0["cache_hit_slots"]
        miss = cs1["cache_miss_slots"] - cs0["cache_miss_slots"]
        cache = {"gb": a.cache_gb, "lines": int(cs1["cache_lines"]), "resident": int(cs1["cache_resident"]),
                 "admissions": int(cs1["cache_admissions"] - cs0["cache_admissions"]),
                 "last_admitted": int(cs1["last_admitted"]), "last_evicted": int(cs1["last_evicted"]),
                 "host_tier_slots_timed": int(hit + miss),
                 "hit_fraction": round(hit / max(hit + miss, 1), 4)}
    # ---------------- e2e (host pinned inputs, summaries read back)
    # The same snapshots as the device-timed region, on the graph loaded
    # afresh: the warm-up snapshots are replayed from device memory (untimed;
    # the last of them is the pipeline's untimed first step), then the timed
    # steps.  Later snapshots of the stream cost more -- its uniform inserts
    # replace skewed R-MAT edges, so fewer state reads hit L2 -- and timing
    # them would not compare with `value`.
    e2e = None
    if not a.no_e2e:
        e.load_rmat(a.scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
        if a.permute:
            permute_graph(e, a.seed)
        queries = [e.add_query(sgs.SSSP, source), e.add_query(sgs.BFS, source), e.add_query(sgs.CC, 0)]
        e.cache_refresh()
        w0k = max(a.warmup - 1, 0)
        for k in range(w0k):
            run_dev(to_dev(batch(k)))
        host = []
        for k in range(w0k, a.warmup + a.steps):  # the untimed pipelined step first (if any)
            arrs = batch(k)
            pinned = []
            for x in arrs:
                t = torch.empty(len(x), dtype=torch.int32, pin_memory=True)
                t.numpy()[:] = x.view(np.int32)
                pinned.append(t)
            host.append(pinned)
        R.barrier()
        torch.cuda.synchronize()
        e_edges, e_ms = 0, 0.0
        out_bytes = 0

        lead = a.warmup - w0k  # 1: host[0] is the last warm-up snapshot

        def stage(k):
            isrc, idst, iw, dsrc, ddst = host[k + lead]
            e.stage_batch_ptr(isrc.data_ptr(), idst.data_ptr(), iw.data_ptr(), half,
                              dsrc.data_ptr(), ddst.data_ptr(), half, sgs.MEM_HOST)

        if lead:
            stage(-1)  # warm-up: copy stream, staging slots and events set up
            e.apply_staged()
        torch.cuda.synchronize()

        # pipelined: step k's pinned-host batch is copied while step k-1 runs
        # (sgs_stage_batch on the copy stream), then applied and every query's
        # summary read back; all copies lie inside the timed region
        import gc
        gc.disable()  # no collector pauses inside the timed loop
        step_ms = []
        t1 = time.perf_counter()
        stage(0)
        for k in range(a.steps):
            tk = time.perf_counter()
            if k + 1 < a.steps:
                stage(k + 1)
            e.apply_staged()
            sums = e.summaries(queries)
            out_bytes = sums.nbytes
            e_edges += sum(q.stats()["edges_traversed"] for q in queries)
            step_ms.append(round((time.perf_counter() - tk) * 1e3, 3))
        e_ms = (time.perf_counter() - t1) * 1e3
        gc.enable()
        R.barrier()
        e2e_ms = R.max(e_ms)
        e2e = {"value": R.sum(e_edges) / (e2e_ms * 1e6), "unit": UNIT,
               "h2d_bytes_per_step": half * 3 * 4 + half * 2 * 4,
               "d2h_bytes_per_step": out_bytes,
               "ms_per_step": e2e_ms / a.steps, "step_ms": step_ms,
               "note": "the device-timed snapshots again, on the graph loaded afresh, through the C ABI "
                       "from pinned host batches (pipelined staging), summaries read back every step"}
    # ---------------- full-size self check: incremental == from-scratch
    # (parents are not unique, so the check compares reached count, value sum
    # and max value)
    fresh = [e.add_query(sgs.SSSP, source), e.add_query(sgs.BFS, source), e.add_query(sgs.CC, 0)]
    selfcheck = {}
    for name, q, f in zip(("sssp", "bfs", "cc"), queries, fresh):
        selfcheck[name] = bool(np.array_equal(q.summary()[:3], f.summary()[:3]))
    fs = fresh[0].stats()
    static_gteps = fs["edges_traversed"] / (fs["ms"] * 1e6) if fs["ms"] > 0 else None
    st = e.engine_stats()
    # ---------------- aggregate over ranks (replicas)
    T = R.max(dev_ms)
    tot_edges = R.sum(edges)
    value = tot_edges / (T * 1e6)
    # roofline of the dominant kernel class
    dom = max(kst, key=lambda k: kst[k]["ms"])
    kd = kst[dom]
    peak, peak_src = measured_peak_hbm()
    achieved = kd["bytes_alg"] / (kd["ms"] * 1e-3) / 1e9 if kd["ms"] > 0 else 0.0
    # traffic: DRAM bytes per walked slot of this kernel from the committed
    # ncu capture (profiles/relax_traffic.json), scaled to the average launch
    tr = profile_traffic()
    traffic = None
    if tr and dom in tr.get("per_kind", {}) and kd["launches"]:
        traffic = round(tr["per_kind"][dom]["dram_bytes_per_slot"] * kd["slots"] / kd["launches"])
    roof = {"bound": "hbm", "kernel": f"group_map<{dom}>", "achieved": round(achieved, 1),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_source": peak_src, "traffic": traffic,
            "launches": kd["launches"], "avg_launch_ms": kd["ms"] / max(kd["launches"], 1),
            "alg_bytes_per_launch": kd["bytes_alg"] / max(kd["launches"], 1)}
    if kd["max_ms"] > 0:
        sweep = kd["max_bytes_alg"] / (kd["max_ms"] * 1e-3) / 1e9
        roof["largest_launch"] = {"slots": kd["max_slots"], "entries": kd["max_entries"],
                                  "ms": round(kd["max_ms"], 4), "achieved": round(sweep, 1),
                                  "frac": round(sweep / peak, 4)}
        hs = kd.get("max_host_slots", 0)
        if hs:
            # blocks in the pinned-host tier are read over the host link: 4-B
            # ids (+4-B weights) per slot against the measured pinned H2D rate
            h2d = measure_h2d_gbs(dev)
            hb = hs * 8  # explicit weights: the SSSP lane reads them
            got = hb / (kd["max_ms"] * 1e-3) / 1e9
            roof["largest_launch"]["host_link"] = {
                "host_slots": int(hs), "host_bytes": int(hb), "achieved": round(got, 1),
                "peak": round(h2d, 1), "unit": "GB/s", "frac": round(got / h2d, 4),
                "peak_source": "measured here (pinned H2D copy, 1 GiB, best of 3)"}
            if hs > kd["max_slots"] // 2:
                # most of the sweep crosses the host link: that is its bound
                roof.update({"bound": "host-link", "achieved": round(got, 1), "peak": round(h2d, 1),
                             "frac": round(got / h2d, 4), "peak_source": "measured pinned H2D",
                             "note": "dominant launch (the sweep) reads mostly host-resident blocks"})
    launches = int(sum(k["launches"] for k in kst.values()))
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": R.world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(T / a.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (device R-MAT, seeded weights and update stream)",
        "config": snapshot_config(a, nv, st0["ne"]),
        "engine": {"ne_final": int(st["ne"]),
                   "hbm_resident_fraction": st["hbm_resident_vertices"] / max(nv, 1),
                   "arena_bytes_hbm": int(st["arena_bytes_hbm"]),
                   "arena_bytes_host": int(st["arena_bytes_host"]),
                   "edge_arena_vs_l2": "edge arena %.1f GB vs %d MB L2" % (
                       st["arena_bytes_hbm"] / 1e9, L2_BYTES // 2**20),
                   "parallelism": "replicas" if R.world > 1 else "single GPU",
                   "autotune": tune, "persistent": a.persistent, "edge_cache": cache,
                   "host_policy": a.host_policy, "host_stagings": int(st["host_stagings"]),
                   "repair": a.repair},
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "roofline": roof,
        "clocks": clk,
        "wall_ms_timed": round(wall_ms, 2),
        "edges_per_step": round(edges / a.steps),
        "selfcheck_incremental_eq_static": selfcheck,
        "static_sssp_gteps": round(static_gteps, 3) if static_gteps else None,
        "gen_s": round(t_gen, 2),
        "kernel_stats": {k: {kk: (round(vv, 4) if isinstance(vv, float) else vv) for kk, vv in v.items()}
                         for k, v in kst.items()},
    }
    out["gpu_launches_relax"] = launches
    out["gpu_launches_note"] = "own kernels only; CUB sorts/scans of the update batch not counted"
    if R.rank == 0 and R.world == 1 and not a.no_cpu:
        out["cpu_baseline"] = cpu_baseline(e, a)
    e.close()
    return out


def cpu_baseline(e, a):
    """The oracle's restatements of the reference's serial host oracles
    (SSSPHostNaive FIFO Bellman-Ford with the explicit weights, BFSHost, and
    the directed min-label CC), from scratch on the final graph, each stopped
    after an edge budget sized for about a third of --cpu-seconds; 1 thread."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O

    row, col, w = e.export(weights=True)
    nv = len(row) - 1
    parts = {}
    per = a.cpu_seconds / 3.0
    # calibrate the relax rate on a small budget, then size each run
    t = time.perf_counter()
    _, e0 = O.sssp_fifo(nv, row, col, w, 0, max_edges=20_000_000)
    rate = e0 / max(time.perf_counter() - t, 1e-6)
    budget = int(rate * per)
    t = time.perf_counter()
    _, es = O.sssp_fifo(nv, row, col, w, 0, max_edges=budget)
    ts = time.perf_counter() - t
    parts["sssp_fifo"] = (es, ts)
    t = time.perf_counter()
    _, eb = O.bfs_fifo(nv, row, col, 0, max_edges=budget)
    tb = time.perf_counter() - t
    parts["bfs_fifo"] = (eb, tb)
    t = time.perf_counter()
    O.cc(nv, row, col)
    tc = time.perf_counter() - t
    parts["cc"] = (int(row[-1]), tc)
    tot_e = sum(p[0] for p in parts.values())
    tot_t = sum(p[1] for p in parts.values())
    return {"value": round(tot_e / tot_t / 1e9, 4), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "from-scratch SSSP (FIFO, restating SSSPHostNaive) and BFS (restating BFSHost) "
                      "from source 0, each stopped after %d relaxations, plus full directed CC, on the "
                      "final scale-%d graph; single thread" % (budget, a.scale),
            "parts": {k: {"edges": int(v[0]), "s": round(v[1], 3)} for k, v in parts.items()}}


# ----------------------------------------------------------------- batched arm
BATCHED_METRIC = ("GTEPS per snapshot, batched multi-source ({nb} BFS + {ns} SSSP, R-MAT s{scale}, "
                  "{upd} updates/snapshot)")


def largest_wcc_sources(nv, row, col, n, seed):
    """n distinct vertices uniform from the largest weakly connected
    component (scipy's connected components on the exported CSR)."""
    import scipy.sparse as sp
    import scipy.sparse.csgraph as cg

    A = sp.csr_matrix((np.ones(len(col), np.int8), col.astype(np.int64), row.astype(np.int64)),
                      shape=(nv, nv))
    _, lab = cg.connected_components(A, directed=True, connection="weak")
    big = int(np.argmax(np.bincount(lab)))
    cand = np.nonzero(lab == big)[0]
    rng = np.random.default_rng(seed)
    return rng.choice(cand, n, replace=False).astype(np.uint32), len(cand)


def run_snapshots(e, queries, batches, dev_of, warmup, steps):
    """Applies warm-up then timed snapshots (device-resident batches);
    returns (lane-edges traversed, device ms) over the timed ones."""
    edges, ms = 0, 0.0
    for k in range(warmup + steps):
        isrc, idst, iw, dsrc, ddst, half = dev_of(batches[k])
        e.apply_batch_ptr(isrc.data_ptr(), idst.data_ptr(), iw.data_ptr(), half,
                          dsrc.data_ptr(), ddst.data_ptr(), half, 1)
        if k >= warmup:
            edges += sum(q.stats()["edges_traversed"] for q in queries)
            ms += e.engine_stats()["last_batch_ms"]
    return edges, ms


def batched_arm(a, R):
    """N1: 256 BFS + 256 SSSP queries with sources uniform from the largest
    WCC, kept up to date over snapshots.  value = (query, edge) relaxations
    of all queries per second of device time (batched: group_size 64).  The
    plain figure runs a sample of the same sources one query per edge pass
    (group_size 1) over the same snapshots."""
    import torch

    import sgs

    dev = torch.device("cuda", R.local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    e = sgs.Engine(device=R.local, weight_mode=sgs.W_EXPLICIT, group_size=a.group_size, **pers(a))
    e.load_rmat(a.batched_scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
    nv = int(e.engine_stats()["nv"])
    row, col, _ = e.export()
    nq = a.batched_bfs + a.batched_sssp
    srcs, wcc = largest_wcc_sources(nv, row, col, nq, a.seed)
    specs = [(sgs.BFS, int(x)) for x in srcs[:a.batched_bfs]] + \
            [(sgs.SSSP, int(x)) for x in srcs[a.batched_bfs:]]
    half = a.batched_updates // 2
    nb = a.warmup + a.steps + (0 if a.no_e2e else a.steps)
    i_s, i_d, d_s, d_d = sgs.gen_update_stream(nv, row, col, a.seed * 1000003, nb * half, nb * half)
    i_w = sgs.hash_weights(a.seed, i_s, i_d)
    del row, col
    batches = [tuple(x[k * half:(k + 1) * half] for x in (i_s, i_d, i_w, d_s, d_d)) for k in range(nb)]
    dev_b = {}

    def dev_of(b):
        key = id(b)
        if key not in dev_b:
            dev_b[key] = [torch.from_numpy(x.view(np.int32)).to(dev) for x in b] + [half]
        return dev_b[key]

    t_gen = time.time() - t0
    tune = e.autotune() if a.autotune else None
    # static start of all queries together
    e.synchronize()
    ts = time.perf_counter()
    qs = e.add_queries(specs)
    e.synchronize()
    static_s = time.perf_counter() - ts
    static_edges = sum(q.stats()["edges_traversed"] for q in qs)
    static_ms = sum(q.stats()["ms"] for q in qs[::a.group_size])
    # ---------------- timed snapshots
    e.kernel_timing(True)
    clocks = Clocks(R.local)
    R.barrier()
    torch.cuda.synchronize()
    l0 = e.engine_stats()["kernel_launches"]
    clocks.start()
    w0 = time.perf_counter()
    edges, dev_ms = run_snapshots(e, qs, batches, dev_of, a.warmup, a.steps)
    torch.cuda.synchronize()
    R.barrier()
    wall_ms = (time.perf_counter() - w0) * 1e3
    clk = clocks.stop()
    launches = int(e.engine_stats()["kernel_launches"] - l0)
    kst = e.kernel_stats()
    e.kernel_timing(False)
    # ---------------- e2e: pinned host batches + every query's summary read back
    e2e = None
    if not a.no_e2e:
        pinned = []
        for k in range(a.warmup + a.steps, nb):
            ps = []
            for x in batches[k]:
                t = torch.empty(len(x), dtype=torch.int32, pin_memory=True)
                t.numpy()[:] = x.view(np.int32)
                ps.append(t)
            pinned.append(ps)
        R.barrier()
        import gc
        gc.disable()  # no collector pauses inside the timed loop
        e_edges, e_ms, out_b = 0, 0.0, 0
        for ps in pinned:
            t1 = time.perf_counter()
            e.apply_batch_ptr(*(x.data_ptr() for x in ps[:3]), half, ps[3].data_ptr(), ps[4].data_ptr(),
                              half, sgs.MEM_HOST)
            sums = e.summaries(qs)  # every query's summary, one read-back
            e_ms += (time.perf_counter() - t1) * 1e3
            out_b = sums.nbytes
            e_edges += sum(q.stats()["edges_traversed"] for q in qs)
        gc.enable()
        e_ms = R.max(e_ms)
        e2e = {"value": round(R.sum(e_edges) / (e_ms * 1e6), 3), "unit": UNIT,
               "h2d_bytes_per_step": half * 5 * 4, "d2h_bytes_per_step": int(out_b),
               "ms_per_step": round(e_ms / a.steps, 2)}
    # ---------------- self check at full size: incremental == from scratch for a few lanes
    chk = {}
    for q in qs[:: max(1, nq // 4)][:4]:
        f = e.add_query(q.algo, q.source)
        chk[f"{'bfs' if q.algo == sgs.BFS else 'sssp'}:{q.source}"] = bool(
            np.array_equal(q.summary()[:3], f.summary()[:3]))
        e.remove_query(f)
    e.close()
    # ---------------- plain: a sample of the same sources, one query per pass
    plain = None
    if a.plain_sample > 0:
        k = min(a.plain_sample, nq)
        sample = specs[:k // 2] + specs[a.batched_bfs:a.batched_bfs + (k - k // 2)]
        p = sgs.Engine(device=R.local, weight_mode=sgs.W_EXPLICIT, group_size=1, **pers(a))
        p.load_rmat(a.batched_scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
        pq = p.add_queries(sample)
        pe, pms = run_snapshots(p, pq, batches, dev_of, a.warmup, a.steps)
        p.close()
        plain = {"queries": k, "gteps": round(pe / (pms * 1e6), 3),
                 "ms_per_snapshot_per_query": round(pms / a.steps / k, 3),
                 "note": "same snapshots, each query its own edge pass (group_size 1)"}
    T = R.max(dev_ms)
    value = R.sum(edges) / (T * 1e6)
    peak, peak_src = measured_peak_hbm()
    dom = max(kst, key=lambda kk: kst[kk]["ms"])
    kd = kst[dom]
    achieved = kd["bytes_alg"] / (kd["ms"] * 1e-3) / 1e9 if kd["ms"] > 0 else 0.0
    roof = {"bound": "hbm", "kernel": f"wide_map ({dom})" if dom.startswith("wide") else dom,
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_source": peak_src, "traffic": None, "launches": kd["launches"],
            "avg_launch_ms": round(kd["ms"] / max(kd["launches"], 1), 4),
            "alg_bytes_per_launch": kd["bytes_alg"] / max(kd["launches"], 1),
            # the bytes count the (lane, edge) pairs the kernel evaluates: a
            # repair's first round walks every reached vertex's out-edges but
            # evaluates only the lanes reset at each destination, so its time
            # goes to the walk (4-B ids, 8-B reset-lane probes of the L2), which
            # this model counts at 4 B per slot
            "slots_walked_per_s": round(kd["slots"] / (kd["ms"] * 1e-3), 1) if kd["ms"] > 0 else None,
            "pairs_evaluated": int(max(0.0, (kd["bytes_alg"] - 4.0 * kd["slots"] - 20.0 * kd["entries"]) / 8.0))}
    out = {
        "metric": BATCHED_METRIC.format(nb=a.batched_bfs, ns=a.batched_sssp, scale=a.batched_scale,
                                        upd=a.batched_updates),
        "value": round(value, 3), "unit": UNIT, "n_gpus": R.world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": round(T / a.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (device R-MAT, seeded weights and update stream; sources from the largest WCC)",
        "config": {"workload": f"{a.batched_bfs} BFS + {a.batched_sssp} SSSP queries, R-MAT scale "
                               f"{a.batched_scale} ef {a.edge_factor} seed {a.seed}, {a.batched_updates} "
                               f"updates/snapshot (50/50), group_size {a.group_size}",
                   "nv": nv, "largest_wcc": int(wcc), "autotune": tune, "persistent": a.persistent,
                   "l2": "inputs larger than L2 (per-group state %.1f GB)" % (nv * 64 * 12 / 1e9),
                   "parallelism": "replicas" if R.world > 1 else "single GPU"},
        "e2e": e2e, "gpu_launches": launches, "roofline": roof, "clocks": clk,
        "wall_ms_timed": round(wall_ms, 2),
        "static_start": {"queries": nq, "gteps": round(static_edges / (static_ms * 1e6), 3),
                         "device_ms": round(static_ms, 2), "wall_s": round(static_s, 3)},
        "plain": plain, "selfcheck_incremental_eq_static": chk, "gen_s": round(t_gen, 2),
        "kernel_stats": {kk: {k2: (round(v2, 4) if isinstance(v2, float) else v2) for k2, v2 in v.items()}
                         for kk, v in kst.items()},
    }
    return out


# ----------------------------------------------------------------- served arm
SERVED_METRIC = ("GTEPS served (R-MAT s{scale}, {budget} GB HBM budget, Poisson {rate}/s: update "
                 "batches log-uniform 1k-1M and PR/BFS/SSSP queries)")


def served_trace(nv, row, col, a):
    """Poisson arrivals over --served-seconds: half update batches (size
    log-uniform in [1k, 1M], half inserts of new edges, half deletes of
    existing ones, from the seeded stream generator), half one-shot queries
    (2 % PR, 49 % BFS, 49 % SSSP) from uniform random sources.  A PageRank
    from scratch at scale 26 needs about 200 full passes to guarantee
    L-inf <= 1e-6, several seconds, hence the small share."""
    import sgs

    rng = np.random.default_rng(a.seed + 26)
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / a.served_rate)
        if t > a.served_seconds:
            break
        arrivals.append(t)
    kinds = rng.random(len(arrivals)) < 0.5
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(1e6), len(arrivals))).astype(np.int64)
    n_upd = int(kinds.sum())
    half = [int(x) // 2 for x in sizes[kinds]]
    tot = int(sum(half))
    i_s, i_d, d_s, d_d = sgs.gen_update_stream(nv, row, col, a.seed * 7919, tot, tot)
    i_w = sgs.hash_weights(a.seed, i_s, i_d)
    reqs, off, u = [], 0, 0
    for k, t in enumerate(arrivals):
        if kinds[k]:
            h = half[u]
            sl = slice(off, off + h)
            off += h
            u += 1
            reqs.append({"kind": "update", "arrival_s": t, "ins_src": i_s[sl], "ins_dst": i_d[sl],
                         "ins_w": i_w[sl], "del_src": d_s[sl], "del_dst": d_d[sl]})
        else:
            x = rng.random()
            algo = sgs.PR if x < 0.02 else sgs.BFS if x < 0.51 else sgs.SSSP
            reqs.append({"kind": "query", "algo": algo, "source": int(rng.integers(0, nv)), "arrival_s": t})
    return reqs, n_upd


def served_arm(a, R):
    """N2: a served loop (sgs_serve) on one GPU: requests arrive on the wall
    clock, updates are applied in order, queries are admitted together up to
    --slots per step.  value = edges traversed by all requests / busy time of
    the loop (host wall clock, host->device copies of the batches and the
    result reads included), with p50/p99 latency per request kind."""
    import torch

    import sgs

    dev = torch.device("cuda", R.local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    e = sgs.Engine(device=R.local, weight_mode=sgs.W_EXPLICIT, hbm_budget_gb=a.served_budget_gb,
                   group_size=a.served_group_size, serve_restarts=a.serve_restarts)
    e.load_rmat(a.served_scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
    st0 = e.engine_stats()
    nv = int(st0["nv"])
    row, col, _ = e.export()
    reqs, n_upd = served_trace(nv, row, col, a)
    del row, col
    t_gen = time.time() - t0
    # warm-up: a few requests of each kind outside the trace
    warm = [{"kind": "query", "algo": alg, "source": 1, "arrival_s": 0.0} for alg in (sgs.BFS, sgs.SSSP, sgs.PR)]
    e.serve(warm, slots=a.slots, realtime=False)
    clocks = Clocks(R.local)
    R.barrier()
    torch.cuda.synchronize()
    l0 = e.engine_stats()["kernel_launches"]
    e.kernel_timing(True)
    clocks.start()
    w0 = time.perf_counter()
    res = e.serve(reqs, slots=a.slots, realtime=True)
    wall = time.perf_counter() - w0
    clk = clocks.stop()
    kst = e.kernel_stats()
    e.kernel_timing(False)
    launches = int(e.engine_stats()["kernel_launches"] - l0)
    st = e.engine_stats()
    # roofline of the kernel class with the most timed device time (the
    # flight's round launches are not timed per launch; updates' repairs and
    # the PageRank job's sweeps are)
    roof = None
    timed = {k: v for k, v in kst.items() if v["ms"] > 0}
    if timed:
        dom = max(timed, key=lambda k: timed[k]["ms"])
        kd = timed[dom]
        peak, src = measured_peak_hbm()
        ach = kd["bytes_alg"] / (kd["ms"] * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "peak_source": src, "traffic": None,
                "launches": kd["launches"], "avg_launch_ms": round(kd["ms"] / max(kd["launches"], 1), 4)}
    e.close()
    plain = served_plain(a, R, reqs) if a.served_plain else None
    ok = [c["status"] == 0 for c in res]
    # busy time: union of the steps' [start, done] intervals
    steps = sorted({(c["start_s"], c["done_s"]) for c in res})
    busy, last = 0.0, -1.0
    for s0, s1 in steps:
        s0 = max(s0, last)
        if s1 > s0:
            busy += s1 - s0
        last = max(last, s1)
    edges = sum(c["edges"] for c in res)

    def pct(kind, algo=None):
        lat = [c["latency_s"] * 1e3 for c, r in zip(res, reqs)
               if r["kind"] == kind and (algo is None or r.get("algo") == algo)]
        if not lat:
            return None
        return {"n": len(lat), "p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2), "max_ms": round(max(lat), 2)}

    qb = [c["batch"] for c, r in zip(res, reqs) if r["kind"] == "query"]
    value = edges / busy / 1e9 if busy > 0 else 0.0
    h2d = sum((len(r["ins_src"]) * 3 + len(r["del_src"]) * 2) * 4 for r in reqs if r["kind"] == "update")
    out = {
        "metric": SERVED_METRIC.format(scale=a.served_scale, budget=a.served_budget_gb, rate=a.served_rate),
        "value": round(R.sum(value), 3), "unit": UNIT, "n_gpus": R.world, "steps": len(reqs),
        "warmup": len(warm), "ms_per_step": round(busy * 1e3 / max(len(reqs), 1), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (device R-MAT, seeded update stream, Poisson arrivals)",
        "config": {"workload": f"served loop, R-MAT scale {a.served_scale} ef {a.edge_factor} seed {a.seed}, "
                               f"HBM budget {a.served_budget_gb} GB, {a.served_seconds} s of Poisson "
                               f"arrivals at {a.served_rate}/s, slots {a.slots}, "
                               f"group_size {a.served_group_size}",
                   "nv": nv, "ne_initial": int(st0["ne"]), "ne_final": int(st["ne"]),
                   "hbm_resident_fraction": st["hbm_resident_vertices"] / max(nv, 1),
                   "requests": len(reqs), "updates": n_upd, "queries": len(reqs) - n_upd,
                   "parallelism": "replicas" if R.world > 1 else "single GPU"},
        "latency": {"update": pct("update"), "query": pct("query"), "bfs": pct("query", sgs.BFS),
                    "sssp": pct("query", sgs.SSSP), "pr": pct("query", sgs.PR)},
        "lanes_in_flight_at_admission": {"mean": round(float(np.mean(qb)), 2) if qb else 0,
                                         "max": int(max(qb)) if qb else 0},
        "restarts": {"allowed_per_query": a.serve_restarts,
                     "queries_restarted": int(sum(1 for c in res if c["restarts"])),
                     "total": int(sum(c["restarts"] for c in res))},
        "failed": int(len(res) - sum(ok)),
        "busy_s": round(busy, 3), "wall_s": round(wall, 3), "utilisation": round(busy / wall, 3),
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d / max(len(reqs), 1)),
                "d2h_bytes_per_step": 32, "note": "the served loop is end to end: host batches in, "
                                                  "summaries out, wall clock"},
        "gpu_launches": launches, "clocks": clk, "gen_s": round(t_gen, 2),
        "roofline": roof,
        "plain": plain,
    }
    return out


def served_plain(a, R, reqs):
    """The plain per-query engine on the same graph and request mix: a sample
    of the trace's BFS and SSSP queries, each alone (group_size 1, one query
    per edge pass) from scratch on the initial graph, plus one PageRank from
    scratch; the mix's GTEPS weights them by the trace's composition (its
    BFS/SSSP and PageRank counts): total edges / total device time."""
    import sgs

    e = sgs.Engine(device=R.local, weight_mode=sgs.W_EXPLICIT, hbm_budget_gb=a.served_budget_gb,
                   group_size=1, pr_warm=0)
    e.load_rmat(a.served_scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
    lane = [r for r in reqs if r["kind"] == "query" and r["algo"] in (sgs.BFS, sgs.SSSP)]
    n_pr = sum(1 for r in reqs if r["kind"] == "query" and r["algo"] == sgs.PR)
    qs = lane[:a.served_plain]
    e.remove_query(e.add_query(qs[0]["algo"], qs[0]["source"]))  # warm-up
    edges, ms = 0, 0.0
    for r in qs:
        q = e.add_query(r["algo"], r["source"])
        st = q.stats()
        edges += st["edges_traversed"]
        ms += st["ms"]
        e.remove_query(q)
    pr_e = pr_ms = 0.0
    if n_pr:
        q = e.add_query(sgs.PR, 0)
        st = q.stats()
        pr_e, pr_ms = float(st["edges_traversed"]), float(st["ms"])
        e.remove_query(q)
    e.close()
    k = len(qs)
    lane_e, lane_ms = edges / max(k, 1), ms / max(k, 1)
    mix_e = len(lane) * lane_e + n_pr * pr_e
    mix_ms = len(lane) * lane_ms + n_pr * pr_ms
    return {"queries_timed": k, "bfs_sssp_gteps": round(edges / (ms * 1e6), 3) if ms > 0 else None,
            "bfs_sssp_ms_per_query": round(lane_ms, 3),
            "pagerank_ms": round(pr_ms, 1) if n_pr else None,
            "gteps": round(mix_e / (mix_ms * 1e6), 3) if mix_ms > 0 else None,
            "note": "plain engine (group_size 1, each query alone, from scratch) on the initial graph, "
                    "weighted by the trace's %d BFS/SSSP and %d PageRank queries" % (len(lane), n_pr)}


# ----------------------------------------------------------------- PPR adjoint arm
PPR_METRIC = ("PPR forward+adjoint relaxations/s (weighted personalized PageRank, R-MAT s{scale}, "
              "{K} vectors x {seeds} seeds, loss on {targets} targets)")
PPR_UNIT = "G edge-vector relaxations/s"


def ppr_inputs(nv, ne, a):
    """Seeded synthetic inputs: fp32 weights log-uniform in [0.1, 10] (the
    row normalisation happens inside P), K teleport vectors with mass 1/seeds
    on `seeds` random vertices each, and `targets` random target vertices
    (loss = sum of all K scores over the targets, so dL/dX = 1 on their rows)."""
    rng = np.random.default_rng(a.seed)
    w32 = np.exp(rng.uniform(np.log(0.1), np.log(10.0), ne)).astype(np.float32)
    K = a.ppr_vectors
    T = np.zeros((nv, K), np.float32)
    for k in range(K):
        T[rng.choice(nv, a.ppr_seeds, replace=False), k] = 1.0 / a.ppr_seeds
    targets = np.sort(rng.choice(nv, a.ppr_targets, replace=False)).astype(np.int64)
    return w32, T, targets


def ppr_arm(a, R):
    """One step = forward solve of all K vectors + adjoint solve + per-edge and
    teleport gradients, through the C ABI on device-resident FP64 inputs;
    device time from the library's CUDA events.  e2e: the torch op
    (sgs.autograd.personalized_pagerank) from pinned host fp32 inputs to the
    loss and dL/dw back on the host."""
    import torch

    import sgs
    from sgs.autograd import personalized_pagerank

    dev = torch.device("cuda", R.local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    e = sgs.Engine(device=R.local, weight_mode=sgs.W_UNIT)
    e.load_rmat(a.ppr_scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
    g = sgs.Ppr(engine=e)
    e.close()
    nv, ne, K = g.nv, g.ne, a.ppr_vectors
    w32, T32, targets = ppr_inputs(nv, ne, a)
    t_gen = time.time() - t0
    w = torch.from_numpy(w32).to(dev).double()
    T = torch.from_numpy(T32).to(dev).double()
    G = torch.zeros(nv, K, dtype=torch.float64, device=dev)
    G[torch.from_numpy(targets).to(dev)] = 1.0
    tol = 1e-10 * nv * K

    def step():
        X = g.forward(w, T, tol=tol)
        sf = g.stats()
        gw, gT = g.backward(w, X, G, tol=tol)
        sb = g.stats()
        return sf, sb

    for _ in range(a.warmup):
        step()
    g.timing(True)
    clocks = Clocks(R.local)
    R.barrier()
    torch.cuda.synchronize()
    clocks.start()
    w0 = time.perf_counter()
    dev_ms, steps_ms, relax, nbytes, nsteps, it_f, it_b = 0.0, 0.0, 0, 0.0, 0, 0, 0
    l0 = g.stats()["kernel_launches"]
    for _ in range(a.steps):
        sf, sb = step()
        dev_ms += sf["ms"] + sb["ms"]
        steps_ms += sf["steps_ms"] + sb["steps_ms"]
        nsteps += sf["iters"] + sb["iters"]
        it_f, it_b = sf["iters"], sb["iters"]
        relax += ne * K * (sf["iters"] + sb["iters"])
        nbytes += sf["bytes_alg_step"] * sf["iters"] + sb["bytes_alg_step"] * sb["iters"]
    torch.cuda.synchronize()
    R.barrier()
    wall_ms = (time.perf_counter() - w0) * 1e3
    clk = clocks.stop()
    launches = int(g.stats()["kernel_launches"] - l0)
    g.timing(False)
    st = g.stats()
    T_ms = R.max(dev_ms)
    value = R.sum(relax) / (T_ms * 1e6)
    peak, peak_src = measured_peak_hbm()
    achieved = nbytes / (steps_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": "k_ppr_step (+ k_ppr_finalize for hub pieces)",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_src, "traffic": None,
            "launches": nsteps, "avg_launch_ms": round(steps_ms / nsteps, 4),
            "alg_bytes_per_launch": sf["bytes_alg_step"]}
    # ---------------- e2e through the torch op from pinned host memory
    e2e = None
    if not a.no_e2e:
        wp = torch.from_numpy(w32).pin_memory()
        Tp = torch.from_numpy(T32).pin_memory()
        tp = torch.from_numpy(targets).pin_memory()
        R.barrier()
        torch.cuda.synchronize()
        e_ms, d2h = 0.0, 0
        for _ in range(a.steps):
            t1 = time.perf_counter()
            wd = wp.to(dev, non_blocking=True).requires_grad_(True)
            Td = Tp.to(dev, non_blocking=True)
            td = tp.to(dev, non_blocking=True)
            X = personalized_pagerank(g, wd, Td, tol=tol)
            loss = X[td].sum()
            loss.backward()
            lh = loss.detach().cpu()
            gh = wd.grad.cpu()
            e_ms += (time.perf_counter() - t1) * 1e3
            d2h = lh.numel() * lh.element_size() + gh.numel() * gh.element_size()
            del X, loss, wd
        e_ms = R.max(e_ms)
        e2e = {"value": round(R.sum(relax) / (e_ms * 1e6), 3), "unit": PPR_UNIT,
               "h2d_bytes_per_step": int(w32.nbytes + T32.nbytes + targets.nbytes),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e_ms / a.steps, 2),
               "path": "sgs.autograd.personalized_pagerank forward + loss.backward()"}
    out = {
        "metric": PPR_METRIC.format(scale=a.ppr_scale, K=K, seeds=a.ppr_seeds, targets=a.ppr_targets),
        "value": round(value, 3), "unit": PPR_UNIT, "n_gpus": R.world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(T_ms / a.steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (device R-MAT; seeded fp32 log-uniform weights, teleport seeds, targets)",
        "config": {"workload": f"PPR forward + adjoint, R-MAT scale {a.ppr_scale} ef {a.edge_factor} "
                               f"seed {a.seed}, {K} vectors x {a.ppr_seeds} seeds, {a.ppr_targets} targets, "
                               f"alpha 0.85, stop at L1 step change < {tol:.3g}",
                   "nv": nv, "ne": ne, "iters_forward": it_f, "iters_adjoint": it_b,
                   "hub_pieces_csc": st["pieces_in"], "hub_pieces_csr": st["pieces_out"],
                   "l2": "inputs larger than L2 (state %.1f GB vs %d MB L2)" % (
                       nv * K * 8 / 1e9, L2_BYTES // 2**20),
                   "parallelism": "replicas" if R.world > 1 else "single GPU"},
        "e2e": e2e, "gpu_launches": launches, "roofline": roof, "clocks": clk,
        "wall_ms_timed": round(wall_ms, 2), "gen_s": round(t_gen, 2),
    }
    if R.rank == 0 and R.world == 1 and not a.no_cpu:
        out["cpu_baseline"] = ppr_cpu_baseline(g, w32, T32, a)
    g.close()
    return out


def ppr_cpu_baseline(g, w32, T32, a):
    """The same Jacobi step on the host (scipy CSR times the [nv, K] state,
    single thread), a bounded number of steps; relaxations/s."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ppr_dense as D

    row, col = g.export()
    nv, ne, K = g.nv, g.ne, T32.shape[1]
    PT = D.sparse_pt(nv, row, col, w32.astype(np.float64))
    t = time.perf_counter()
    X, k = D.ppr_jacobi_sparse(nv, row, col, None, T32, iters=1, PT=PT)
    dt = time.perf_counter() - t
    more = int(a.cpu_seconds / max(dt, 1e-3)) - 1
    if more > 0:
        t = time.perf_counter()
        _, k2 = D.ppr_jacobi_sparse(nv, row, col, None, T32, iters=min(more, 20), X0=X, PT=PT)
        dt += time.perf_counter() - t
        k += k2
    return {"value": round(ne * K * k / dt / 1e9, 4), "unit": PPR_UNIT, "cores": 1, "kind": "port",
            "sample": f"{k} Jacobi steps of the forward solve (all {K} vectors) on the same graph, "
                      "scipy CSR times the dense state on one thread (matrix build not timed)"}


# ----------------------------------------------------------------- reference arm
class _quiet_stdout:
    """Sends file descriptor 1 to /dev/null for the duration (native code
    that prints would otherwise mix with the JSON line)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


def snapshot_config(a, nv, ne0):
    """The `config` of the snapshot workload, identical in both arms (the
    engine's own settings go under `engine` in its line)."""
    return {"workload": f"incremental SSSP/BFS/CC, R-MAT scale {a.scale} ef {a.edge_factor} seed {a.seed}, "
                        f"{a.updates} updates/snapshot (50/50), source 0, HBM budget {a.budget_gb} GB"
                        + (f" ({a.cache_gb} GB of it as edge cache)" if a.cache_gb > 0 else "")
                        + (", vertex ids randomly permuted" if getattr(a, "permute", False) else ""),
            "nv": int(nv), "ne_initial": int(ne0),
            "queries": ["sssp:0", "bfs:0", "cc"],
            "l2": "inputs larger than L2 (the edge arena and the per-vertex state exceed the 126 MB L2)"}


def reference_arm(a, R):
    """The reference's own CPU path for one snapshot, on the host cores.

    The reference computes its snapshots on the GPU; its CPU path is the
    serial host PMA update plus the samples' serial host oracles.  One step =
    one snapshot of the same update stream as the engine arm:

    * the batch applied to the reference's host::PMAGraph with its own
      insert / del_edge, inserts then deletes (include/groute/graphs/
      csr_graph.cuh:658-811, through oracle/_ref), one thread;
    * then, concurrently on three host threads, SSSPHostNaive from source 0
      (samples/hybrid_sssp/hybrid_sssp_host.cu:35-63), BFSHost from source 0
      (samples/hybrid_bfs/hybrid_bfs_host.cpp:33-60) -- both compiled from
      the reference sources -- and the directed min-label CC (the reference
      ships no CC host code; the oracle's restatement of hybrid_cc.cu:96-110).

    Traversed edges per query = out-edges of the vertices it reached (CC: all
    edges), the count the engine arm uses for one pass.  The host oracles
    read a CSR, so the updated PMA is exported into one between the apply
    and the traversals (not timed).  Every step applies its batch (timed);
    the traversals run on the timed steps until --ref-seconds of traversal
    time is spent, and GTEPS = their edges / (their time + the mean apply
    time per step for each of them).  SSSPHostNaive synthesizes its weights
    ((u+v)%128), where the engine arm stores weights uniform in [1,64]: the
    same graph and the same per-edge work, different weight values."""
    if R.rank != 0:
        return None
    import threading as _th

    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O

    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True,
            "n_gpus": R.world, "steps": a.steps, "warmup": a.warmup}
    if O.ref_lib() is None:
        base["unavailable"] = "oracle/_ref (the reference's host code) was not built"
        return base
    t0 = time.time()
    nv, row, col = O.rmat_csr_par(a.scale, a.edge_factor, a.seed)
    ne0 = len(col)
    half = a.updates // 2
    nb = a.warmup + a.steps
    i_s, i_d, d_s, d_d = O.gen_updates(nv, row, col, a.seed * 1000003, nb * half, nb * half)
    with _quiet_stdout():  # the reference's PMA Bind prints diagnostics to stdout
        pma = O.RefPMA(nv, row, col)
    del row, col
    setup_s = time.time() - t0
    apply_s, trav_s, trav_edges, step_ms = [], 0.0, 0, []
    parts = {"sssp": 0.0, "bfs": 0.0, "cc": 0.0}
    n_trav = 0
    for k in range(nb):
        s = slice(k * half, (k + 1) * half)
        t1 = time.perf_counter()
        pma.apply(i_s[s], i_d[s], d_s[s], d_d[s])
        ta = time.perf_counter() - t1
        if k < a.warmup:
            continue
        apply_s.append(ta)
        if trav_s >= a.ref_seconds:
            continue
        prow, pcol = pma.export()
        g = O.RefGraph(nv, prow, pcol)
        deg = np.diff(prow)
        outs = {"sssp": np.empty(nv, np.uint32), "bfs": np.empty(nv, np.uint32)}
        took = {}

        def timed(name, fn):
            t = time.perf_counter()
            fn()
            took[name] = time.perf_counter() - t

        ths = [_th.Thread(target=timed, args=("sssp", lambda: g.sssp(0, outs["sssp"]))),
               _th.Thread(target=timed, args=("bfs", lambda: g.bfs(0, outs["bfs"]))),
               _th.Thread(target=timed, args=("cc", lambda: O.cc(nv, prow, pcol)))]
        t2 = time.perf_counter()
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        tt = time.perf_counter() - t2
        g.close()
        edges = int(deg[outs["sssp"] != O.INF].sum()) + int(deg[outs["bfs"] != O.INF].sum()) + int(len(pcol))
        trav_s += tt
        trav_edges += edges
        n_trav += 1
        for n in parts:
            parts[n] += took[n]
        step_ms.append((ta + tt) * 1e3)
    mean_apply = statistics.mean(apply_s)
    value = trav_edges / (trav_s + mean_apply * n_trav) / 1e9
    base.update({
        "value": round(value, 4), "ms_per_step": round(statistics.mean(step_ms), 2),
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (CPU R-MAT and update stream, same graph and stream as the engine arm)",
        "config": snapshot_config(a, nv, ne0),
        "reference_steps": {"applied": len(apply_s), "traversed": n_trav,
                            "apply_ms_mean": round(mean_apply * 1e3, 1),
                            "traversal_ms_mean": round(trav_s / max(n_trav, 1) * 1e3, 1),
                            "per_query_ms_mean": {n: round(v / max(n_trav, 1) * 1e3, 1)
                                                  for n, v in parts.items()},
                            "edges_per_snapshot": round(trav_edges / max(n_trav, 1)),
                            "setup_s": round(setup_s, 1)},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": 3, "kind": "reference",
                         "sample": "per snapshot: the batch applied with the reference's host PMA "
                                   "insert/del_edge (1 thread), then SSSPHostNaive(0) and BFSHost(0) "
                                   "(reference code) and the directed CC restatement concurrently on 3 "
                                   "threads, on %d of the %d timed snapshots (traversal budget %.0f s); "
                                   "every snapshot's apply timed" % (n_trav, a.steps, a.ref_seconds)},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    pma.close()
    return base


def _basic_line(a, R, metric, value, ms, cfg, extra):
    out = {"metric": metric, "value": round(value, 3), "unit": UNIT, "n_gpus": R.world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (device R-MAT)",
           "config": cfg}
    out.update(extra)
    return out


def pagerank_arm(a, R):
    """Plain incremental PageRank (by default R-MAT scale 16 with 10k + 10k
    updates per snapshot): R-MAT scale --pr-scale, snapshots of --pr-updates
    updates (50/50); one step =
    one snapshot (cancel + compensate + sweeps to the L1 tolerance).  value =
    edges traversed (active vertices' out-degrees summed over rounds) per
    second of device time; the static start is reported beside it."""
    import torch

    import sgs

    dev = torch.device("cuda", R.local)
    torch.cuda.set_device(dev)
    e = sgs.Engine(device=R.local, weight_mode=sgs.W_EXPLICIT, **pers(a))
    e.load_rmat(a.pr_scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
    nv = int(e.engine_stats()["nv"])
    row, col, _ = e.export()
    half = a.pr_updates // 2
    nb = a.warmup + a.steps
    i_s, i_d, d_s, d_d = sgs.gen_update_stream(nv, row, col, a.seed * 1000003, nb * half, nb * half)
    i_w = sgs.hash_weights(a.seed, i_s, i_d)
    del row, col
    e.kernel_timing(True)
    q = e.add_query(sgs.PR)
    st0 = q.stats()
    kinds0 = e.kernel_stats()
    edges, ms = 0, 0.0
    clocks = Clocks(R.local)
    for k in range(nb):
        if k == a.warmup:
            torch.cuda.synchronize()
            clocks.start()
        sl = slice(k * half, (k + 1) * half)
        e.apply_batch(i_s[sl], i_d[sl], i_w[sl], d_s[sl], d_d[sl])
        if k >= a.warmup:
            edges += q.stats()["edges_traversed"]
            ms += e.engine_stats()["last_batch_ms"]
    clk = clocks.stop()
    ks = e.kernel_stats()
    sweep = "pr_pull" if ks["pr_pull"]["launches"] > kinds0["pr_pull"]["launches"] else "pr_push"
    kd = {k: ks[sweep][k] - kinds0[sweep][k] for k in ("launches", "slots", "bytes_alg", "ms")}
    peak, src = measured_peak_hbm()
    ach = kd["bytes_alg"] / (kd["ms"] * 1e-3) / 1e9 if kd["ms"] > 0 else 0.0
    T = R.max(ms)
    st = e.engine_stats()
    e.close()
    return _basic_line(
        a, R, f"GTEPS per snapshot (incremental PageRank, R-MAT s{a.pr_scale}, {a.pr_updates} updates/snapshot)",
        R.sum(edges) / (T * 1e6), T / a.steps,
        {"workload": f"incremental PageRank, R-MAT scale {a.pr_scale} ef {a.edge_factor} seed {a.seed}, "
                     f"{a.pr_updates} updates/snapshot (50/50), alpha 0.85, L1 tolerance of the library",
         "pull": a.pull, "sweep_kernel": sweep, "in_store_bytes": int(st["in_store_bytes"]),
         "l2": "graph L2-resident at scale 16" if a.pr_scale <= 18 else "graph larger than L2"},
        {"static": {"ms": round(st0["ms"], 3), "rounds": st0["rounds"],
                    "gteps": round(st0["edges_traversed"] / (st0["ms"] * 1e6), 3) if st0["ms"] else None},
         "sweep": {"launches": kd["launches"], "ms": round(kd["ms"], 3), "achieved_gbs": round(ach, 1),
                   "frac_of_measured_hbm": round(ach / peak, 4), "peak_source": src},
         "roofline": {"bound": "hbm", "kernel": sweep, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                      "frac": round(ach / peak, 4), "peak_source": src, "traffic": None,
                      "launches": kd["launches"],
                      "note": "graph L2-resident at this scale: the HBM fraction is not a bound"
                              if a.pr_scale <= 18 else None},
         "clocks": clk})


def bfs_arm(a, R):
    """Static BFS from scratch (the hybrid_bfs sample's Start): R-MAT scale
    --scale, --bfs-sources sources (vertex 0 and seeded random ones), each
    one query in its own group; value = traversed edges (frontier
    out-degrees summed over rounds, the reference's count) per second of
    device time.  With --pull 3 the large middle rounds run bottom-up."""
    import torch

    import sgs

    dev = torch.device("cuda", R.local)
    torch.cuda.set_device(dev)
    e = sgs.Engine(device=R.local, weight_mode=sgs.W_EXPLICIT, group_size=1, **pers(a))
    e.load_rmat(a.scale, a.edge_factor, a.seed, 0.57, 0.19, 0.19, wseed=a.seed)
    nv = int(e.engine_stats()["nv"])
    rng = np.random.default_rng(a.seed)
    srcs = [0] + [int(x) for x in rng.integers(0, nv, a.bfs_sources - 1)]
    for s_ in srcs[:a.warmup]:  # warm-up starts (and the in-edge store, if used)
        e.remove_query(e.add_query(sgs.BFS, s_))
    clocks = Clocks(R.local)
    torch.cuda.synchronize()
    clocks.start()
    edges, ms, reached = 0, 0.0, []
    for s_ in srcs:
        q = e.add_query(sgs.BFS, s_)
        st = q.stats()
        edges += st["edges_traversed"]
        ms += st["ms"]
        reached.append(int(q.summary()[0]))
        e.remove_query(q)
    clk = clocks.stop()
    est = e.engine_stats()
    e.close()
    T = R.max(ms)
    return _basic_line(
        a, R, f"GTEPS (static BFS from scratch, R-MAT s{a.scale})", R.sum(edges) / (T * 1e6),
        T / len(srcs),
        {"workload": f"static BFS, R-MAT scale {a.scale} ef {a.edge_factor} seed {a.seed}, "
                     f"{len(srcs)} sources (0 and seeded random)", "pull": a.pull,
         "reached": reached},
        {"steps": len(srcs), "bottom_up_rounds": int(est["bfs_bottom_up_rounds"]),
         "in_store_bytes": int(est["in_store_bytes"]), "clocks": clk})


def _condense(out):
    """The figures of a workload's line kept in the headline's sub-record."""
    keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "roofline", "clocks", "gpu_launches",
            "latency", "plain", "utilisation", "lanes_in_flight_at_admission", "restarts", "static", "sweep",
            "selfcheck_incremental_eq_static", "static_start", "failed", "grad_check")
    rec = {k: out[k] for k in keep if k in out}
    cfg = out.get("config") or {}
    rec["workload"] = cfg.get("workload")
    e2e = out.get("e2e")
    if isinstance(e2e, dict):
        rec["e2e"] = {k: e2e[k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step",
                                          "ms_per_step") if k in e2e}
    eng = out.get("engine") or {}
    for k in ("hbm_resident_fraction", "arena_bytes_host", "repair"):
        if k in eng:
            rec[k] = eng[k]
    if isinstance(rec.get("roofline"), dict):
        rec["roofline"] = {k: v for k, v in rec["roofline"].items() if not isinstance(v, (dict, list))
                           or k == "largest_launch"}
    return rec


def config_records(a, R):
    """The benchmark's other configurations, each run after the headline in
    its own engine (with its own clocks and roofline) and kept as a
    sub-record of the one JSON line: the first (incremental PageRank, R-MAT
    s16, 2 snapshots of 10k inserts + 10k deletes), the headline's
    out-of-HBM regime (0.5 GB budget: most blocks host-resident) and its
    work-efficient pull repair, the batched third (256 BFS + 256 SSSP at
    s22), the fourth (PPR adjoint at s22, K = 64) and the served fifth (s26,
    16 GB budget, Poisson arrivals), each at its own default sizes."""
    import copy

    recs = {}

    def sub(name, fn, **kw):
        b = copy.copy(a)
        for k, v in kw.items():
            setattr(b, k, v)
        t = time.time()
        try:
            rec = _condense(fn(b, R))
        except Exception as ex:  # a failing sub-workload is reported, not fatal
            rec = {"error": repr(ex)[:400]}
        rec["wall_s"] = round(time.time() - t, 1)
        recs[name] = rec

    base = dict(no_e2e=True, no_cpu=True, autotune=False)
    sub("pagerank_cfg1", pagerank_arm, steps=2, warmup=1, pr_scale=16, pr_updates=20_000, workload="pagerank")
    sub("out_of_hbm_cfg2", engine_arm, budget_gb=0.5, steps=5, warmup=2, **base)
    sub("repair1_cfg2", engine_arm, repair=1, steps=10, warmup=3, **base)
    sub("batched_cfg3", batched_arm, steps=4, warmup=1, no_e2e=True, workload="batched")
    sub("ppr_cfg4", ppr_arm, steps=2, warmup=1, no_e2e=True, no_cpu=True, workload="ppr")
    sub("served_cfg5", served_arm, served_seconds=15.0, workload="served")
    return recs


def main():
    a = parse()
    R = Ranks()
    try:
        if a.impl == "reference" and a.workload == "served":
            out = None if R.rank else {
                "impl": "reference", "unavailable": "the reference has no request loop (its drivers "
                "run one source through a fixed snapshot list)"}
        elif a.impl == "reference" and a.workload == "ppr":
            out = None if R.rank else {
                "impl": "reference", "unavailable": "the reference has no personalized PageRank "
                "or adjoint (its PageRank is the single unweighted vector of the snapshot workload)"}
        elif a.impl == "reference":
            if a.workload == "batched":
                a.scale, a.updates = a.batched_scale, a.batched_updates
            out = reference_arm(a, R)
        elif a.workload == "ppr":
            out = ppr_arm(a, R)
        elif a.workload == "batched":
            out = batched_arm(a, R)
        elif a.workload == "served":
            out = served_arm(a, R)
        elif a.workload == "pagerank":
            out = pagerank_arm(a, R)
        elif a.workload == "bfs":
            out = bfs_arm(a, R)
        else:
            out = engine_arm(a, R)
            if R.world == 1 and not a.no_configs:
                out["configs"] = config_records(a, R)
        if R.rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        R.close()


if __name__ == "__main__":
    main()
