#!/usr/bin/env python
"""Benchmark of the compact-hashing neighbour search on B200.

Workload (one step = one full search, structure build included): 1,048,576 float32 points
uniform in [-1,1]^3 (torch.manual_seed(0)), non-periodic, per-point support
h_i = h0*U(0.9,1.1) with h0 = cbrt(3*50*dx^3/(4*pi)), dx = 2/102 (about 50 neighbours),
symmetric mode, CSR output -- 51,798,992 pairs per step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line.  `value` is pairs/s with inputs resident in HBM and L2 flushed (a 256 MiB
write) between timed steps, each step one whole search (build + count + emit) recorded once as a
CUDA graph and replayed, timed with CUDA events on the launching stream (max over ranks under
torchrun; every rank runs an independent replica, "replicas only").  `e2e` is the same metric
through the public radiusSearch with the inputs copied from pinned host memory and the whole CSR
result copied back every step.  `roofline` covers the dominant kernel (the count walk, timed live
inside the replays), `search_roofline` the whole search, `cpu_baseline` the reference's own CPU
operators on this host.  `batched`, `graphs` and `served` measure the other forms: 256 clouds per
launch against the per-call loop, graph replay against the eager API, and a request trace served
with continuous batching against per-call searches.  `adaptive` compares the multi-level search
with single-level cells on variable supports; `scatter` times the per-particle scatter_sum over
the neighbour list against its HBM roofline.
"""
import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "neighbor pairs/s, 3D 1M pts; batched/served vs per-call; p50/p99 ms"
WORKLOAD = "3d_1m_uniform_symmetric_csr"
N_POINTS = 1 << 20
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form measurement")
    ap.add_argument("--details", default="bench_details.json",
                    help="file that receives the full measurement (the printed line keeps a summary of each form)")
    ap.add_argument("--profile-searches", type=int, default=0,
                    help="only run this many eager searches of the workload (a small case for ncu captures)")
    ap.add_argument("--profile-scatter", type=int, default=0,
                    help="only search the workload once and run this many scatter_sum calls over its neighbour list")
    ap.add_argument("--profile-f64", type=int, default=0,
                    help="only run this many float64 searches of the workload (a small case for ncu captures)")
    return ap.parse_args()


def make_workload():
    import numpy as np
    import torch
    torch.manual_seed(0)
    pos = torch.rand(N_POINTS, 3) * 2 - 1
    dx = 2 / 102
    h0 = (3 * 50 * dx ** 3 / (4 * np.pi)) ** (1 / 3)
    sup = h0 * (0.9 + 0.2 * torch.rand(N_POINTS))
    return pos.contiguous(), sup.to(torch.float32).contiguous()


def make_batched_workload(seed=4, n_clouds=256):
    """256 independent clouds: sizes log-uniform in [1e3, 2e5], half 2D and half 3D, uniform in
    [-1, 1]^d, per-dimension periodicity Bernoulli(0.5), one support per cloud for about 32 (2D)
    or 50 (3D) neighbours at the cloud's spacing dx = 2 / n^(1/d).  Returns per-cloud host
    tensors (positions, supports) and descriptors."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(2e5), n_clouds)).astype(np.int64)
    dims = np.array([2] * (n_clouds // 2) + [3] * (n_clouds - n_clouds // 2))
    rng.shuffle(dims)
    per = rng.random((n_clouds, 3)) < 0.5
    gen = torch.Generator().manual_seed(seed)
    clouds = []
    for k in range(n_clouds):
        n, d = int(sizes[k]), int(dims[k])
        dx = 2.0 / n ** (1.0 / d)
        h = (32 * dx * dx / np.pi) ** 0.5 if d == 2 else (3 * 50 * dx ** 3 / (4 * np.pi)) ** (1 / 3)
        x = (torch.rand(n, d, generator=gen) * 2 - 1).contiguous()
        hx = torch.full((n,), float(h), dtype=torch.float32)
        clouds.append(dict(x=x, h=hx, dim=d, periodic=[bool(v) for v in per[k, :d]]))
    return clouds


def config(pairs):
    return {"workload": WORKLOAD, "n_points": N_POINTS, "dim": 3, "mode": "symmetric", "format": "csr",
            "periodic": [False, False, False], "hashMapLength": 4096, "pairs_per_step": pairs,
            "l2": "flushed between timed steps (256 MiB device write)", "parallelism": "replicas"}


def gpu_local_cpus(index):
    """The CPUs NVML reports as local to CUDA device `index` (read-only query), or None."""
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(index)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        words = pynvml.nvmlDeviceGetCpuAffinity(pynvml.nvmlDeviceGetHandleByPciBusId(bus), (os.cpu_count() + 63) // 64)
        cpus = {64 * i + b for i, word in enumerate(words) for b in range(64) if (word >> b) & 1}
        return (cpus & os.sched_getaffinity(0)) or None
    except Exception:
        return None


class near_gpu:
    """Runs the block on the CPUs local to the GPU, so that pinned host buffers allocated inside it
    come from the GPU's NUMA node (host<->device copies from the far node run at a fraction of the
    link's speed); restores the affinity afterwards."""

    def __init__(self, index):
        self.cpus = gpu_local_cpus(index)
        self.old = None

    def __enter__(self):
        if self.cpus:
            self.old = os.sched_getaffinity(0)
            os.sched_setaffinity(0, self.cpus)
        return self

    def __exit__(self, *exc):
        if self.old is not None:
            os.sched_setaffinity(0, self.old)


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def candidate_tests(pos, sup):
    """(query, candidate) pairs the count walk tests on the 1M workload: every query against every
    point of its cell's 3^3 stencil, on the reference's grid (compute_h of util.py:28-79 over the
    domain [-1, 1]^3 and the largest support); computed with torch on the points' device."""
    import torch
    ext, hmax = 2.0, float(sup.max())
    n = int(ext / hmax)
    if ext / hmax - n > 0:
        n -= 1
    n = max(n, 1)
    h = ext / n
    if math.ceil(ext / h) > ext / h:
        h *= 1 + 1e-4
    cnt = int(math.ceil(ext / h))
    c = torch.clamp(torch.floor((pos + 1.0) / h).long(), 0, cnt - 1)
    occ = torch.bincount((c[:, 0] * cnt + c[:, 1]) * cnt + c[:, 2], minlength=cnt ** 3).view(1, 1, cnt, cnt, cnt)
    stencil = torch.nn.functional.conv3d(occ.double(), torch.ones(1, 1, 3, 3, 3, dtype=torch.float64, device=occ.device),
                                         padding=1)
    return int((occ.double() * stencil).sum())


def ncu_issue_active():
    """smsp__issue_active (percent of peak) of the count walk from the committed ncu summary."""
    p = os.path.join(REPO, "profiles", "walk_count_3d_1m.txt")
    try:
        with open(p) as f:
            m = re.search(r"smsp__issue_active\.avg\.pct_of_peak_sustained_active\s+([0-9.]+)", f.read())
        return float(m.group(1)) / 100 if m else None
    except OSError:
        return None


def ncu_traffic():
    """dram bytes per launch of the count walk from the committed ncu summary, if any."""
    p = os.path.join(REPO, "profiles", "walk_count_3d_1m.txt")
    try:
        with open(p) as f:
            m = re.search(r"dram_bytes_per_launch_full_size:\s*([0-9.eE+]+)", f.read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline_reference(pos, sup, budget_s=25.0):
    """The reference's own CPU operators (oracle/_ref) through its driver, on all host threads."""
    import torch
    from oracle import ref_pipeline
    torch.set_num_threads(os.cpu_count() or 1)
    cores = torch.get_num_threads()
    lo, hi, per = [-1.0] * 3, [1.0] * 3, [False] * 3
    t0 = time.perf_counter()
    out = ref_pipeline.radius_search(pos, sup, None, None, lo, hi, per, "symmetric", 4096, "csr")
    t1 = time.perf_counter()
    pairs = int(out[0].numel())
    reps = max(1, min(3, int(budget_s / max(t1 - t0, 1e-3)) - 1))
    times = []
    for _ in range(reps):
        s = time.perf_counter()
        ref_pipeline.radius_search(pos, sup, None, None, lo, hi, per, "symmetric", 4096, "csr")
        times.append(time.perf_counter() - s)
    t = statistics.median(times)
    return {"value": pairs / t, "unit": "pairs/s", "cores": cores, "kind": "reference",
            "sample": f"the full workload ({pairs} pairs), 1 warm-up + median of {reps} runs, "
                      f"torch.set_num_threads({cores})", "seconds_per_search": t}, pairs


def cpu_baseline_port(pos, sup, max_queries=131072):
    """The C restatement (oracle/compact_oracle.c) on a query subset, OpenMP over host threads."""
    from oracle import compact
    q = pos[:max_queries].numpy()
    hq = sup[:max_queries].numpy()
    t0 = time.perf_counter()
    r = compact.radius_search(q, hq, pos.numpy(), sup.numpy(), [-1] * 3, [1] * 3, [False] * 3, "symmetric", 4096)
    t = time.perf_counter() - t0
    return {"value": len(r.col) / t, "unit": "pairs/s", "cores": compact.num_threads(), "kind": "port",
            "sample": f"first {max_queries} queries against all {pos.shape[0]} points, one run"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import torch
    from oracle import ref_pipeline
    pos, sup = make_workload()
    if not ref_pipeline.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's CPU operators) is not "
                                                               "built; run oracle/build_ref.py where the reference "
                                                               "checkout exists"}))
        return 0
    torch.set_num_threads(os.cpu_count() or 1)
    cores = torch.get_num_threads()
    lo, hi, per = [-1.0] * 3, [1.0] * 3, [False] * 3
    # size each step so that warm-up + steps stay within ~3 minutes
    t0 = time.perf_counter()
    out = ref_pipeline.radius_search(pos, sup, None, None, lo, hi, per, "symmetric", 4096, "csr")
    full_t = time.perf_counter() - t0
    full_pairs = int(out[0].numel())
    total_steps = args.steps + args.warmup
    frac = min(1.0, 170.0 / max(total_steps * full_t, 1e-9))
    nq = max(1024, int(N_POINTS * frac)) if frac < 1.0 else N_POINTS
    if nq >= N_POINTS:
        q, hq, r, hr, sample = pos, sup, None, None, f"the full workload ({full_pairs} pairs) per step"
    else:
        q, hq, r, hr = pos[:nq], sup[:nq], pos, sup
        sample = f"first {nq} queries against all {N_POINTS} points per step (time-bounded)"
    for _ in range(args.warmup):
        ref_pipeline.radius_search(q, hq, r, hr, lo, hi, per, "symmetric", 4096, "csr")
    times, pairs = [], 0
    for _ in range(args.steps):
        s = time.perf_counter()
        o = ref_pipeline.radius_search(q, hq, r, hr, lo, hi, per, "symmetric", 4096, "csr")
        times.append(time.perf_counter() - s)
        pairs = int(o[0].numel())
    tot = sum(times)
    value = pairs * len(times) / tot
    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": config(pairs),
            "p50_ms": 1e3 * statistics.median(times), "p99_ms": 1e3 * sorted(times)[min(len(times) - 1,
                                                                                     int(0.99 * len(times)))],
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def bench_batched(dev, stream, flush, steps, warmup, with_cpu):
    """The batched form on the 256-cloud workload: one batched search per step (device-timed, L2
    flushed between steps, walk parameters autotuned on it first) against the per-call loop of
    radiusSearch over the same clouds on the same GPU, plus the end-to-end batched call from pinned
    host memory."""
    import numpy as np
    import torch

    from torchcompactradius_b200.tuning import Autotuner

    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200 import batched

    clouds = make_batched_workload()
    C = len(clouds)
    parts = {2: [c for c in clouds if c["dim"] == 2], 3: [c for c in clouds if c["dim"] == 3]}
    with near_gpu(dev.index):
        host = {d: (torch.cat([c["x"] for c in parts[d]]).pin_memory(),
                    torch.cat([c["h"] for c in parts[d]]).pin_memory()) for d in (2, 3)}
    devx = {d: (host[d][0].to(dev), host[d][1].to(dev)) for d in (2, 3)}
    table = batched.cloud_table(C)
    off = {2: 0, 3: 0}
    views = []
    for k, c in enumerate(clouds):
        d, n = c["dim"], c["x"].shape[0]
        x, h = devx[d][0][off[d]:off[d] + n], devx[d][1][off[d]:off[d] + n]
        off[d] += n
        views.append((x, h))
        table["dim"][k] = d
        table["periodic_mask"][k] = sum(1 << i for i, p in enumerate(c["periodic"]) if p)
        table["domain_min"][k, :d] = -1.0
        table["domain_max"][k, :d] = 1.0
        table["n_query"][k] = table["n_ref"][k] = n
        table["query_pos"][k] = table["ref_pos"][k] = x.data_ptr()
        table["query_sup"][k] = table["ref_sup"][k] = h.data_ptr()
    n_points = int(table["n_query"].sum())
    bufs = batched.BatchBuffers(dev)

    def step():
        return batched.run_batch(table, "gather", True, "csr", dev, buffers=bufs, stream=stream)

    for _ in range(warmup):
        out = step()
    pairs = out["total"]
    tuner = Autotuner(reps=2)
    tuned = tuner.tune(step, key="batched")
    ms = []
    for k in range(steps):
        flush.fill_(k & 0xff)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        step()
        e.record(stream)
        e.synchronize()
        ms.append(s.elapsed_time(e))
    batched_value = pairs * len(ms) / (sum(ms) / 1e3)

    # per-call loop: one radiusSearch per cloud through the public API, inputs already on the GPU
    doms = [tcr.DomainDescription(torch.full((c["dim"],), -1.0), torch.full((c["dim"],), 1.0),
                                  torch.tensor(c["periodic"]), c["dim"]) for c in clouds]

    def per_call():
        tot = 0
        for (x, h), dom in zip(views, doms):
            adj = tcr.radiusSearch(tcr.PointCloud(x, h), mode="gather", domain=dom, hashMapLength=4096,
                                   algorithm="compact", format="csr")
            tot += adj.indices.numel()
        return tot

    per_call()
    pc_ms = []
    for k in range(max(2, min(steps, 4))):
        flush.fill_(k & 0xff)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        tot = per_call()
        e.record(stream)
        e.synchronize()
        pc_ms.append(s.elapsed_time(e))
    per_call_value = tot * len(pc_ms) / (sum(pc_ms) / 1e3)

    # end to end: inputs from pinned host memory, batched search, CSR back to pinned host memory
    with near_gpu(dev.index):
        out_idx = torch.empty(pairs, dtype=torch.int64, pin_memory=True)
        out_ptr = torch.empty(n_points + 1, dtype=torch.int32, pin_memory=True)
    e2e_ms = []
    for k in range(max(3, min(steps, 10))):
        flush.fill_(k & 0xff)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for d in (2, 3):
            devx[d][0].copy_(host[d][0], non_blocking=True)
            devx[d][1].copy_(host[d][1], non_blocking=True)
        o = step()
        out_idx.copy_(o["col"], non_blocking=True)
        out_ptr.copy_(o["indptr"], non_blocking=True)
        e.record(stream)
        e.synchronize()
        e2e_ms.append(s.elapsed_time(e))
    h2d = sum(host[d][0].numel() * 4 + host[d][1].numel() * 4 for d in (2, 3))
    res = {"workload": "256 clouds, sizes log-uniform [1e3, 2e5] (seed 4), 128 2D + 128 3D, uniform in [-1,1]^d, "
                       "per-dim periodicity Bernoulli(0.5), 32 (2D) / 50 (3D) neighbours, gather, CSR",
           "clouds": C, "points": n_points, "pairs_per_step": pairs,
           "tuning": {"chosen": {"queries_per_unit": tuned[0], "walk_blocks_per_sm": tuned[1]},
                      "ms_per_step": {f"{c[0]}q/{c[1]}b": round(v, 3) for c, v in tuner.timings["batched"].items()}},
           "value": batched_value, "unit": "pairs/s", "ms_per_step": statistics.mean(ms),
           "p50_ms": statistics.median(ms), "p99_ms": sorted(ms)[min(len(ms) - 1, int(0.99 * len(ms)))],
           "per_call": {"value": per_call_value, "unit": "pairs/s", "ms_per_batch": statistics.mean(pc_ms),
                        "pairs_match": tot == pairs, "what": "loop of radiusSearch(algorithm='compact') per cloud"},
           "speedup_vs_per_call": batched_value / per_call_value,
           "e2e": {"value": pairs * len(e2e_ms) / (sum(e2e_ms) / 1e3), "unit": "pairs/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8 * pairs + 4 * (n_points + 1),
                   "ms_per_step": statistics.mean(e2e_ms)}}
    if with_cpu:
        res["cpu_baseline"] = cpu_baseline_batched(clouds)
    return res


def make_served_workload(seed=5, n_scenes=64, rate=2000.0, seconds=1.0):
    """64 persistent 3D scenes (sizes log-uniform in [1e3, 1e6], uniform in the periodic box
    [-1, 1]^3, one support per scene for about 50 neighbours) and a Poisson arrival trace
    (rate per second over `seconds`), each request naming a scene uniformly at random."""
    import numpy as np
    import torch
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(1e6), n_scenes)).astype(np.int64)
    gen = torch.Generator().manual_seed(seed)
    scenes = []
    for n in sizes:
        dx = 2.0 / float(n) ** (1.0 / 3.0)
        h = (3 * 50 * dx ** 3 / (4 * np.pi)) ** (1 / 3)
        scenes.append((torch.rand(int(n), 3, generator=gen) * 2 - 1, float(h)))
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        arrivals.append((t, int(rng.integers(0, n_scenes))))
    return scenes, arrivals


HBM_BUDGET = 40e9  # the served form's admission budget: about three groups of all 64 scenes in flight;
# larger budgets let the torch allocator's cache fill the 180 GB and stall on a free-and-retry


def bench_served(dev, seconds=1.0, slots=2):
    """The served form: requests arrive on a Poisson trace; each jitters its scene by
    N(0, (0.05 h)^2) per coordinate and searches it (gather, COO).  The search server (resident
    scenes, incremental re-sort, HBM-budget admission, continuous batching with groups enqueued
    without host waits) and the per-call path (one radiusSearch per request, in arrival order)
    replay the same trace;
    latency = completion - arrival, host clock."""
    import torch

    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.serving import Request, Scene, SearchServer
    from torchcompactradius_b200.tuning import Autotuner

    scenes, arrivals = make_served_workload(seconds=seconds)
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.tensor([True] * 3), 3)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # both forms start from an empty allocator cache

    def pct(v, q):
        v = sorted(v)
        return v[min(len(v) - 1, int(q * len(v)))]

    # ---- served -------------------------------------------------------------------------
    srv = SearchServer(dev, mode="gather", hbm_budget=HBM_BUDGET, slots=slots)
    for x, h in scenes:
        srv.add_scene(Scene(x.to(dev), torch.full((x.shape[0],), h, device=dev), dom, expected_neighbours=50))
    with srv:
        for k in range(len(scenes)):  # warm-up: one search per scene (first build, caches)
            srv.search(k, timeout=120)

        def all_scenes():  # one request per scene, together: the server's typical batch
            for r in [srv.submit(Request(k)) for k in range(len(scenes))]:
                r.wait(120)

        tuner = Autotuner(reps=2)
        tuned = tuner.tune(all_scenes, key="served", apply=srv.set_tuning)
        srv.batches = srv.batched_requests = 0
        torch.cuda.synchronize()
        reqs = []
        counted = []

        def consume(r):  # count the pairs and drop the result as soon as a request completes
            counted.append(r.result.row.numel())
            r.result = None

        t0 = time.perf_counter()
        for ta, k in arrivals:
            while time.perf_counter() - t0 < ta:
                time.sleep(0.0001)
            reqs.append(srv.submit(Request(k, arrival=t0 + ta, jitter=0.05 * scenes[k][1], on_done=consume)))
        for r in reqs:
            r.wait(300)
        pairs = sum(counted)
        t_end = max(r.finish for r in reqs)
        lat = [1e3 * r.latency for r in reqs]
        queue = [1e3 * (r.admitted - r.arrival) for r in reqs]
        service = [1e3 * (r.finish - r.admitted) for r in reqs]
        served = {"value": pairs / (t_end - t0), "unit": "pairs/s", "requests": len(reqs),
                  "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99), "batches": srv.batches,
                  "mean_batch": srv.batched_requests / max(srv.batches, 1), "seconds": t_end - t0,
                  "queue_p50_ms": pct(queue, 0.5), "queue_p99_ms": pct(queue, 0.99),
                  "service_p50_ms": pct(service, 0.5), "service_p99_ms": pct(service, 0.99)}
        # capacity: the whole trace submitted at once
        counted.clear()
        srv.batches = srv.batched_requests = 0
        t0 = time.perf_counter()
        reqs = [srv.submit(Request(k, arrival=t0, jitter=0.05 * scenes[k][1], on_done=consume)) for _, k in arrivals]
        for r in reqs:
            r.wait(300)
        t_end = max(r.finish for r in reqs)
        served_capacity = {"value": sum(counted) / (t_end - t0), "unit": "pairs/s", "seconds": t_end - t0,
                           "batches": srv.batches, "mean_batch": srv.batched_requests / max(srv.batches, 1)}

    # ---- per call (the same engine tuning as the server) ---------------------------------
    from torchcompactradius_b200 import context
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    pos = [x.to(dev) for x, h in scenes]
    sup = [torch.full((x.shape[0],), h, device=dev) for x, h in scenes]
    with context.use(context.SearchContext(unit_queries=tuned[0], walk_blocks_per_sm=tuned[1])):
        for k in range(len(scenes)):
            tcr.radiusSearch(tcr.PointCloud(pos[k], sup[k]), mode="gather", domain=dom, algorithm="compact")
        torch.cuda.synchronize()
        lat, pairs = [], 0
        t0 = time.perf_counter()
        for ta, k in arrivals:
            while time.perf_counter() - t0 < ta:
                time.sleep(0.0001)
            pos[k] = pos[k] + torch.randn(pos[k].shape, device=dev) * (0.05 * scenes[k][1])
            adj = tcr.radiusSearch(tcr.PointCloud(pos[k], sup[k]), mode="gather", domain=dom, algorithm="compact")
            pairs += adj.row.numel()  # radiusSearch returns after the host has read the pair count
            lat.append(1e3 * (time.perf_counter() - (t0 + ta)))
        t_end = time.perf_counter()
    per_call = {"value": pairs / (t_end - t0), "unit": "pairs/s", "requests": len(arrivals),
                "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99), "seconds": t_end - t0,
                "note": "falls behind the arrivals, so value is its capacity"}
    return {"workload": f"64 persistent 3D scenes, sizes log-uniform [1e3, 1e6] (seed 5), periodic [-1,1]^3, "
                        f"50 neighbours, gather, COO; Poisson arrivals 2000/s for {seconds:g} s, each request "
                        f"jitters its scene by N(0, (0.05 h)^2); {HBM_BUDGET / 1e9:g} GB admission budget, {slots} worker stream(s)",
            "points": int(sum(x.shape[0] for x, h in scenes)),
            "tuning": {"chosen": {"queries_per_unit": tuned[0], "walk_blocks_per_sm": tuned[1]},
                       "ms_per_batch_of_all_scenes": {f"{c[0]}q/{c[1]}b": round(v, 3)
                                                      for c, v in tuner.timings.get("served", {}).items()}},
            "served": served, "served_capacity": served_capacity, "per_call": per_call,
            "speedup_vs_per_call": served_capacity["value"] / per_call["value"],
            "p99_ratio_per_call_over_served": per_call["p99_ms"] / served["p99_ms"]}


def make_small_workload(seed=0):
    """The reference's CPU-runnable case: 64 x 64 cell centres in the periodic [-1, 1]^2, jittered by
    U(-0.1 dx, 0.1 dx), dx = 2/64, uniform support sqrt(32 dx^2 / pi) (about 32 neighbours)."""
    import numpy as np
    import torch
    g = torch.Generator().manual_seed(seed)
    dx = 2.0 / 64
    c = -1.0 + dx * (torch.arange(64, dtype=torch.float32) + 0.5)
    pos = torch.stack(torch.meshgrid(c, c, indexing="ij"), -1).reshape(-1, 2)
    pos = pos + (torch.rand(pos.shape, generator=g) * 0.2 - 0.1) * dx
    h = torch.full((pos.shape[0],), float((32 * dx * dx / np.pi) ** 0.5))
    return pos.contiguous(), h


def bench_graphs(dev, flush, steps=200):
    """CUDA-graph replay (graphs.StaticSearch) against the eager public API: host-observed latency
    of one search of the small 2D workload, and device time of the 1M-point search."""
    import torch

    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.graphs import StaticSearch

    def pct(v, q):
        v = sorted(v)
        return v[min(len(v) - 1, int(q * len(v)))]

    pos, h = make_small_workload()
    pos, h = pos.to(dev), h.to(dev)
    dom = tcr.DomainDescription(torch.full((2,), -1.0), torch.full((2,), 1.0), torch.tensor([True, True]), 2)
    ss = StaticSearch(tcr.PointCloud(pos, h), dom, mode="gather", format="coo")
    eager, graph = [], []
    for k in range(steps + 10):
        t = time.perf_counter()
        a = tcr.radiusSearch(tcr.PointCloud(pos, h), mode="gather", domain=dom, algorithm="compact", format="coo")
        t1 = time.perf_counter()
        b = ss.run()
        t2 = time.perf_counter()
        if k >= 10:
            eager.append(1e3 * (t1 - t))
            graph.append(1e3 * (t2 - t1))
    same = torch.equal(a.row, b.row) and torch.equal(a.col, b.col)
    small = {"workload": "4096-point jittered 64x64 grid, periodic [-1,1]^2, gather, COO (host-observed latency "
                         "per search, output on the device)", "pairs": int(a.row.numel()),
             "eager_p50_ms": pct(eager, 0.5), "eager_p99_ms": pct(eager, 0.99),
             "graph_p50_ms": pct(graph, 0.5), "graph_p99_ms": pct(graph, 0.99), "same_result": bool(same)}
    pos_h, sup_h = make_workload()
    p1, h1 = pos_h.to(dev), sup_h.to(dev)
    dom3 = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.tensor([False] * 3), 3)
    big = StaticSearch(tcr.PointCloud(p1, h1), dom3, mode="symmetric", format="csr")
    stream = big.plan.stream
    ms = []
    for k in range(13):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        with torch.cuda.stream(stream):
            big.plan.graph.replay()
        e.record(stream)
        e.synchronize()
        if k >= 3:
            ms.append(s.elapsed_time(e))
    pairs = int(big.run().indices.numel())
    return {"small": small,
            "big": {"workload": WORKLOAD, "graph_replay_ms": statistics.mean(ms),
                    "value": pairs / (statistics.mean(ms) / 1e3), "unit": "pairs/s"}}


def make_adaptive_workload(seed=6, n=1 << 22, k_target=32.0):
    """Adaptive resolution: 2^22 points, 70% from 8 Gaussian blobs (sigma 0.1, centres
    U[-0.8, 0.8]^3) and 30% uniform in [-1, 1]^3; x periodic (wrapped), y and z clamped; supports
    h_i = cbrt(3 K / (4 pi rho(x_i))) from the mixture's own density, clamped to [h_max/4, h_max]
    with h_max the background's (K = 32 gives about 40 neighbours per point)."""
    import numpy as np
    import torch
    g = torch.Generator().manual_seed(seed)
    nb = int(0.7 * n)
    centres = torch.rand(8, 3, generator=g) * 1.6 - 0.8
    pick = torch.randint(0, 8, (nb,), generator=g)
    x = torch.cat([centres[pick] + 0.1 * torch.randn(nb, 3, generator=g), torch.rand(n - nb, 3, generator=g) * 2 - 1])
    x[:, 0] = torch.remainder(x[:, 0] + 1.0, 2.0) - 1.0
    x[:, 1:] = x[:, 1:].clamp(-1.0, 0.999999)
    sigma = 0.1
    rho = torch.full((n,), 0.3 * n / 8.0)
    norm = 0.7 * n / 8.0 / (2 * np.pi * sigma * sigma) ** 1.5
    for c in centres:
        d = x - c
        d[:, 0] = torch.remainder(d[:, 0] + 1.0, 2.0) - 1.0  # periodic in x
        rho += norm * torch.exp(-(d * d).sum(1) / (2 * sigma * sigma))
    h = (3 * k_target / (4 * np.pi * rho)) ** (1.0 / 3.0)
    hmax = float((3 * k_target / (4 * np.pi * 0.3 * n / 8.0)) ** (1.0 / 3.0))
    h = h.clamp(hmax / 4, hmax)
    return x.contiguous(), h.to(torch.float32).contiguous()


def bench_adaptive(dev, flush, steps=5):
    """The adaptive workload in scatter mode, COO: single-level compact cells (sized for the
    largest support) against the exact multi-level search, same pair set checked."""
    import torch

    import torchcompactradius_b200 as tcr
    x, h = make_adaptive_workload()
    x, h = x.to(dev), h.to(dev)
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.tensor([True, False, False]), 3)
    stream = torch.cuda.current_stream(dev)
    res = {}
    keys = {}
    for algo in ("mlm", "compact"):
        for _ in range(2):  # warm-up: kernels loaded, allocator pools grown
            adj = tcr.radiusSearch(tcr.PointCloud(x, h), mode="scatter", domain=dom, algorithm=algo, format="coo")
        ms = []
        for k in range(steps):
            flush.fill_(k & 0xff)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            adj = tcr.radiusSearch(tcr.PointCloud(x, h), mode="scatter", domain=dom, algorithm=algo, format="coo")
            e.record(stream)
            e.synchronize()
            ms.append(s.elapsed_time(e))
        pairs = int(adj.row.numel())
        keys[algo] = torch.sort(adj.row * x.shape[0] + adj.col)[0]
        del adj
        res[algo] = {"ms_per_search": statistics.median(ms), "value": pairs / (statistics.median(ms) / 1e3),
                     "unit": "pairs/s", "pairs": pairs, "ms_all": ms}
    same = bool(torch.equal(keys["mlm"], keys["compact"]))
    del keys
    return {"workload": "2^22 points, 70% in 8 Gaussian blobs (sigma 0.1) + 30% uniform, periodic in x, supports "
                        "from the mixture density (ratio up to 4), scatter, COO (seed 6)",
            "mlm": res["mlm"], "compact": res["compact"], "same_pair_set": same,
            "speedup_mlm_vs_compact": res["compact"]["ms_per_search"] / res["mlm"]["ms_per_search"]}


def bench_scatter(dev, flush, steps=10):
    """scatter_sum of one float32 value per pair onto the rows of the 1M-point neighbour list (COO,
    rows non-decreasing): the per-particle sum an SPH density or a GNN aggregation does next.
    Device time per call (L2 flushed), against the HBM roofline of reading the index and the
    values once and writing the sums; torch's atomic index_add_ and the reference's own CPU
    operator on the same data beside it."""
    import torch

    import torchcompactradius_b200 as tcr
    pos, sup = make_workload()
    x, h = pos.to(dev), sup.to(dev)
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.zeros(3, dtype=torch.bool), 3)
    adj = tcr.radiusSearch(tcr.PointCloud(x, h), None, mode="symmetric", domain=dom, algorithm="compact", format="coo")
    row = adj.row
    del adj
    n, P = x.shape[0], row.numel()
    vals = torch.rand(P, device=dev, generator=torch.Generator(dev).manual_seed(9))
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(3):
            fn()
        ms = []
        for k in range(steps):
            flush.fill_(k & 0xff)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            r = fn()
            e.record(stream)
            e.synchronize()
            ms.append(s.elapsed_time(e))
        return statistics.median(ms), r

    l0 = tcr_launches()
    ms, sums = timed(lambda: tcr.scatter_sum(vals, row, 0, None, n))
    launches = (tcr_launches() - l0) // (steps + 3)
    again = tcr.scatter_sum(vals, row, 0, None, n)
    ms_ia, ref_ia = timed(lambda: torch.zeros(n, device=dev).index_add_(0, row, vals))
    alg = 8 * P + 4 * P + 4 * n  # index and values read once, sums written once
    peak, peak_kind = measured_peak()
    res = {"workload": "scatter_sum of one float32 per pair onto the rows of the 3D 1M symmetric neighbour list "
                       f"({P} pairs, {n} rows, COO rows non-decreasing)",
           "ms_per_call": ms, "value": P / (ms / 1e3), "unit": "pairs/s", "launches_per_call": int(launches),
           "roofline": {"bound": "hbm", "algorithmic_bytes": alg, "achieved": alg / (ms / 1e3) / 1e9, "peak": peak,
                        "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
           "repeatable": bool(torch.equal(sums, again)),
           "torch_index_add_ms": ms_ia,
           "torch_index_add_max_abs_diff": float((ref_ia - sums).abs().max())}
    try:
        from oracle import ref_pipeline
        if ref_pipeline.available():
            ops = ref_pipeline.ops()
            torch.set_num_threads(os.cpu_count() or 1)
            v_h, r_h = vals.cpu(), row.cpu()
            ops.scatter_sum(v_h, r_h, 0, None, n)
            t0 = time.perf_counter()
            ref = ops.scatter_sum(v_h, r_h, 0, None, n)
            dt = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": P / dt, "unit": "pairs/s", "cores": 1, "kind": "reference",
                                   "sample": "the full reduction, one call after a warm-up (the reference's CPU "
                                             "scatter loop is serial)", "seconds": dt,
                                   "bit_identical": bool(torch.equal(ref, sums.cpu()))}
    except Exception as ex:  # the compiled reference is optional on the GPU box
        res["cpu_baseline"] = {"unavailable": str(ex)}
    return res


def tcr_launches():
    from torchcompactradius_b200 import _lib
    return int(_lib.load().tcr_kernel_launches())


def bench_fixed_support(dev, flush, steps=5):
    """One support for every point (supportOverride): the 1M-point workload's positions with the
    mean support, symmetric CSR, searched once with the supports given as an array (the two-support
    symmetric walk) and once with supportOverride (the fixed-radius form: the gather walk); the
    same CSR both ways."""
    import torch

    import torchcompactradius_b200 as tcr
    pos, sup = make_workload()
    x = pos.to(dev)
    hval = float(sup.mean())
    hs = torch.full((x.shape[0],), hval, device=dev)
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.zeros(3, dtype=torch.bool), 3)
    stream = torch.cuda.current_stream(dev)

    def run(fixed):
        if fixed:
            return tcr.radiusSearch(tcr.PointCloud(x, None), None, supportOverride=hval, mode="symmetric",
                                    domain=dom, algorithm="compact", format="csr")
        return tcr.radiusSearch(tcr.PointCloud(x, hs), None, mode="symmetric", domain=dom, algorithm="compact",
                                format="csr")

    out = {}
    for fixed in (False, True):
        adj = run(fixed)
        ms = []
        for k in range(steps):
            flush.fill_(k & 0xff)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            adj = run(fixed)
            e.record(stream)
            e.synchronize()
            ms.append(s.elapsed_time(e))
        out["fixed" if fixed else "array"] = (statistics.median(ms), adj)
    (ta, a), (tf, f) = out["array"], out["fixed"]
    return {"workload": f"3d_1m positions, one support {hval:.6g} for every point, symmetric CSR",
            "pairs": int(f.indices.numel()), "supports_array_ms": ta, "support_override_ms": tf,
            "speedup": ta / tf, "same_csr": bool(torch.equal(a.indices, f.indices) and torch.equal(a.indptr, f.indptr))}


def bench_f64(dev, flush, steps=3, cpu=True):
    """The 1M-point workload in float64 (positions, supports and domain): the reference's double
    search, symmetric CSR, timed per search with events (L2 flushed), and the reference's own double
    operators on the host beside it."""
    import torch

    import torchcompactradius_b200 as tcr
    pos, sup = make_workload()
    x, h = pos.double().to(dev), sup.double().to(dev)
    dom = tcr.DomainDescription(torch.full((3,), -1.0, dtype=torch.float64), torch.full((3,), 1.0, dtype=torch.float64),
                                torch.zeros(3, dtype=torch.bool), 3)
    stream = torch.cuda.current_stream(dev)
    adj = tcr.radiusSearch(tcr.PointCloud(x, h), None, mode="symmetric", domain=dom, algorithm="compact", format="csr")
    ms = []
    for k in range(steps):
        flush.fill_(k & 0xff)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        adj = tcr.radiusSearch(tcr.PointCloud(x, h), None, mode="symmetric", domain=dom, algorithm="compact",
                               format="csr")
        e.record(stream)
        e.synchronize()
        ms.append(s.elapsed_time(e))
    pairs = int(adj.indices.numel())
    res = {"workload": "3d_1m_uniform_symmetric_csr in float64 (positions, supports, domain)", "pairs": pairs,
           "ms_per_search": statistics.median(ms), "value": pairs / (statistics.median(ms) / 1e3), "unit": "pairs/s",
           "note": "the float32 walk over float32 copies; pairs within the widened rounding band decided in double"}
    if cpu:
        try:
            from oracle import ref_pipeline
            if ref_pipeline.available():
                torch.set_num_threads(os.cpu_count() or 1)
                t0 = time.perf_counter()
                ref = ref_pipeline.radius_search(pos.double(), sup.double(), None, None, [-1.0] * 3, [1.0] * 3,
                                                 [False] * 3, "symmetric", 4096, "csr", dtype=torch.float64)
                dt = time.perf_counter() - t0
                res["cpu_baseline"] = {"value": int(ref[0].numel()) / dt, "unit": "pairs/s",
                                       "cores": torch.get_num_threads(), "kind": "reference",
                                       "sample": "the full workload in float64, one run", "seconds": dt,
                                       "pairs_match": int(ref[0].numel()) == pairs,
                                       "indptr_match": bool(torch.equal(ref[1].to(torch.int64),
                                                                        adj.indptr.cpu().to(torch.int64)))}
        except Exception as ex:
            res["cpu_baseline"] = {"unavailable": str(ex)}
    return res


def cpu_baseline_batched(clouds, budget_s=12.0):
    """The reference's own CPU search, one call per cloud (its batched radius() fails), over the
    first clouds of the workload until about budget_s seconds have passed."""
    import torch
    from oracle import ref_pipeline
    if not ref_pipeline.available():
        return None
    torch.set_num_threads(os.cpu_count() or 1)
    pairs, t, k = 0, 0.0, 0
    for c in clouds:
        d = c["dim"]
        s = time.perf_counter()
        o = ref_pipeline.radius_search(c["x"], c["h"], None, None, [-1.0] * d, [1.0] * d, c["periodic"], "gather",
                                       4096, "csr")
        t += time.perf_counter() - s
        pairs += int(o[0].numel())
        k += 1
        if t > budget_s:
            break
    return {"value": pairs / t, "unit": "pairs/s", "cores": torch.get_num_threads(), "kind": "reference",
            "sample": f"the first {k} of {len(clouds)} clouds, one reference call per cloud ({pairs} pairs)"}


class Ranks:
    """The multi-GPU plumbing of the bench: one process per GPU, every rank an independent replica
    of the workload; the only collectives are a barrier around the timed region and a max-reduce of
    each rank's device time (whole-job value = pairs of all ranks / the slowest rank's time)."""

    def __init__(self, world, device=None):
        self.world = world
        self.device = device

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v):
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def value(self, pairs_per_rank, steps, total_ms_this_rank):
        """pairs/s of the whole job: every rank did `pairs_per_rank` pairs per step."""
        slowest = self.max(total_ms_this_rank)
        return pairs_per_rank * steps * self.world / (slowest / 1e3), slowest


def run_b200(args):
    import torch
    import torch.distributed as dist

    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200 import _lib
    from torchcompactradius_b200.graphs import StaticSearch
    from torchcompactradius_b200.search import compact_search
    from torchcompactradius_b200.tuning import Autotuner, set_tuning

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    ranks = Ranks(world, dev)
    barrier = ranks.barrier
    max_over_ranks = ranks.max

    pos_h, sup_h = make_workload()
    with near_gpu(local):
        pos_pin, sup_pin = pos_h.pin_memory(), sup_h.pin_memory()
    pos_d, sup_d = pos_h.to(dev), sup_h.to(dev)
    dom = tcr.DomainDescription(torch.tensor([-1.0] * 3), torch.tensor([1.0] * 3), torch.tensor([False] * 3), 3)
    lib = _lib.load()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def device_step(events=None):
        (col, indptr, entries), _ = compact_search(pos_d, sup_d, pos_d, sup_d, [-1.0] * 3, [1.0] * 3, 0,
                                                   "symmetric", 4096, "csr", True, events=events)
        return col, indptr, entries

    for _ in range(args.warmup):
        col, indptr, entries = device_step()
    pairs = int(col.numel())
    torch.cuda.synchronize()
    # the walks' run-time parameters, picked on this workload (no result depends on them)
    tuner = Autotuner(reps=3)
    tuned = tuner.tune(lambda: device_step(), key="headline")
    # the cell-size multiplier, on the eager single search it applies to (kept only if it finds the
    # same pairs); the graph-replayed headline keeps the reference's cell
    from torchcompactradius_b200 import context as tcr_context
    scale = tuner.tune_cell_scale(
        lambda: tcr.radiusSearch(tcr.PointCloud(pos_d, sup_d), None, mode="symmetric", domain=dom,
                                 algorithm="compact", format="csr"), key="headline")
    tuning = {"chosen": {"queries_per_unit": tuned[0], "walk_blocks_per_sm": tuned[1], "cell_scale": scale},
              "ms_per_search": {f"{c[0]}q/{c[1]}b": round(v, 4) for c, v in tuner.timings["headline"].items()},
              "eager_ms_per_cell_scale": {str(m): round(v, 4) for m, v in tuner.scale_timings["headline"].items()}}
    tcr_context.current().cell_scale = 1.0

    # ---- phases of the eager path (public API) ------------------------------------------------
    _lib.check(lib.tcr_profile_kernels(1), "tcr_profile_kernels")
    eager_ms, build_ms, count_ms, emit_ms = [], [], [], []
    for k in range(max(3, min(args.steps, 10))):
        flush.fill_(k & 0xff)
        ev = {}
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = lib.tcr_kernel_launches()
        s.record(stream)
        device_step(ev)
        e.record(stream)
        e.synchronize()
        per_search_launches = lib.tcr_kernel_launches() - l0
        eager_ms.append(s.elapsed_time(e))
        build_ms.append(ev["build"][0].elapsed_time(ev["build"][1]))
        count_ms.append(ev["count"][0].elapsed_time(ev["count"][1]))
        emit_ms.append(ev["emit"][0].elapsed_time(ev["emit"][1]))

    # ---- device-resident timing: the search recorded once as a CUDA graph and replayed --------
    # (graphs.StaticSearch; profiling is on while it records, so the count walk and expansion
    # launches carry their timing events inside the graph)
    plan = StaticSearch(tcr.PointCloud(pos_d, sup_d), dom, mode="symmetric", format="csr")
    pstream = plan.plan.stream
    for _ in range(3):
        plan.run()
    clk = Clocks(local)
    clk.start()
    barrier()
    torch.cuda.synchronize()
    step_ms, walk_ms, expand_ms = [], [], []
    for k in range(args.steps):
        flush.fill_(k & 0xff)  # L2 flush outside the step's events
        torch.cuda.current_stream(dev).synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(pstream)
        with torch.cuda.stream(pstream):
            plan.plan.graph.replay()
        e.record(pstream)
        e.synchronize()
        step_ms.append(s.elapsed_time(e))
        walk_ms.append(_lib.profile_kernel_ms(_lib.PROFILE_COUNT_WALK))
        expand_ms.append(_lib.profile_kernel_ms(_lib.PROFILE_EXPAND))
    torch.cuda.synchronize()
    barrier()
    launches = per_search_launches * args.steps  # kernel nodes of the recorded search, per replay
    clocks = clk.stop()
    _lib.check(lib.tcr_profile_kernels(0), "tcr_profile_kernels")
    replay = plan.run()
    assert replay.indices.numel() == pairs and torch.equal(replay.indptr, indptr)
    value, total_ms = ranks.value(pairs, args.steps, sum(step_ms))

    # ---- end to end through the public API (pinned host in, host out) ----------------------
    nq = N_POINTS
    with near_gpu(local) as near:
        out_idx = torch.empty(pairs, dtype=torch.int64, pin_memory=True)
        out_ptr = torch.empty(nq + 1, dtype=torch.int32, pin_memory=True)
        out_ent = torch.empty(nq, dtype=torch.int64, pin_memory=True)
    e2e_ms = []
    barrier()
    for k in range(max(3, min(args.steps, 30))):
        flush.fill_(k & 0xff)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        p = pos_pin.to(dev, non_blocking=True)
        h = sup_pin.to(dev, non_blocking=True)
        adj = tcr.radiusSearch(tcr.PointCloud(p, h), mode="symmetric", domain=dom, hashMapLength=4096,
                               algorithm="compact", format="csr")
        out_idx.copy_(adj.indices, non_blocking=True)
        out_ptr.copy_(adj.indptr, non_blocking=True)
        out_ent.copy_(adj.rowEntries, non_blocking=True)
        e.record(stream)
        e.synchronize()
        e2e_ms.append(s.elapsed_time(e))
    # the device->host copy of the column indices alone: the link's share of the step
    d2h = []
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        out_idx.copy_(adj.indices, non_blocking=True)
        e.record(stream)
        e.synchronize()
        d2h.append(s.elapsed_time(e))
    d2h_gbs = 8 * pairs / (statistics.median(d2h) / 1e3) / 1e9
    barrier()
    e2e_total = max_over_ranks(sum(e2e_ms))
    e2e_value = pairs * len(e2e_ms) * world / (e2e_total / 1e3)
    ok = torch.equal(out_ptr, indptr.cpu()) and int(out_ent.sum()) == pairs

    # ---- roofline of the dominant kernel (the count walk) and of the whole search ----------
    peak, peak_kind = measured_peak()
    walk_bytes = 16 * N_POINTS + 4 * N_POINTS + 4 * N_POINTS  # sorted float4 points, sort index, counts
    walk_s = statistics.mean(walk_ms) / 1e3
    achieved = walk_bytes / walk_s / 1e9
    search_bytes = 16 * N_POINTS + 8 * pairs + 4 * (N_POINTS + 1) + 8 * N_POINTS
    search_s = statistics.mean(step_ms) / 1e3
    traffic = ncu_traffic()
    tests = candidate_tests(pos_d, sup_d)
    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "b200", "config": config(pairs),
        "p50_ms": statistics.median(step_ms), "p99_ms": sorted(step_ms)[min(len(step_ms) - 1,
                                                                         int(0.99 * len(step_ms)))],
        "execution": "build+count+emit recorded once as a CUDA graph (graphs.StaticSearch) and replayed per step",
        "eager_ms_per_step": statistics.mean(eager_ms),
        "phases_ms": {"build": statistics.mean(build_ms), "count": statistics.mean(count_ms),
                      "emit": statistics.mean(emit_ms), "count_walk_kernel": statistics.mean(walk_ms),
                      "expand_kernel": statistics.mean(expand_ms), "of": "phases of the eager path; kernels of the "
                      "timed replays"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "walk_count_kernel<3,false,symmetric> (every pair test)",
                     "algorithmic_bytes_per_launch": walk_bytes, "launch_ms": statistics.mean(walk_ms),
                     "pair_tests_note": "bound by candidate tests (instruction issue), not HBM",
                     "candidate_tests_per_launch": tests, "candidate_tests_per_s": tests / walk_s,
                     "issue_active_frac_ncu": ncu_issue_active(),
                     "peak_kind": peak_kind},
        "search_roofline": {"bound": "hbm", "algorithmic_bytes_per_search": search_bytes,
                            "achieved": search_bytes / search_s / 1e9, "peak": peak, "unit": "GB/s",
                            "frac": search_bytes / search_s / 1e9 / peak, "peak_kind": peak_kind},
        "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": 16 * N_POINTS,
                "d2h_bytes_per_step": 8 * pairs + 4 * (N_POINTS + 1) + 8 * N_POINTS,
                "ms_per_step": e2e_total / len(e2e_ms), "output_checked": bool(ok),
                "d2h_indices_GBps": d2h_gbs,
                "host_buffers": "pinned, allocated on the GPU's NUMA node" if near.cpus else "pinned"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "tuning": tuning,
    }
    if world == 1 and not args.no_batched:
        line["batched"] = bench_batched(dev, stream, flush, max(3, min(args.steps, 10)), 3,
                                        rank == 0 and not args.no_cpu_baseline)
        set_tuning(0, 0)  # the other forms run with the defaults
        line["graphs"] = bench_graphs(dev, flush)
        line["adaptive"] = bench_adaptive(dev, flush)
        line["scatter"] = bench_scatter(dev, flush)
        line["f64"] = bench_f64(dev, flush, cpu=rank == 0 and not args.no_cpu_baseline)
        line["fixed_support"] = bench_fixed_support(dev, flush)
        del flush
        line["served"] = bench_served(dev)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb, ref_pairs = cpu_baseline_reference(pos_h, sup_h)
            cb["pairs_match"] = ref_pairs == pairs
        except Exception as ex:  # the compiled reference is missing: time the C restatement instead
            cb = cpu_baseline_port(pos_h, sup_h)
            cb["note"] = f"reference operators unavailable: {ex}"
        line["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(summarize(line, args.details)))
    return 0


def _pick(d, *keys):
    return {k: d[k] for k in keys if isinstance(d, dict) and k in d}


def summarize(line, details_path):
    """The printed line: the headline keys in full and a summary of every other form; the full
    record goes to `details_path` (the line names it)."""
    out = dict(line)
    try:
        with open(details_path, "w") as f:
            json.dump(line, f, indent=1)
        out["details"] = os.path.abspath(details_path)
    except OSError as ex:
        out["details"] = f"not written: {ex}"
    if "tuning" in out:
        out["tuning"] = out["tuning"].get("chosen", out["tuning"])
    b = line.get("batched")
    if b:
        out["batched"] = dict(_pick(b, "value", "unit", "ms_per_step", "p99_ms", "speedup_vs_per_call"),
                              clouds=b.get("clouds"), per_call_pairs_match=b.get("per_call", {}).get("pairs_match"),
                              e2e=_pick(b.get("e2e", {}), "value", "unit"),
                              cpu_baseline=_pick(b.get("cpu_baseline", {}), "value", "unit", "cores", "kind"))
    g = line.get("graphs")
    if g:
        out["graphs"] = {"small_graph_p50_ms": g.get("small", {}).get("graph_p50_ms"),
                         "small_eager_p50_ms": g.get("small", {}).get("eager_p50_ms"),
                         "big_graph_replay_ms": g.get("big", {}).get("graph_replay_ms")}
    a = line.get("adaptive")
    if a:
        out["adaptive"] = {"mlm_ms": a.get("mlm", {}).get("ms_per_search"),
                           "compact_ms": a.get("compact", {}).get("ms_per_search"),
                           "pairs": a.get("mlm", {}).get("pairs"), "same_pair_set": a.get("same_pair_set"),
                           "speedup_mlm_vs_compact": a.get("speedup_mlm_vs_compact")}
    sc = line.get("scatter")
    if sc:
        out["scatter"] = dict(_pick(sc, "ms_per_call", "value", "unit", "repeatable"),
                              roofline_frac=sc.get("roofline", {}).get("frac"),
                              cpu_bit_identical=sc.get("cpu_baseline", {}).get("bit_identical"))
    f = line.get("f64")
    if f:
        out["f64"] = dict(_pick(f, "ms_per_search", "value", "unit", "pairs"),
                          pairs_match=f.get("cpu_baseline", {}).get("pairs_match"),
                          indptr_match=f.get("cpu_baseline", {}).get("indptr_match"))
    fs = line.get("fixed_support")
    if fs:
        out["fixed_support"] = _pick(fs, "supports_array_ms", "support_override_ms", "speedup", "same_csr")
    sv = line.get("served")
    if sv:
        out["served"] = {"speedup_vs_per_call": sv.get("speedup_vs_per_call"),
                         "served_capacity": _pick(sv.get("served_capacity", {}), "value", "unit", "mean_batch"),
                         "served": _pick(sv.get("served", {}), "value", "p50_ms", "p99_ms", "requests"),
                         "per_call": _pick(sv.get("per_call", {}), "value", "p50_ms", "p99_ms"),
                         "tuning": sv.get("tuning", {}).get("chosen")}
    return out


def profile_searches(n):
    """n eager searches of the 1M-point workload through the public engine, nothing else."""
    import torch
    from torchcompactradius_b200.search import compact_search
    pos, sup = make_workload()
    p, h = pos.cuda(), sup.cuda()
    for _ in range(n):
        (col, _, _), _ = compact_search(p, h, p, h, [-1.0] * 3, [1.0] * 3, 0, "symmetric", 4096, "csr", True)
    torch.cuda.synchronize()
    print(json.dumps({"profile_searches": n, "pairs": int(col.numel())}))
    return 0


def profile_scatter(n):
    """One search of the 1M-point workload (COO) and n scatter_sum calls over its rows."""
    import torch

    import torchcompactradius_b200 as tcr
    pos, sup = make_workload()
    p, h = pos.cuda(), sup.cuda()
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.zeros(3, dtype=torch.bool), 3)
    adj = tcr.radiusSearch(tcr.PointCloud(p, h), None, mode="symmetric", domain=dom, algorithm="compact", format="coo")
    vals = torch.rand(adj.row.numel(), device="cuda")
    for _ in range(n):
        s = tcr.scatter_sum(vals, adj.row, 0, None, p.shape[0])
    torch.cuda.synchronize()
    print(json.dumps({"profile_scatter": n, "pairs": int(adj.row.numel()), "checksum": float(s.double().sum())}))
    return 0


def profile_f64(n):
    """n float64 searches of the 1M-point workload through the public API, nothing else."""
    import torch

    import torchcompactradius_b200 as tcr
    pos, sup = make_workload()
    x, h = pos.double().cuda(), sup.double().cuda()
    dom = tcr.DomainDescription(torch.full((3,), -1.0, dtype=torch.float64), torch.full((3,), 1.0, dtype=torch.float64),
                                torch.zeros(3, dtype=torch.bool), 3)
    for _ in range(n):
        adj = tcr.radiusSearch(tcr.PointCloud(x, h), None, mode="symmetric", domain=dom, algorithm="compact",
                               format="csr")
    torch.cuda.synchronize()
    print(json.dumps({"profile_f64": n, "pairs": int(adj.indices.numel())}))
    return 0


def main():
    args = parse()
    if args.profile_searches:
        return profile_searches(args.profile_searches)
    if args.profile_scatter:
        return profile_scatter(args.profile_scatter)
    if args.profile_f64:
        return profile_f64(args.profile_f64)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
