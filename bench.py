"""Benchmark of the B200 SCC pipeline on the social-network workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload social|rmat16|web|batch] [--scale S]

Workload (default "social"): a seeded synthetic directed power-law graph with
the sizes of the Twitter crawl the reference reports on (41,652,231 vertices,
~1.47 B edges after dedupe, ~80 % of the vertices in one giant SCC, the rest
in size-1/2/3 SCCs and a power-law tail of cycles), int32 ids and int64
offsets, generated on the GPU.  One step = one full SCC detection over that
graph (trim, FW/BW, peel, trim-2/3, WCC, mice, canonical labels).

Metric: SCC GTEPS = E / t_step / 1e9 (the reference's convention: whole
pipeline time, graph load excluded).  ``value`` is measured with the CSR
resident in HBM; ``e2e`` through the public API with pinned host buffers,
the H2D upload of the CSR and the D2H copy of the labels inside the timed
region.  Multi-GPU: the single-graph pipeline does not shard; N ranks run N
independent replicas (weak scaling, no collective on the data path).

--impl reference runs the reference's own OpenMP pipeline (its unmodified
CLI, compiled from its sources into oracle/_ref/) on the host cores, on the
same graph written in its int32 binary format.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

REF_PARAMS = ("30", "200", "10", "0.1")  # src/bash_one.sh:4
KERNELS_PER_STEP = 18  # stage kernels enqueued per pipeline run (pipeline.cu: enqueue)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU, torchrun)

def dist_init():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# clocks during the timed region

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None
        self.f = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                   "--format=csv,noheader,nounits", "-lms", "200"],
                                  stdout=self.f, stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.p:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# workloads

def make_graph(workload, seed, scale):
    from ispan_b200 import gen
    if workload == "social":
        g = gen.social(seed=seed, scale=scale)
        desc = {"workload": "social-network SCC (Twitter-sized synthetic power-law digraph)",
                "vertices": g.V, "edges": g.E, "giant_frac_target": 0.80, "offsets": "int64",
                "ids": "int32", "seed": seed, "scale": scale}
    elif workload == "rmat16":
        g = gen.rmat(16, 16, seed)
        desc = {"workload": "R-MAT scale 16 edge factor 16 (a,b,c)=(.57,.19,.19)", "vertices": g.V,
                "edges": g.E, "offsets": "int64", "ids": "int32", "seed": seed}
    elif workload == "web":
        g = gen.web(seed=seed, scale=scale)
        desc = {"workload": "web-crawl SCC (giant 35%, trivial 50%, planted mid-size SCCs in a DAG)",
                "vertices": g.V, "edges": g.E, "offsets": "int64", "ids": "int32", "seed": seed, "scale": scale}
    else:
        raise SystemExit(f"unknown workload {workload}")
    return g, desc


def alg_bytes(st, o=8, s=1):
    """Algorithmic bytes of the FW and BW searches: 4 B per edge of the
    reached set, two offsets and one status byte per reached vertex."""
    fw = 4 * st["fw_edges"] + 2 * o * st["fw_size"] + s * st["fw_size"]
    bw = 4 * st["bw_edges"] + 2 * o * st["giant_size"] + s * st["giant_size"]
    return fw, bw


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get(kernel)
    return None


# ---------------------------------------------------------------------------
# the reference's own CLI on the host

def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def write_ref_files(g, d):
    """The graph in the reference's binary format (int32 offsets and ids)."""
    from ispan_b200.graphs import write_bin
    csr = g.to_host(np.int32)
    return write_bin(csr, d, np.int32), csr


def run_reference_cli(paths, threads, runs, timeout):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not os.path.exists(oracle.REF_BIN):
        raise FileNotFoundError("oracle/_ref/ispan not built (make -C oracle ref where the reference tree is)")
    cmd = [oracle.REF_BIN, *paths, str(threads), *REF_PARAMS, str(runs)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference exited {r.returncode}: {r.stderr[-300:]}")
    totals = [float(line.split(",")[1]) for line in r.stdout.splitlines() if line.startswith("total time,")]
    if not totals:
        raise RuntimeError("reference printed no per-run total time")
    return totals, r.stdout


def tmpdir_for(nbytes):
    for base in ("/dev/shm", tempfile.gettempdir()):
        try:
            if shutil.disk_usage(base).free > nbytes * 1.2:
                return tempfile.mkdtemp(dir=base, prefix="ispan_ref_")
        except OSError:
            pass
    return tempfile.mkdtemp(prefix="ispan_ref_")


def host_mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


REF_MAX_E = (1 << 31) - 1  # the reference keeps int32 offsets (src/util.h, src/graph.cpp:10-13)


def cpu_sample_graph(workload, seed, scale, E):
    """The graph the reference CLI can run: the workload itself, or, when its
    edge count needs int64 offsets, the same generator at a scale that fits
    int32 offsets (about 2^30 edges)."""
    if E <= REF_MAX_E:
        return None, scale
    s = scale * (1 << 30) / E
    g2, _ = make_graph(workload, seed, s)
    return g2, s


def cpu_baseline(g, args):
    try:
        g2, s = cpu_sample_graph(args.workload, args.seed, args.scale, g.E)
        gg = g2 or g
        cap = 600 if g2 is None else 180
        try:
            totals = reference_timing(gg, args.ref_steps, 1, timeout=cap)
        except subprocess.TimeoutExpired:
            return {"value": None, "unit": "GTEPS", "cores": host_threads(), "kind": "reference",
                    "sample": f"unavailable: the reference CLI did not finish {args.ref_steps + 1} runs in {cap} s on "
                              f"{gg.V} vertices / {gg.E} edges (its mice stage, one serial forward-backward search "
                              f"per WCC, is superlinear on DAGs of planted SCCs)"}
        finally:
            if g2 is not None:
                g2.free()
        cms = statistics.mean(totals)
        sample = f"the full graph, {len(totals)} runs of the reference CLI after 1 warm-up run" if g2 is None else \
            (f"the same generator at scale {s:.4f} ({gg.V} vertices, {gg.E} edges: the reference's int32 offsets "
             f"cannot hold {g.E} edges), {len(totals)} runs after 1 warm-up run")
        return {"value": gg.E / (cms / 1e3) / 1e9, "unit": "GTEPS", "cores": host_threads(), "kind": "reference",
                "ms_per_run": cms, "sample": sample}
    except Exception as e:  # noqa: BLE001
        return {"value": None, "unit": "GTEPS", "cores": host_threads(), "kind": "reference",
                "sample": f"unavailable: {str(e).splitlines()[0][:200]}"}


def reference_timing(g, steps, warmup, timeout=900):
    """Per-run totals (ms) of the reference's unmodified CLI on this graph."""
    d = tmpdir_for(8 * g.E + 8 * g.V)
    try:
        paths, _ = write_ref_files(g, d)
        totals, out = run_reference_cli(paths, host_threads(), warmup + steps, timeout)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return totals[warmup:] if len(totals) > warmup else totals


def reference_per_graph(graphs_host, cap_s):
    """The reference CLI once per graph (one warm-up + one timed run each),
    each capped at cap_s seconds of wall time; returns (times_ms, capped)."""
    times, capped = [], 0
    for csr in graphs_host:
        d = tmpdir_for(8 * csr.E + 8 * csr.V + (1 << 20))
        try:
            from ispan_b200.graphs import write_bin
            paths = write_bin(csr, d, np.int32)
            try:
                totals, _ = run_reference_cli(paths, host_threads(), 2, cap_s)
                times.append(totals[-1])
            except subprocess.TimeoutExpired:
                times.append(cap_s * 1e3)
                capped += 1
        finally:
            shutil.rmtree(d, ignore_errors=True)
    return times, capped


def batch_sample_host(args, n, seed_shift=0):
    """A seeded sample of the batch workload's graphs as host CSRs (int32)."""
    from ispan_b200 import gen
    from ispan_b200.graphs import CSR
    nseg = max(2, int(4096 * args.scale))
    rng = np.random.default_rng(args.seed + 99 + seed_shift)
    pick = sorted(rng.choice(nseg, size=min(n, nseg), replace=False).tolist())
    g = gen.batch(nseg=nseg, vmin=1000, vmax=1_000_000, ef_min=8, ef_max=32, max_cycle=1000, seed=args.seed)
    out = []
    for i in pick:
        fb, fa, bb, ba = g.extract(i, "int32")
        out.append(CSR(int(fb.numel()) - 1, int(fa.numel()), fb.cpu().numpy(), fa.cpu().numpy(),
                       bb.cpu().numpy(), ba.cpu().numpy()))
    g.free()
    return pick, out


def reference_batch_arm(args):
    """Reference arm of the batched/served workloads: the unmodified reference
    CLI once per graph on a seeded sample of the batch's graphs, each capped
    (its mice stage is superlinear on planted-cycle DAGs)."""
    try:
        pick, graphs = batch_sample_host(args, args.ref_graphs)
        times, capped = reference_per_graph(graphs, args.ref_cap)
    except (FileNotFoundError, RuntimeError) as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e).splitlines()[0][:300]}))
        return
    gps = len(times) / (sum(times) / 1e3)
    th = host_threads()
    sample = (f"{len(times)} seeded graphs of the batch workload (ids {pick[:8]}...), the reference CLI once "
              f"per graph after a warm-up run, each capped at {args.ref_cap:.0f} s ({capped} hit the cap and "
              f"count as {args.ref_cap:.0f} s)")
    print(json.dumps({
        "impl": "reference", "metric": "batched graphs/s", "value": gps, "unit": "graphs/s", "n_gpus": 1,
        "steps": len(times), "warmup": 1, "ms_per_step": sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"{args.workload} SCC, per-graph reference runs on a sample", "scale": args.scale,
                   "parallelism": f"openmp{th}"},
        "cpu_baseline": {"value": gps, "unit": "graphs/s", "cores": th, "kind": "reference", "sample": sample},
        "e2e": {"value": gps, "unit": "graphs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# ---------------------------------------------------------------------------
# batched form: many independent graphs in one set of stage launches

def bench_batch(args, ws, rank, local):
    """4096 graphs (V log-uniform in [1e3, 1e6]; even: R-MAT-like with edge
    factor 8..32, odd: random DAGs of planted cycles of length 2..1000) as one
    disjoint union, detected with one ispan_scc_run_batch per step; compared
    with the plain pipeline launched per graph on a seeded sample of the same
    graphs.  Multi-GPU: each rank runs its own batch (graphs shard by rank,
    no collective)."""
    import torch
    from ispan_b200 import Context, gen
    nseg = max(2, int(4096 * args.scale))
    g = gen.batch(nseg=nseg, vmin=1000, vmax=1_000_000, ef_min=8, ef_max=32, max_cycle=1000,
                  seed=args.seed + 1000 * rank)
    vb = g.vbase
    log(f"[rank {rank}] batch: {nseg} graphs, V={g.V} E={g.E}")
    fwb, fwa, bwb, bwa = g.ptrs
    stream = torch.cuda.Stream()
    ctx = Context(g.V, g.E)
    ctx.set_stream(stream)
    labels = torch.empty(g.V, dtype=torch.int32, device="cuda")
    from ispan_b200 import autotune
    tp = autotune.apply(ctx, g.V, g.E, nseg)
    tun = dict(alpha=tp["alpha"], beta=tp["beta"], gamma=tp["gamma"])
    run = lambda: ctx.run_raw(g.V, g.E, fwb, fwa, bwb, bwa, 8, labels, vbase=vb, stage_times=True, **tun)  # noqa: E731
    for _ in range(args.warmup):
        run()
    torch.cuda.synchronize()
    barrier(ws)
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        _, st = run()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), ws) / args.steps
    # the plain pipeline per graph, on a seeded sample of the graphs
    rng = np.random.default_rng(args.seed)
    sample = sorted(rng.choice(nseg, size=min(nseg, 48), replace=False).tolist())
    maxv = int(max(vb[i + 1] - vb[i] for i in sample))
    plain = None
    per_ms, mism = [], 0
    lab_host = labels.cpu().numpy()
    for i in sample:
        fb, fa, bb, ba = g.extract(i, "int64")
        if plain is None:
            plain = Context(maxv, max(int(fa.numel()), 1) * 4)
            plain.set_stream(stream)
        if fa.numel() > plain.max_E:
            plain.close()
            plain = Context(maxv, int(fa.numel()) * 2)
            plain.set_stream(stream)
        out = torch.empty(fb.numel() - 1, dtype=torch.int32, device="cuda")
        tpp = autotune.apply(plain, int(fb.numel()) - 1, int(fa.numel()))  # tuned like the batch
        tpl = dict(alpha=tpp["alpha"], beta=tpp["beta"], gamma=tpp["gamma"])
        plain.run(fb, fa, bb, ba, labels_out=out, **tpl)  # warm (captures the graph for this shape)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        plain.run(fb, fa, bb, ba, labels_out=out, **tpl)
        a1.record(stream)
        torch.cuda.synchronize()
        per_ms.append(a0.elapsed_time(a1))
        # batching changes the schedule, not the answer
        mism += int((out.cpu().numpy() + vb[i] != lab_host[vb[i]:vb[i + 1]]).sum())
    plain_gps = 1000.0 / statistics.mean(per_ms)
    gps = ws * nseg / (ms / 1e3)
    # the reference CLI per graph on the first sampled graphs (capped)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from ispan_b200.graphs import CSR
        hosts = []
        for i in sample[:args.ref_graphs]:
            a, b_, c_, d_ = g.extract(i, "int32")
            hosts.append(CSR(int(a.numel()) - 1, int(b_.numel()), a.cpu().numpy(), b_.cpu().numpy(),
                             c_.cpu().numpy(), d_.cpu().numpy()))
        try:
            times, capped = reference_per_graph(hosts, args.ref_cap)
            cpu = {"value": len(times) / (sum(times) / 1e3), "unit": "graphs/s", "cores": host_threads(),
                   "kind": "reference",
                   "sample": f"{len(times)} of the sampled graphs, the reference CLI once per graph after a "
                             f"warm-up run, capped at {args.ref_cap:.0f} s ({capped} capped)"}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "graphs/s", "cores": host_threads(), "kind": "reference",
                   "sample": f"unavailable: {str(e).splitlines()[0][:200]}"}
    # end to end: the union from pinned host memory through the batched call
    e2e = None
    h2d = 2 * (g.V + 1) * 8 + 2 * g.E * 4
    if args.e2e_steps > 0 and host_mem_available() < 1.25 * h2d:
        e2e = {"value": None, "unit": "graphs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4,
               "unavailable": f"host memory: {host_mem_available() / 1e9:.0f} GB available"}
    elif args.e2e_steps > 0:
        hfb, hfa, hbb, hba = g.to_pinned()
        hlab = torch.empty(g.V, dtype=torch.int32, pin_memory=True)
        np_args = [t.numpy() for t in (hfb, hfa, hbb, hba)]
        g.free()
        torch.cuda.empty_cache()
        ctx.run(*np_args, V=g.V, labels_out=hlab.numpy(), vbase=vb)  # warm (upload buffers)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            ctx.run(*np_args, V=g.V, labels_out=hlab.numpy(), vbase=vb)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1), ws) / args.e2e_steps
        e2e = {"value": ws * nseg / (ems / 1e3), "unit": "graphs/s", "ms_per_step": ems,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4}
    if rank == 0:
        print(json.dumps({
            "metric": "batched graphs/s", "value": gps, "unit": "graphs/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "batched SCC: 4096 independent graphs, V log-uniform [1e3,1e6], half R-MAT "
                                   "(ef 8-32) half planted-cycle DAGs, one launch sequence per batch",
                       "graphs": nseg, "vertices": g.V, "edges": g.E, "scale": args.scale,
                       "parallelism": "graphs sharded by rank" if ws > 1 else "single-gpu"},
            "edges_per_s": ws * g.E / (ms / 1e3), "gteps": ws * g.E / (ms / 1e3) / 1e9,
            "latency_ms": {"p50": ms, "p99": ms, "note": "every graph of a batch completes with the batch"},
            "plain_per_graph": {"graphs_sampled": len(sample), "ms_mean": statistics.mean(per_ms),
                                "ms_p50": float(np.percentile(per_ms, 50)), "ms_p99": float(np.percentile(per_ms, 99)),
                                "graphs_per_s": plain_gps},
            "batched_over_plain": gps / ws / plain_gps,
            "labels_batched_vs_plain_mismatches": mism,
            "e2e": e2e, "cpu_baseline": cpu,
            "gpu_launches": KERNELS_PER_STEP * args.steps, "clocks": clk,
            "scc": {k: st[k] for k in ("scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3", "n_mice_scc",
                                       "local_wcc", "color_rounds")},
            "stage_ms": {"total": st["stage_ms"][3], "trim": st["stage_ms"][0], "elephant": st["stage_ms"][1],
                         "mice": st["stage_ms"][2]}}))
    ctx.close()
    if plain is not None:
        plain.close()


def bench_served(args, ws, rank, local):
    """Served form: Poisson arrivals (--rate requests/s for --duration s)
    replayed from a seeded trace, each request one graph drawn from a pool of
    device-resident graphs (V log-uniform in [64, 5e5] times edge factor 8..32,
    so E is roughly log-uniform in [1e3, 1e7]; half R-MAT-like, half
    planted-cycle DAGs), submitted one at a time to an ispan_server holding a
    64 GiB device-memory budget.  Latency runs from the scheduled arrival to
    the request's labels being written.  Multi-GPU: each rank serves its own
    trace (requests shard by rank, no collective)."""
    import torch
    from ispan_b200 import Context, Server, gen
    pool_n = args.pool
    g = gen.batch(nseg=pool_n, vmin=64, vmax=500_000, ef_min=8, ef_max=32, max_cycle=1000,
                  seed=args.seed + 1000 * rank)
    pool = [g.extract(i, "int32") for i in range(pool_n)]
    pool_E = np.array([int(p[1].numel()) for p in pool], np.int64)
    pool_V = np.array([int(p[0].numel()) - 1 for p in pool], np.int64)
    g.free()
    outs = [torch.empty(max(int(v), 1), dtype=torch.int32, device="cuda") for v in pool_V]
    torch.cuda.synchronize()
    log(f"[rank {rank}] served: pool {pool_n} graphs, E mean {pool_E.mean():.0f}, max {pool_E.max()}")
    rng = np.random.default_rng(args.seed + 7 * rank)
    n_req = int(args.rate * args.duration)
    arrive = np.cumsum(rng.exponential(1.0 / args.rate, n_req))
    pick = rng.integers(0, pool_n, n_req)
    srv = Server(hbm_budget_bytes=64 << 30, max_batch_graphs=4096)
    # warm-up: every pool graph once
    for _ in range(args.warmup):
        ts = [srv.submit(*pool[i], outs[i]) for i in range(pool_n)]
        for t in ts:
            srv.wait(t)
    c0 = srv.counters()
    barrier(ws)
    clocks = Clocks(local)
    clocks.start()
    t0 = time.monotonic_ns() + 20_000_000
    tickets = []
    for k in range(n_req):
        target = t0 + int(arrive[k] * 1e9)
        while True:
            d = target - time.monotonic_ns()
            if d <= 0:
                break
            time.sleep(min(d, 2_000_000) / 1e9)
        tickets.append((srv.submit(*pool[pick[k]], outs[pick[k]]), target))
    infos = [(srv.wait(t), target) for t, target in tickets]
    clk = clocks.stop()
    c1 = srv.counters()
    lat = np.array([(inf["t_done_ns"] - target) / 1e6 for inf, target in infos])
    bsz = np.array([inf["batch_graphs"] for inf, _ in infos])
    end = max(inf["t_done_ns"] for inf, _ in infos)
    wall_s = max_over_ranks((end - t0) / 1e9, ws)
    gps = ws * n_req / wall_s
    eps = ws * float(pool_E[pick].sum()) / wall_s
    # served results equal the graph run alone (a seeded sample of the pool)
    chk = sorted(rng.choice(pool_n, size=min(pool_n, 16), replace=False).tolist())
    mism = 0
    with Context(int(pool_V[chk].max()), int(max(pool_E[chk].max(), 1))) as ctx:
        for i in chk:
            alone, _ = ctx.run(*pool[i])
            mism += int((alone != outs[i][:pool_V[i]]).sum())
    srv.close()
    if rank == 0:
        print(json.dumps({
            "metric": "served graphs/s", "value": gps, "unit": "graphs/s", "n_gpus": ws, "steps": n_req,
            "warmup": args.warmup, "ms_per_step": 1000.0 / gps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "served SCC: Poisson arrivals, one graph per request from a device-resident "
                                   "pool (E ~ log-uniform 1e3-1e7, half R-MAT half planted-cycle DAGs), "
                                   "continuous batching, 64 GiB admission budget",
                       "rate_per_s": args.rate, "duration_s": args.duration, "requests": n_req,
                       "pool_graphs": pool_n, "parallelism": "requests sharded by rank" if ws > 1 else "single-gpu"},
            "offered_edges_per_s": float(pool_E[pick].sum()) / args.duration,
            "edges_per_s": eps, "achieved_over_offered": (n_req / wall_s) / args.rate,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max()), "from": "scheduled arrival to labels written"},
            "batches": c1["batches"] - c0["batches"], "batch_graphs_mean": float(bsz.mean()),
            "busy_frac": (c1["busy_ns"] - c0["busy_ns"]) / max(1, end - t0),
            "labels_served_vs_alone_mismatches": mism,
            "gpu_launches": (KERNELS_PER_STEP + 3) * (c1["batches"] - c0["batches"]), "clocks": clk}))


# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="social")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-steps", type=int, default=2, help="reference runs for cpu_baseline")
    ap.add_argument("--ref-graphs", type=int, default=8, help="batch/served: graphs the reference runs")
    ap.add_argument("--ref-cap", type=float, default=20.0, help="batch/served: seconds per reference graph")
    ap.add_argument("--rate", type=float, default=2000.0, help="served: requests per second")
    ap.add_argument("--duration", type=float, default=10.0, help="served: seconds of arrivals")
    ap.add_argument("--pool", type=int, default=256, help="served: distinct graphs in the request pool")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warmup raised to 3 (timing rule)")
        args.warmup = 3

    ws, rank, local = dist_init()
    import torch

    if args.workload in ("batch", "served") and args.impl == "ours":
        (bench_batch if args.workload == "batch" else bench_served)(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload in ("batch", "served"):
            return reference_batch_arm(args)
        g, desc = make_graph(args.workload, args.seed, args.scale)
        g2, s = cpu_sample_graph(args.workload, args.seed, args.scale, g.E)
        sample_note = ""
        if g2 is not None:  # the reference's int32 offsets cannot hold the full graph
            g.free()
            g = g2
            sample_note = f"; the same generator at scale {s:.4f} (int32 offsets of the reference)"
        try:
            totals = reference_timing(g, args.steps, args.warmup)
        except (FileNotFoundError, RuntimeError, subprocess.TimeoutExpired) as e:
            print(json.dumps({"impl": "reference", "unavailable": str(e).splitlines()[0][:300]}))
            return
        ms = statistics.mean(totals)
        val = g.E / (ms / 1e3) / 1e9
        th = host_threads()
        desc = dict(desc, sampled_vertices=g.V, sampled_edges=g.E) if g2 is not None else desc
        print(json.dumps({
            "impl": "reference", "metric": "SCC GTEPS", "value": val, "unit": "GTEPS", "n_gpus": ws,
            "steps": len(totals), "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": dict(desc, parallelism=f"openmp{th}"),
            "cpu_baseline": {"value": val, "unit": "GTEPS", "cores": th, "kind": "reference",
                             "sample": f"full graph, {len(totals)} timed runs of the reference CLI "
                                       f"(src/scc_main.cpp) after {args.warmup} warm-up runs{sample_note}"},
            "e2e": {"value": val, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    from ispan_b200 import Context
    g, desc = make_graph(args.workload, args.seed, args.scale)
    log(f"[rank {rank}] graph V={g.V} E={g.E}")
    stream = torch.cuda.Stream()
    ctx = Context(g.V, g.E)
    ctx.set_stream(stream)
    fb, fa, bb, ba = g.ptrs  # the generator's device arrays, no copy
    labels = torch.empty(g.V, dtype=torch.int32, device="cuda")
    from ispan_b200 import autotune
    tp = autotune.apply(ctx, g.V, g.E)  # the tuned launch parameters of this graph's shape class
    tun = dict(alpha=tp["alpha"], beta=tp["beta"], gamma=tp["gamma"])
    run = lambda: ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, labels, stage_times=True, **tun)  # noqa: E731
    for _ in range(args.warmup):
        _, st = run()
    torch.cuda.synchronize()

    # ---- timed region: K steps, inputs resident in HBM (12 GB > L2) ----
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    stages = []
    ev[0].record(stream)
    for k in range(args.steps):
        _, st = run()
        ev[k + 1].record(stream)
        stages.append(st)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    total_ms_max = max_over_ranks(total_ms, ws)
    ms_per_step = total_ms_max / args.steps
    value = ws * g.E / (ms_per_step / 1e3) / 1e9

    # roofline of the dominant kernel (the longer of the FW and BW searches);
    # the degree sums of the reached sets come from one extra, untimed run
    _, st_x = ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, labels, exact_stats=True, **tun)
    st = dict(st, fw_edges=st_x["fw_edges"], bw_edges=st_x["bw_edges"])
    fw_b, bw_b = alg_bytes(st)
    fw_ms = statistics.mean(s["stage_ms"][7] for s in stages)
    bw_ms = statistics.mean(s["stage_ms"][8] for s in stages)
    kern, by, kms = ("k_bfs<int64,0> (forward reach)", fw_b, fw_ms) if fw_ms >= bw_ms else \
        ("k_bfs<int64,1> (backward reach)", bw_b, bw_ms)
    peak, peak_kind = measured_peak()
    achieved = by / (kms / 1e3) / 1e9
    # DRAM bytes per launch from the committed ncu capture (social workload only)
    traffic = traffic_from_profiles("k_bfs_fw" if "0>" in kern else "k_bfs_bw") \
        if args.workload == "social" and args.scale == 1.0 else None
    roof = {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
            "alg_bytes_per_launch": by, "kernel_ms": kms}
    stage_mean = [statistics.mean(s["stage_ms"][i] for s in stages) for i in range(16)]

    # exactness at full size: the generator's planted SCC partition
    planted = g.planted_labels()
    planted_mism = None if planted is None else int((labels != planted).sum())
    del planted

    # ---- CPU baseline: the reference's own OpenMP build on this host ----
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(g, args)

    # ---- end to end through the public API with pinned host buffers ----
    e2e = None
    h2d = 2 * (g.V + 1) * 8 + 2 * g.E * 4
    if args.e2e_steps > 0 and host_mem_available() < 1.25 * h2d:
        e2e = {"value": None, "unit": "GTEPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4,
               "unavailable": f"host memory: {host_mem_available() / 1e9:.0f} GB available, "
                              f"{h2d / 1e9:.0f} GB of pinned input needed"}
    elif args.e2e_steps > 0:
        hfb, hfa, hbb, hba = g.to_pinned()
        hlab = torch.empty(g.V, dtype=torch.int32, pin_memory=True)
        np_args = [t.numpy() for t in (hfb, hfa, hbb, hba)]
        g.free()  # the upload buffers take the generator's place on the device
        torch.cuda.empty_cache()
        ctx.run(*np_args, V=g.V, labels_out=hlab.numpy(), **tun)  # warm (allocates the upload buffers)
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            ctx.run(*np_args, V=g.V, labels_out=hlab.numpy(), **tun)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), ws) / args.e2e_steps
        e2e = {"value": ws * g.E / (e2e_ms / 1e3) / 1e9, "unit": "GTEPS", "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4}

    if rank == 0:
        out = {
            "metric": "SCC GTEPS", "value": value, "unit": "GTEPS", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": dict(desc, parallelism="replicas" if ws > 1 else "single-gpu",
                           l2="inputs larger than L2 (CSR resident in HBM)",
                           tuning=dict(tp, shape_class=autotune.shape_class(g.V, g.E))),
            "e2e": e2e, "gpu_launches": KERNELS_PER_STEP * args.steps, "roofline": roof, "cpu_baseline": cpu,
            "clocks": clk,
            "stage_ms": {"trim": stage_mean[0], "elephant": stage_mean[1], "mice": stage_mean[2],
                         "total": stage_mean[3], "fw": stage_mean[7], "bw": stage_mean[8], "wcc": stage_mean[9],
                         "mice_scc": stage_mean[10], "trim2": stage_mean[5], "trim3": stage_mean[13]},
            "scc": {k: st[k] for k in ("scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3",
                                       "n_mice_scc", "fw_size", "fw_levels", "bw_levels", "color_rounds")},
            "step_ms_min": min(step_ms), "step_ms_max": max(step_ms),
            "labels_vs_planted_partition_mismatches": planted_mism,
        }
        print(json.dumps(out))
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
