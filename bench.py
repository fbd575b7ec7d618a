"""Benchmark of the B200 SCC engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload social|rmat16|web|batch|served] [--scale S] [--no-configs]

Headline workload (default "social"): a seeded synthetic directed power-law
graph with the sizes of the Twitter crawl the reference reports on
(41,652,231 vertices, ~1.47 B edges after dedupe, ~80 % of the vertices in
one giant SCC, the rest in size-1/2/3 SCCs and a power-law tail of cycles),
int32 ids and int64 offsets, generated on the GPU.  One step = one full SCC
detection over that graph (trim, FW/BW, peel, trim-2/3, WCC, mice, canonical
labels).

Metric: SCC GTEPS = E / t_step / 1e9 (the reference's convention: whole
pipeline time, graph load excluded).  ``value`` is measured with the CSR
resident in HBM; ``e2e`` through the public API with pinned host buffers,
the H2D upload of the CSR and the D2H copy of the labels inside the timed
region.  Multi-GPU: the single-graph pipeline does not shard; N ranks run N
independent replicas (weak scaling, no collective on the data path).

At one GPU the line also carries ``configs``, one record per other workload,
each with its own value, stage rooflines, CPU baseline, end-to-end figure and
exactness counters:
  rmat16  R-MAT scale 16, edge factor 16, seeds 1-10 (labels against the
          reference's own answers, tests/golden/rmat16, and the oracle)
  web     700 M vertices / 3.3 B edges, web-crawl shape (labels against the
          generator's planted partition; the CPU baseline is the reference
          built with 64-bit types, run under a wall-clock cap)
  batch   4096 graphs in one launch sequence against the plain pipeline per
          graph (sampled graphs checked against the oracle)
  served  Poisson arrivals at 2,000 requests/s for 60 s, E log-uniform in
          [1e3, 1e7], continuous batching in a 64 GiB budget (sampled
          requests checked against the oracle)
The oracle (oracle/) is used only to check labels and as the CPU baseline,
always outside the timed regions.

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


def checker():
    """The CPU oracle, used only to check labels (never timed, never the
    thing measured)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


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
            return self
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                   "--format=csv,noheader,nounits", "-lms", "200"],
                                  stdout=self.f, stderr=subprocess.DEVNULL)
        return self

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
# measurement helpers

def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p)).get(kernel)
    return None


def stage_roofline(st, stage_ms, V, o):
    """Per-stage algorithmic bytes (one launch over the stage's set) against
    the stage's event-timed device time.  st needs the exact statistics
    (fw_edges, bw_edges, resid_edges, peeled_residual_edges); o is the
    offset width in bytes, 1 status byte per vertex."""
    peak, kind = measured_peak()
    F, S = st["fw_size"], st["giant_size"]
    Q1, Q1d = st["residual"], st["resid_edges"]
    Q2, Q2d = st["peeled_residual"], st["peeled_residual_edges"]
    defs = {
        "trim1_first": ("k_trim1_first", 2 * o * (V + 1) + V, 6),
        "fw": ("k_bfs<.,0>", 4 * st["fw_edges"] + 2 * o * F + F, 7),
        "bw": ("k_bfs<.,1>", 4 * st["bw_edges"] + 2 * o * S + S, 8),
        "trim1_peel": ("k_trim1 (first peel)", 4 * Q1d + 4 * o * Q1 + 4 * Q1, 15),
        "trim2": ("k_trim2", 4 * Q2d + 4 * o * Q2 + 4 * Q2, 5),
        "trim3": ("k_trim3", 4 * Q2d + 4 * o * Q2 + 4 * Q2, 13),
    }
    out = {}
    for name, (kern, by, slot) in defs.items():
        ms = stage_ms[slot]
        gbs = by / (ms / 1e3) / 1e9 if ms > 0 else None
        out[name] = {"kernel": kern, "alg_bytes": int(by), "ms": ms, "achieved_gbs": gbs,
                     "frac": (gbs / peak) if gbs else None}
    out["peak_gbs"] = peak
    out["peak_kind"] = kind
    return out


def mean_stage_ms(stats):
    return [statistics.mean(s["stage_ms"][i] for s in stats) for i in range(16)]


def stage_summary(m):
    return {"trim": m[0], "elephant": m[1], "mice": m[2], "total": m[3], "trim1_first": m[6], "fw": m[7],
            "bw": m[8], "residual_list": m[14], "peel1": m[15], "trim2": m[5], "trim3": m[13], "peel2": m[12],
            "wcc": m[9], "mice_fw_bw": m[10], "colouring": m[11]}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def host_mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def tmpdir_for(nbytes):
    for base in ("/dev/shm", tempfile.gettempdir()):
        try:
            if shutil.disk_usage(base).free > nbytes * 1.2:
                return tempfile.mkdtemp(dir=base, prefix="ispan_ref_")
        except OSError:
            pass
    return tempfile.mkdtemp(prefix="ispan_ref_")


# ---------------------------------------------------------------------------
# the reference's own CLI on the host

REF_MAX_E = (1 << 31) - 1  # the reference keeps int32 offsets (src/util.h:17, src/graph.cpp:10-13)


def write_ref_files(g, d):
    """The graph in the reference's binary format (int32 offsets and ids)."""
    from ispan_b200.graphs import write_bin
    csr = g.to_host(np.int32)
    return write_bin(csr, d, np.int32), csr


def run_reference_cli(paths, threads, runs, timeout):
    oracle = checker()
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
    from ispan_b200.graphs import write_bin
    times, capped = [], 0
    for csr in graphs_host:
        d = tmpdir_for(8 * csr.E + 8 * csr.V + (1 << 20))
        try:
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


# ---------------------------------------------------------------------------
# workloads

def make_graph(workload, seed, scale):
    from ispan_b200 import gen
    if workload == "social":
        g = gen.social(seed=seed, scale=scale)
        desc = {"workload": "social-network SCC (Twitter-sized synthetic power-law digraph)",
                "vertices": g.V, "edges": g.E, "giant_frac_target": 0.80, "offsets": "int64",
                "ids": "int32", "seed": seed, "scale": scale}
    elif workload == "web":
        g = gen.web(seed=seed, scale=scale)
        desc = {"workload": "web-crawl SCC (giant 35%, trivial 50%, planted mid-size SCCs in a DAG)",
                "vertices": g.V, "edges": g.E, "offsets": "int64", "ids": "int32", "seed": seed, "scale": scale}
    else:
        raise SystemExit(f"unknown workload {workload}")
    return g, desc


def cpu_sample_graph(workload, seed, scale, E):
    """The graph the reference CLI can run: the workload itself, or, when its
    edge count needs int64 offsets, the same generator at a scale that fits
    int32 offsets (about 2^30 edges)."""
    if E <= REF_MAX_E:
        return None, scale
    s = scale * (1 << 30) / E
    g2, _ = make_graph(workload, seed, s)
    return g2, s


def cpu_baseline_social(g, args):
    try:
        totals = reference_timing(g, args.ref_steps, 1, timeout=600)
    except Exception as e:  # noqa: BLE001
        return {"value": None, "unit": "GTEPS", "cores": host_threads(), "kind": "reference",
                "sample": f"unavailable: {str(e).splitlines()[0][:200]}"}
    cms = statistics.mean(totals)
    return {"value": g.E / (cms / 1e3) / 1e9, "unit": "GTEPS", "cores": host_threads(), "kind": "reference",
            "ms_per_run": cms, "sample": f"the full graph, {len(totals)} runs of the reference CLI after 1 warm-up run"}


def e2e_plain(ctx, g, stream, steps, tun, ws):
    """End to end through the public API: pinned host CSR uploaded every step,
    labels copied back.  Frees the generator's device arrays first (the
    upload buffers take their place)."""
    import torch
    h2d = 2 * (g.V + 1) * 8 + 2 * g.E * 4
    if host_mem_available() < 1.25 * h2d:
        return {"value": None, "unit": "GTEPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4,
                "unavailable": f"host memory: {host_mem_available() / 1e9:.0f} GB available, "
                               f"{h2d / 1e9:.0f} GB of pinned input needed"}
    hfb, hfa, hbb, hba = g.to_pinned()
    hlab = torch.empty(g.V, dtype=torch.int32, pin_memory=True)
    np_args = [t.numpy() for t in (hfb, hfa, hbb, hba)]
    g.free()
    torch.cuda.empty_cache()
    ctx.run(*np_args, V=g.V, labels_out=hlab.numpy(), **tun)  # warm (allocates the upload buffers)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        ctx.run(*np_args, V=g.V, labels_out=hlab.numpy(), **tun)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), ws) / steps
    del np_args, hfb, hfa, hbb, hba, hlab
    return {"value": ws * g.E / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms_per_step": ms,
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4}


def timed_runs(run, stream, steps, warmup, ws):
    """W untimed runs, then K runs bracketed by a barrier and synchronize,
    CUDA events on the library's stream; returns (ms per step max over
    ranks, per-step ms, stats of each run, clocks)."""
    import torch
    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    local = torch.cuda.current_device()
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    stats = []
    ev[0].record(stream)
    for k in range(steps):
        _, st = run()
        ev[k + 1].record(stream)
        stats.append(st)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
    total = max_over_ranks(ev[0].elapsed_time(ev[-1]), ws)
    return total / steps, step_ms, stats, clk


# ---------------------------------------------------------------------------
# headline: the social-network graph

def bench_social(args, ws, rank, local):
    import torch
    from ispan_b200 import Context, autotune
    g, desc = make_graph("social", args.seed, args.scale)
    log(f"[rank {rank}] social graph V={g.V} E={g.E}")
    stream = torch.cuda.Stream()
    ctx = Context(g.V, g.E)
    ctx.set_stream(stream)
    fb, fa, bb, ba = g.ptrs  # the generator's device arrays, no copy
    labels = torch.empty(g.V, dtype=torch.int32, device="cuda")
    tp = autotune.apply(ctx, g.V, g.E)  # the tuned launch parameters of this graph's shape class
    tun = dict(alpha=tp["alpha"], beta=tp["beta"], gamma=tp["gamma"])
    run = lambda: ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, labels, stage_times=True, **tun)  # noqa: E731
    ms_per_step, step_ms, stages, clk = timed_runs(run, stream, args.steps, args.warmup, ws)
    value = ws * g.E / (ms_per_step / 1e3) / 1e9
    st = stages[-1]

    # roofline of the dominant kernel (the longer of the FW and BW searches);
    # the degree sums of the reached sets come from one extra, untimed run
    _, st_x = ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, labels, exact_stats=True, **tun)
    m = mean_stage_ms(stages)
    stages_roof = stage_roofline(st_x, m, g.V, 8)
    fw, bw = stages_roof["fw"], stages_roof["bw"]
    kname, sr = ("k_bfs<int64,0> (forward reach)", fw) if fw["ms"] >= bw["ms"] else \
        ("k_bfs<int64,1> (backward reach)", bw)
    peak, peak_kind = measured_peak()
    traffic = traffic_from_profiles("k_bfs_fw" if "0>" in kname else "k_bfs_bw") if args.scale == 1.0 else None
    roof = {"bound": "hbm", "kernel": kname, "achieved": sr["achieved_gbs"], "peak": peak, "unit": "GB/s",
            "frac": sr["frac"], "peak_kind": peak_kind, "traffic": traffic, "alg_bytes_per_launch": sr["alg_bytes"],
            "kernel_ms": sr["ms"]}

    # exactness at full size: the generator's planted SCC partition
    planted = g.planted_labels()
    planted_mism = None if planted is None else int((labels != planted).sum())
    del planted

    cpu = cpu_baseline_social(g, args) if rank == 0 and ws == 1 and not args.no_cpu_baseline else None
    e2e = e2e_plain(ctx, g, stream, args.e2e_steps, tun, ws) if args.e2e_steps > 0 else None
    ctx.close()
    torch.cuda.empty_cache()
    return {
        "metric": "SCC GTEPS", "value": value, "unit": "GTEPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": dict(desc, parallelism="replicas" if ws > 1 else "single-gpu",
                       l2="inputs larger than L2 (CSR resident in HBM)",
                       tuning=dict(tp, shape_class=autotune.shape_class(g.V, g.E))),
        "e2e": e2e, "gpu_launches": KERNELS_PER_STEP * args.steps, "roofline": roof, "cpu_baseline": cpu,
        "clocks": clk, "stage_ms": stage_summary(m), "stage_roofline": stages_roof,
        "scc": {k: st[k] for k in ("scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3",
                                   "n_mice_scc", "fw_size", "fw_levels", "bw_levels", "color_rounds")},
        "step_ms_min": min(step_ms), "step_ms_max": max(step_ms),
        "labels_vs_planted_partition_mismatches": planted_mism,
    }


# ---------------------------------------------------------------------------
# R-MAT scale 16, edge factor 16, seeds 1-10

def bench_rmat16(args):
    """The plain pipeline's small workload: ten seeded R-MAT graphs (scale 16,
    edge factor 16, (a,b,c) = (.57,.19,.19), self-loops and duplicates
    removed, int32 offsets), each run from device memory and end to end from
    pinned host memory; labels checked against the reference's own answers
    (tests/golden/rmat16, canonicalised) and against the oracle."""
    import torch
    from ispan_b200 import Context, graphs as G
    oracle = checker()
    seeds = list(range(1, 11))
    stream = torch.cuda.Stream()
    ctx = Context(1 << 16, 1 << 21)
    ctx.set_stream(stream)
    per, cpu_ms, e2e_ms, st_last = [], [], [], None
    mism_oracle = mism_ref = 0
    roofs = []
    clk = None
    for seed in seeds:
        csr = G.rmat(16, 16, seed)
        d = [torch.from_numpy(a).cuda() for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj)]
        lab = torch.empty(csr.V, dtype=torch.int32, device="cuda")
        run = lambda: ctx.run_raw(csr.V, csr.E, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),  # noqa: E731
                                  d[3].data_ptr(), 4, lab, stage_times=True)
        ms, _, stats, c = timed_runs(run, stream, args.small_steps, args.warmup, 1)
        clk = clk or c
        _, st_x = ctx.run_raw(csr.V, csr.E, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(),
                              4, lab, exact_stats=True)
        roofs.append(stage_roofline(st_x, mean_stage_ms(stats), csr.V, 4))
        st_last = stats[-1]
        got = lab.cpu().numpy()
        exact = oracle.tarjan(csr)
        mism_oracle += int((got != exact).sum())
        fx = os.path.join(ROOT, "tests", "golden", "rmat16", f"s{seed}.npz")
        if os.path.exists(fx):
            z = np.load(fx)
            mism_ref += int((got != oracle.canon_codes(csr, z["ref_codes_t16"])).sum())
        else:
            mism_ref = None if mism_ref in (None, 0) else mism_ref
        per.append({"seed": seed, "V": csr.V, "E": csr.E, "ms": ms})
        # end to end: pinned host CSR in, labels out, through the public API
        pin = [torch.from_numpy(a).pin_memory() for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj)]
        hl = torch.empty(csr.V, dtype=torch.int32, pin_memory=True)
        host = [p.numpy() for p in pin]
        for _ in range(args.warmup):
            ctx.run(*host, V=csr.V, labels_out=hl.numpy())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.small_steps):
            ctx.run(*host, V=csr.V, labels_out=hl.numpy())
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1) / args.small_steps)
        if not args.no_cpu_baseline:
            try:
                cpu_ms.append(statistics.mean(reference_timing_host(csr, 10, 2)))
            except Exception as e:  # noqa: BLE001
                cpu_ms = f"unavailable: {str(e).splitlines()[0][:200]}"
                args.no_cpu_baseline = True
    ctx.close()
    E_mean = statistics.mean(p["E"] for p in per)
    ms_mean = statistics.mean(p["ms"] for p in per)
    gteps = statistics.mean(p["E"] / (p["ms"] / 1e3) / 1e9 for p in per)
    roof = {k: {"kernel": roofs[0][k]["kernel"], "alg_bytes": statistics.mean(r[k]["alg_bytes"] for r in roofs),
                "ms": statistics.mean(r[k]["ms"] for r in roofs),
                "frac": statistics.mean(r[k]["frac"] or 0.0 for r in roofs)}
            for k in ("trim1_first", "fw", "bw", "trim1_peel")}
    if isinstance(cpu_ms, list) and cpu_ms:
        cpu = {"value": statistics.mean(p["E"] / (c / 1e3) / 1e9 for p, c in zip(per, cpu_ms)), "unit": "GTEPS",
               "cores": host_threads(), "kind": "reference", "ms_per_run": statistics.mean(cpu_ms),
               "sample": "each of the ten graphs, 10 runs of the reference CLI after 2 warm-up runs"}
    else:
        cpu = {"value": None, "unit": "GTEPS", "cores": host_threads(), "kind": "reference",
               "sample": cpu_ms if isinstance(cpu_ms, str) else "not run"}
    return {
        "workload": "R-MAT scale 16, edge factor 16, (a,b,c)=(.57,.19,.19), seeds 1-10, int32 offsets",
        "metric": "SCC GTEPS", "value": gteps, "unit": "GTEPS", "ms_per_step": ms_mean, "steps": args.small_steps,
        "warmup": args.warmup, "mean_edges": E_mean, "per_seed": per,
        "roofline": roof, "cpu_baseline": cpu,
        "e2e": {"value": statistics.mean(p["E"] / (e / 1e3) / 1e9 for p, e in zip(per, e2e_ms)), "unit": "GTEPS",
                "ms_per_step": statistics.mean(e2e_ms), "h2d_bytes_per_step": int(2 * 4 * (65537 + E_mean)),
                "d2h_bytes_per_step": 65536 * 4},
        "labels_vs_oracle_mismatches": mism_oracle, "labels_vs_reference_fixture_mismatches": mism_ref,
        "stage_ms": stage_summary(mean_stage_ms([st_last])), "clocks": clk,
        "l2": "the whole graph fits L2 (8 MB); repeated runs hit a warm L2, as the reference's runs hit its caches",
    }


def reference_timing_host(csr, steps, warmup, timeout=300):
    """reference_timing for a host CSR."""
    from ispan_b200.graphs import write_bin
    d = tmpdir_for(8 * csr.E + 8 * csr.V)
    try:
        paths = write_bin(csr, d, np.int32)
        totals, _ = run_reference_cli(paths, host_threads(), warmup + steps, timeout)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return totals[warmup:]
