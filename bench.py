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
KERNELS_PER_STEP = 27  # stage kernels enqueued per pipeline run (pipeline.cu: enqueue; the launch list of the social run)


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
    """End to end through the public API: the pinned host graph uploaded every
    step, labels copied back; timed with the forward CSR alone (the library
    builds the reverse on the device, inside the step) and with both CSRs,
    the record chosen by e2e_pick.  Frees the generator's device arrays first
    (the upload buffers take their place)."""
    import torch
    h2d_fw = (g.V + 1) * 8 + g.E * 4
    h2d = 2 * h2d_fw
    if host_mem_available() < 1.25 * h2d:
        return {"value": None, "unit": "GTEPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4,
                "unavailable": f"host memory: {host_mem_available() / 1e9:.0f} GB available, "
                               f"{h2d / 1e9:.0f} GB of pinned input needed"}
    hfb, hfa, hbb, hba = g.to_pinned()
    hlab = torch.empty(g.V, dtype=torch.int32, pin_memory=True)
    np_args = [t.numpy() for t in (hfb, hfa, hbb, hba)]
    g.free()
    torch.cuda.empty_cache()

    def timed(args):
        ctx.run(*args, V=g.V, labels_out=hlab.numpy(), **tun)  # warm (allocates the upload buffers)
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            ctx.run(*args, V=g.V, labels_out=hlab.numpy(), **tun)
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), ws) / steps

    ms_fw = timed(np_args[:2] + [None, None])
    ms_both = timed(np_args)
    del np_args, hfb, hfa, hbb, hba, hlab
    rec = lambda ms, h: {"value": ws * g.E / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms_per_step": ms,  # noqa: E731
                         "h2d_bytes_per_step": h, "d2h_bytes_per_step": g.V * 4}
    return e2e_pick(g.E, rec(ms_fw, h2d_fw), rec(ms_both, h2d))


def e2e_pick(E, fw, both):
    """The end-to-end record: the forward CSR alone is sent where the library
    sorts the reverse chunk by chunk (each of its eight copy chunks below
    2^31 edges), faster than copying the reverse; beyond that the reverse
    would be placed by atomics, slower than the copy, and both directions
    are sent.  The other form is kept as a sub-record."""
    if (E + 7) // 8 < 2**31 - 1:
        return dict(fw, input="the forward CSR from pinned host memory; the reverse CSR is built on the device "
                              "inside the step", both_directions=both)
    return dict(both, input="both CSRs from pinned host memory", forward_only=fw)


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
    tp = autotune.apply(ctx, g.V, g.E, overrides=args.tuning)  # the tuned launch parameters of this graph's shape class
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
    g.free()
    del labels
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
    if args.tuning:
        ctx.set_tuning(**{k: int(v) for k, v in args.tuning.items()})
    per, cpu_ms, e2e_ms, e2e_ms2, st_last = [], [], [], [], None
    mism_oracle = mism_ref = n_fixtures = 0
    roofs = []
    clk = None
    for seed in seeds:
        csr = G.rmat(16, 16, seed)
        d = [torch.from_numpy(a).cuda() for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj)]
        lab = torch.empty(csr.V, dtype=torch.int32, device="cuda")
        # timed without stage times: reading a dozen event pairs back costs
        # ~35 us per call, a sixth of this graph's run; the stage split comes
        # from five more runs right after
        run = lambda st=False: ctx.run_raw(csr.V, csr.E, d[0].data_ptr(), d[1].data_ptr(),  # noqa: E731
                                           d[2].data_ptr(), d[3].data_ptr(), 4, lab, stage_times=st)
        ms, _, _, c = timed_runs(run, stream, args.small_steps, args.warmup, 1)
        stats = [run(True)[1] for _ in range(5)]
        clk = clk or c
        _, st_x = ctx.run_raw(csr.V, csr.E, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(),
                              4, lab, exact_stats=True)
        roofs.append(stage_roofline(st_x, mean_stage_ms(stats), csr.V, 4))
        st_last = stats[-1]
        got = lab.cpu().numpy()
        exact = oracle.tarjan(csr)
        mism_oracle += int((got != exact).sum())
        fx = os.path.join(ROOT, "tests", "golden", "rmat16", f"s{seed}.npz")
        if os.path.exists(fx):  # the reference's own answer for this seed (16 OpenMP threads)
            z = np.load(fx)
            mism_ref += int((got != oracle.canon_codes(csr, z["ref_codes_t16"])).sum())
            n_fixtures += 1
        per.append({"seed": seed, "V": csr.V, "E": csr.E, "ms": ms})
        # end to end: pinned host CSR in, labels out, through the public API
        pin = [torch.from_numpy(a).pin_memory() for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj)]
        hl = torch.empty(csr.V, dtype=torch.int32, pin_memory=True)
        host = [p.numpy() for p in pin]
        for k, args_k in enumerate((host[:2] + [None, None], host)):  # forward CSR only; both directions
            for _ in range(args.warmup):
                ctx.run(*args_k, V=csr.V, labels_out=hl.numpy())
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.small_steps):
                ctx.run(*args_k, V=csr.V, labels_out=hl.numpy())
            e1.record(stream)
            torch.cuda.synchronize()
            (e2e_ms if k == 0 else e2e_ms2).append(e0.elapsed_time(e1) / args.small_steps)
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
        "e2e": e2e_pick(E_mean, {
            "value": statistics.mean(p["E"] / (e / 1e3) / 1e9 for p, e in zip(per, e2e_ms)), "unit": "GTEPS",
            "ms_per_step": statistics.mean(e2e_ms), "h2d_bytes_per_step": int(4 * (65537 + E_mean)),
            "d2h_bytes_per_step": 65536 * 4}, {
            "value": statistics.mean(p["E"] / (e / 1e3) / 1e9 for p, e in zip(per, e2e_ms2)), "unit": "GTEPS",
            "ms_per_step": statistics.mean(e2e_ms2), "h2d_bytes_per_step": int(2 * 4 * (65537 + E_mean)),
            "d2h_bytes_per_step": 65536 * 4}),
        "labels_vs_oracle_mismatches": mism_oracle, "labels_vs_reference_fixture_mismatches": mism_ref,
        "reference_fixtures_checked": n_fixtures,
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


# ---------------------------------------------------------------------------
# web-crawl graph: 700 M vertices, 3.3 B edges

def wide_reference(g, cap_s, threads):
    """The reference's pipeline built with 64-bit types (oracle/Makefile ref64)
    on the full graph, in a child process (oracle/ref_wide.py), stopped after
    cap_s seconds of pipeline time.  Returns the stage lines it printed: its
    DEBUG progress lines as stages finish, and its OUTPUT_TIME lines if the
    run finished (src/scc_core.cpp:254-914, :1062-1068)."""
    from ispan_b200 import gen
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_wide
    if not os.path.exists(ref_wide.LIB):
        raise FileNotFoundError("oracle/_ref/libispan_ref64.so not built (make -C oracle ref64)")
    need = ref_wide.host_bytes(g.V, g.E)
    avail = host_mem_available()
    if avail < 1.15 * need:
        raise MemoryError(f"host memory: {avail / 1e9:.0f} GB available, the 64-bit reference holds "
                          f"{need / 1e9:.0f} GB")
    d = tmpdir_for(8 * (g.V + 1) * 2 + 4 * g.E * 2)
    logf = os.path.join(d, "ref.log")
    proc = None
    try:
        paths = [os.path.join(d, n) for n in ("fw_beg", "fw_adj", "bw_beg", "bw_adj")]
        mm = [np.memmap(p, dtype=dt, mode="w+", shape=(n,)) for p, dt, n in
              zip(paths, (np.int64, np.int32, np.int64, np.int32), (g.V + 1, g.E, g.V + 1, g.E))]
        rc = gen.lib().ispan_gen_copy(g._h, mm[0].ctypes.data, mm[1].ctypes.data, mm[2].ctypes.data,
                                      mm[3].ctypes.data, 8, 0)
        for m in mm:
            m.flush()
        del mm
        if rc:
            raise RuntimeError(f"ispan_gen_copy failed ({rc})")
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        with open(logf, "w") as lf:
            proc = subprocess.Popen([sys.executable, os.path.join(ROOT, "oracle", "ref_wide.py"), str(g.V),
                                     str(g.E), *paths, str(threads)], stdout=lf, stderr=subprocess.STDOUT, env=env)
            t_load = time.time()
            t_start = None
            while proc.poll() is None:
                time.sleep(0.5)
                if t_start is None and "PIPELINE START" in open(logf).read():
                    t_start = time.time()
                if t_start is None and time.time() - t_load > 900:
                    break
                if t_start is not None and time.time() - t_start > cap_s:
                    break
            finished = proc.poll() == 0
            wall = time.time() - (t_start or t_load)
            if proc.poll() is None:
                proc.kill()
                proc.wait()
        out = open(logf).read()
    finally:
        if proc is not None and proc.poll() is None:
            proc.kill()
        shutil.rmtree(d, ignore_errors=True)
    lines = [ln.strip() for ln in out.splitlines() if "," in ln and any(ch.isdigit() for ch in ln)]
    return finished, wall, lines, out


def bench_web(args):
    import torch
    from ispan_b200 import Context, autotune
    g, desc = make_graph("web", args.seed, args.web_scale)
    log(f"web graph V={g.V} E={g.E}")
    stream = torch.cuda.Stream()
    ctx = Context(g.V, g.E)
    ctx.set_stream(stream)
    fb, fa, bb, ba = g.ptrs
    labels = torch.empty(g.V, dtype=torch.int32, device="cuda")
    tp = autotune.apply(ctx, g.V, g.E, overrides=args.tuning)
    tun = dict(alpha=tp["alpha"], beta=tp["beta"], gamma=tp["gamma"])
    run = lambda: ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, labels, stage_times=True, **tun)  # noqa: E731
    ms, step_ms, stats, clk = timed_runs(run, stream, args.big_steps, args.warmup, 1)
    _, st_x = ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, labels, exact_stats=True, **tun)
    m = mean_stage_ms(stats)
    planted = g.planted_labels()
    mism = None if planted is None else int((labels != planted).sum())
    del planted
    st = stats[-1]
    cpu = None
    if not args.no_cpu_baseline:
        th = host_threads()
        try:
            finished, wall, lines, raw = wide_reference(g, args.web_cpu_cap, th)
            # the OUTPUT_TIME block ends with its "total time" line (the DEBUG
            # build prints a second one, the whole call's time, after it)
            tot = [float(ln.split(",")[1]) for i, ln in enumerate(lines)
                   if ln.startswith("total time,") and i > 0 and lines[i - 1].startswith("mice scc time,")]
            cpu = {"value": g.E / (tot[0] / 1e3) / 1e9 if finished and tot else None, "unit": "GTEPS",
                   "cores": th, "kind": "reference",
                   "sample": ("the full graph, one run of the reference built with its 64-bit typedefs "
                              "(src/util.h:12-21), DEBUG progress prints on"),
                   "finished": finished, "pipeline_wall_s": wall,
                   "dnf_after_s": None if finished else args.web_cpu_cap,
                   "stage_lines": lines[:40]}
            if not lines:
                cpu["log_tail"] = raw[-500:]
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "GTEPS", "cores": th, "kind": "reference",
                   "sample": f"unavailable: {str(e).splitlines()[0][:200]}"}
    e2e = e2e_plain(ctx, g, stream, args.e2e_steps, tun, 1) if args.e2e_steps > 0 else None
    ctx.close()
    g.free()
    del labels
    torch.cuda.empty_cache()
    return {
        "workload": desc["workload"], "vertices": desc["vertices"], "edges": desc["edges"], "scale": args.web_scale,
        "metric": "SCC GTEPS", "value": g.E / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms_per_step": ms,
        "steps": args.big_steps, "warmup": args.warmup, "step_ms_min": min(step_ms), "step_ms_max": max(step_ms),
        "roofline": stage_roofline(st_x, m, g.V, 8), "cpu_baseline": cpu, "e2e": e2e,
        "labels_vs_planted_partition_mismatches": mism, "stage_ms": stage_summary(m), "clocks": clk,
        "scc": {k: st[k] for k in ("scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3", "n_mice_scc",
                                   "residual", "local_wcc", "color_rounds", "fw_levels", "bw_levels")},
        "l2": "inputs larger than L2 (37 GB CSR resident in HBM)",
    }


# ---------------------------------------------------------------------------
# batched form: many independent graphs in one set of stage launches

def bench_batch(args, ws, rank, local):
    """4096 graphs (V log-uniform in [1e3, 1e6]; even: R-MAT-like with edge
    factor 8..32, odd: random DAGs of planted cycles of length 2..1000) as one
    disjoint union, detected with one ispan_scc_run_batch per step; compared
    with the plain pipeline launched per graph on a seeded sample of the same
    graphs, and every sampled graph's labels checked against the oracle.
    Multi-GPU: each rank runs its own batch (graphs shard by rank, no
    collective)."""
    import torch
    from ispan_b200 import Context, autotune, gen
    from ispan_b200.graphs import CSR
    oracle = checker()
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
    tp = autotune.apply(ctx, g.V, g.E, nseg, overrides=args.tuning)
    tun = dict(alpha=tp["alpha"], beta=tp["beta"], gamma=tp["gamma"])
    run = lambda: ctx.run_raw(g.V, g.E, fwb, fwa, bwb, bwa, 8, labels, vbase=vb, stage_times=True, **tun)  # noqa: E731
    ms, step_ms, stats, clk = timed_runs(run, stream, args.big_steps, args.warmup, ws)
    st = stats[-1]
    # the plain pipeline per graph, on a seeded sample of the graphs; each
    # sampled graph's batched labels also checked against the oracle
    rng = np.random.default_rng(args.seed)
    sample = sorted(rng.choice(nseg, size=min(nseg, 48), replace=False).tolist())
    maxv = int(max(vb[i + 1] - vb[i] for i in sample))
    plain = None
    per_ms, mism, mism_oracle, hosts = [], 0, 0, []
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
        tpp = autotune.apply(plain, int(fb.numel()) - 1, int(fa.numel()), overrides=args.tuning)  # tuned like the batch
        tpl = dict(alpha=tpp["alpha"], beta=tpp["beta"], gamma=tpp["gamma"])
        plain.run(fb, fa, bb, ba, labels_out=out, **tpl)  # warm
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        plain.run(fb, fa, bb, ba, labels_out=out, **tpl)
        a1.record(stream)
        torch.cuda.synchronize()
        per_ms.append(a0.elapsed_time(a1))
        mine = lab_host[vb[i]:vb[i + 1]] - vb[i]
        mism += int((out.cpu().numpy() != mine).sum())  # batching changes the schedule, not the answer
        csr = CSR(int(fb.numel()) - 1, int(fa.numel()), fb.cpu().numpy(), fa.cpu().numpy(), bb.cpu().numpy(),
                  ba.cpu().numpy())
        mism_oracle += int((oracle.tarjan(csr) != mine).sum())
        if len(hosts) < args.ref_graphs:
            hosts.append(csr)
    plain_gps = 1000.0 / statistics.mean(per_ms)
    gps = ws * nseg / (ms / 1e3)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            times, capped = reference_per_graph(hosts, args.ref_cap)
            cpu = {"value": len(times) / (sum(times) / 1e3), "unit": "graphs/s", "cores": host_threads(),
                   "kind": "reference",
                   "sample": f"{len(times)} of the sampled graphs, the reference CLI once per graph after a "
                             f"warm-up run, capped at {args.ref_cap:.0f} s ({capped} capped)"}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "graphs/s", "cores": host_threads(), "kind": "reference",
                   "sample": f"unavailable: {str(e).splitlines()[0][:200]}"}
    del hosts
    # end to end: the union from pinned host memory through the batched call
    # (the forward CSR, its reverse built on the device; and both directions)
    e2e = None
    h2d_fw = (g.V + 1) * 8 + g.E * 4
    h2d = 2 * h2d_fw
    if args.e2e_steps > 0 and host_mem_available() < 1.25 * h2d:
        e2e = {"value": None, "unit": "graphs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": g.V * 4,
               "unavailable": f"host memory: {host_mem_available() / 1e9:.0f} GB available"}
    elif args.e2e_steps > 0:
        hfb, hfa, hbb, hba = g.to_pinned()
        hlab = torch.empty(g.V, dtype=torch.int32, pin_memory=True)
        np_args = [t.numpy() for t in (hfb, hfa, hbb, hba)]
        g.free()
        torch.cuda.empty_cache()

        def timed(a):
            ctx.run(*a, V=g.V, labels_out=hlab.numpy(), vbase=vb)  # warm (upload buffers)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.e2e_steps):
                ctx.run(*a, V=g.V, labels_out=hlab.numpy(), vbase=vb)
            e1.record(stream)
            torch.cuda.synchronize()
            return max_over_ranks(e0.elapsed_time(e1), ws) / args.e2e_steps

        ems_fw = timed(np_args[:2] + [None, None])
        ems_both = timed(np_args)
        rec = lambda ms, h: {"value": ws * nseg / (ms / 1e3), "unit": "graphs/s", "ms_per_step": ms,  # noqa: E731
                             "h2d_bytes_per_step": h, "d2h_bytes_per_step": g.V * 4}
        e2e = e2e_pick(g.E, rec(ems_fw, h2d_fw), rec(ems_both, h2d))
        del np_args, hfb, hfa, hbb, hba, hlab
    ctx.close()
    if plain is not None:
        plain.close()
    g.free()
    torch.cuda.empty_cache()
    return {
        "metric": "batched graphs/s", "value": gps, "unit": "graphs/s", "n_gpus": ws, "steps": args.big_steps,
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
        "labels_batched_vs_plain_mismatches": mism, "labels_vs_oracle_mismatches": mism_oracle,
        "graphs_checked_against_oracle": len(sample),
        "e2e": e2e, "cpu_baseline": cpu,
        "gpu_launches": KERNELS_PER_STEP * args.big_steps, "clocks": clk,
        "step_ms_min": min(step_ms), "step_ms_max": max(step_ms),
        "scc": {k: st[k] for k in ("scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3", "n_mice_scc",
                                   "local_wcc", "color_rounds")},
        "stage_ms": stage_summary(mean_stage_ms(stats)),
    }


# ---------------------------------------------------------------------------
# served form: Poisson arrivals, continuous batching

def served_pool(args, rank):
    """Device-resident request graphs: R-MAT-like graphs (edge factor 8..32)
    and random DAGs of planted cycles (lengths 2..1000), pool/2 of each kind,
    sized so that their edge counts cover [1e3, 1e7]; int32 offsets."""
    import torch
    from ispan_b200 import gen
    half = max(1, args.pool // 2)
    pool, kind = [], []
    # even graphs of a batch are R-MAT-like, odd ones planted-cycle DAGs (E ~ 3 V)
    for k, (vmin, vmax, efmin, efmax) in enumerate(((40, 1_300_000, 8, 32), (330, 3_400_000, 8, 8))):
        g = gen.batch(nseg=2 * half, vmin=vmin, vmax=vmax, ef_min=efmin, ef_max=efmax, max_cycle=1000,
                      seed=args.seed + 7919 * k + 1000 * rank)
        for i in range(k, 2 * half, 2):
            pool.append(g.extract(i, "int32"))
            kind.append(k)
        g.free()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return pool, np.array(kind)


def bench_served(args, ws, rank, local):
    """Served form: Poisson arrivals (--rate requests/s for --duration s)
    replayed from a seeded trace.  Each request is a device-resident graph
    whose edge count is drawn log-uniform in [1e3, 1e7] (the pool graph of the
    drawn kind -- R-MAT-like or planted-cycle DAG, 50/50 -- nearest to it),
    submitted to an ispan_server holding a 64 GiB device-memory budget.
    Latency runs from the scheduled arrival to the request's labels being
    written.  Multi-GPU: each rank serves its own trace (requests shard by
    rank, no collective)."""
    import torch
    from ispan_b200 import Context, Server
    from ispan_b200.graphs import CSR
    oracle = checker()
    pool, kind = served_pool(args, rank)
    pool_n = len(pool)
    pool_E = np.array([int(p[1].numel()) for p in pool], np.int64)
    pool_V = np.array([int(p[0].numel()) - 1 for p in pool], np.int64)
    outs = [torch.empty(max(int(v), 1), dtype=torch.int32, device="cuda") for v in pool_V]
    torch.cuda.synchronize()
    rng = np.random.default_rng(args.seed + 7 * rank)
    n_req = int(args.rate * args.duration)
    arrive = np.cumsum(rng.exponential(1.0 / args.rate, n_req))
    want_k = rng.integers(0, 2, n_req)
    want_e = np.exp(rng.uniform(np.log(1e3), np.log(1e7), n_req))
    pick = np.empty(n_req, np.int64)
    for k in (0, 1):
        idx = np.nonzero(kind == k)[0]
        idx = idx[np.argsort(pool_E[idx])]
        le = np.log(np.maximum(pool_E[idx], 1))
        sel = want_k == k
        pos = np.clip(np.searchsorted(le, np.log(want_e[sel])), 1, len(idx) - 1)
        nearer = np.where(np.abs(le[pos - 1] - np.log(want_e[sel])) <= np.abs(le[pos] - np.log(want_e[sel])),
                          pos - 1, pos)
        pick[sel] = idx[nearer]
    log(f"[rank {rank}] served: pool {pool_n} graphs, E {pool_E.min()}..{pool_E.max()}, "
        f"requested E mean {pool_E[pick].mean():.0f}")
    srv = Server(hbm_budget_bytes=64 << 30, max_batch_graphs=4096, n_slots=args.lanes)
    # warm-up: every pool graph once
    for _ in range(max(1, args.warmup // 3)):
        ts = [srv.submit(*pool[i], outs[i]) for i in range(pool_n)]
        for t in ts:
            srv.wait(t)
    c0 = srv.counters()
    barrier(ws)
    clocks = Clocks(local).start()
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
    qwait = np.array([(inf["t_start_ns"] - target) / 1e6 for inf, target in infos])
    bsz = np.array([inf["batch_graphs"] for inf, _ in infos])
    end = max(inf["t_done_ns"] for inf, _ in infos)
    wall_s = max_over_ranks((end - t0) / 1e9, ws)
    gps = ws * n_req / wall_s
    eps = ws * float(pool_E[pick].sum()) / wall_s
    busy = c1["busy_ns"] - c0["busy_ns"]
    srv.close()
    # served results equal the graph run alone and the oracle's exact partition
    # (a seeded sample of the requested graphs)
    chk = sorted(rng.choice(np.unique(pick), size=min(len(np.unique(pick)), args.check_graphs),
                            replace=False).tolist())
    mism_alone = mism_oracle = 0
    with Context(int(pool_V[chk].max()), int(max(pool_E[chk].max(), 1))) as ctx:
        for i in chk:
            alone, _ = ctx.run(*pool[i])
            got = outs[i][:pool_V[i]]
            mism_alone += int((alone != got).sum())
            fb, fa, bb, ba = (t.cpu().numpy() for t in pool[i])
            csr = CSR(int(pool_V[i]), int(pool_E[i]), fb, fa, bb, ba)
            mism_oracle += int((oracle.tarjan(csr) != got.cpu().numpy()).sum())
    return {
        "metric": "served graphs/s", "value": gps, "unit": "graphs/s", "n_gpus": ws, "steps": n_req,
        "warmup": args.warmup, "ms_per_step": 1000.0 / gps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": "served SCC: Poisson arrivals, one graph per request, E log-uniform in [1e3, 1e7] "
                               "(R-MAT-like or planted-cycle DAG, 50/50), continuous batching over concurrent "
                               "lanes, 64 GiB device-memory budget",
                   "rate_per_s": args.rate, "duration_s": args.duration, "requests": n_req, "lanes": args.lanes,
                   "pool_graphs": pool_n, "pool_edges_min": int(pool_E.min()), "pool_edges_max": int(pool_E.max()),
                   "parallelism": "requests sharded by rank" if ws > 1 else "single-gpu"},
        "requested_edges_mean": float(pool_E[pick].mean()),
        "offered_edges_per_s": float(pool_E[pick].sum()) / args.duration,
        "edges_per_s": eps, "achieved_over_offered": (n_req / wall_s) / args.rate,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()), "from": "scheduled arrival to labels written"},
        "admission_wait_ms": {"p50": float(np.percentile(qwait, 50)), "p99": float(np.percentile(qwait, 99))},
        "batches": c1["batches"] - c0["batches"], "batch_graphs_mean": float(bsz.mean()),
        "busy_frac": busy / max(1, end - t0), "mean_batches_in_flight": (c1["lane_ns"] - c0["lane_ns"]) / max(1, busy),
        "budget_bytes_peak": c1["bytes_peak"],
        "labels_served_vs_alone_mismatches": mism_alone, "labels_vs_oracle_mismatches": mism_oracle,
        "graphs_checked": len(chk),
        "gpu_launches": (KERNELS_PER_STEP + 3) * (c1["batches"] - c0["batches"]), "clocks": clk}


# ---------------------------------------------------------------------------
# reference arm: the reference's own OpenMP CLI on the host cores

def batch_sample_host(args, n):
    """A seeded sample of the batch workload's graphs as host CSRs (int32)."""
    from ispan_b200 import gen
    from ispan_b200.graphs import CSR
    nseg = max(2, int(4096 * args.scale))
    rng = np.random.default_rng(args.seed + 99)
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


def reference_arm(args):
    if args.workload in ("batch", "served"):
        return reference_batch_arm(args)
    if args.workload not in ("social", "web"):
        print(json.dumps({"impl": "reference", "unavailable": f"no reference arm for workload {args.workload}"}))
        return
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
        "impl": "reference", "metric": "SCC GTEPS", "value": val, "unit": "GTEPS", "n_gpus": 1,
        "steps": len(totals), "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": dict(desc, parallelism=f"openmp{th}"),
        "cpu_baseline": {"value": val, "unit": "GTEPS", "cores": th, "kind": "reference",
                         "sample": f"full graph, {len(totals)} timed runs of the reference CLI "
                                   f"(src/scc_main.cpp) after {args.warmup} warm-up runs{sample_note}"},
        "e2e": {"value": val, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="social", choices=["social", "rmat16", "web", "batch", "served"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-configs", action="store_true", help="headline only (no per-workload sub-records)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-steps", type=int, default=2, help="reference runs for cpu_baseline")
    ap.add_argument("--ref-graphs", type=int, default=4, help="batch: sampled graphs the reference runs")
    ap.add_argument("--ref-cap", type=float, default=15.0, help="batch: seconds per reference graph")
    ap.add_argument("--small-steps", type=int, default=20, help="rmat16: timed runs per seed")
    ap.add_argument("--big-steps", type=int, default=3, help="web, batch: timed runs")
    ap.add_argument("--web-scale", type=float, default=1.0)
    ap.add_argument("--web-cpu-cap", type=float, default=60.0, help="web: seconds of reference pipeline time")
    ap.add_argument("--rate", type=float, default=2000.0, help="served: requests per second")
    ap.add_argument("--duration", type=float, default=60.0, help="served: seconds of arrivals")
    ap.add_argument("--pool", type=int, default=1024, help="served: distinct graphs in the request pool")
    ap.add_argument("--lanes", type=int, default=4, help="served: concurrent server lanes")
    ap.add_argument("--check-graphs", type=int, default=16, help="served: requested graphs checked")
    ap.add_argument("--tuning", type=lambda t: dict(kv.split("=") for kv in t.split(",") if kv), default={},
                    help="launch tunables over the autotuner's, e.g. color_compact=-1,pair_searches=1")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warmup raised to 3 (timing rule)")
        args.warmup = 3

    ws, rank, local = dist_init()
    import torch

    if args.impl == "reference":
        if rank == 0:  # one CPU run; the other ranks have no work
            reference_arm(args)
    elif args.workload == "social":
        out = bench_social(args, ws, rank, local)
        if ws == 1 and not args.no_configs:
            legs = (("rmat16", lambda: bench_rmat16(args)), ("web", lambda: bench_web(args)),
                    ("batch", lambda: bench_batch(args, ws, rank, local)),
                    ("served", lambda: bench_served(args, ws, rank, local)))
            out["configs"] = {}
            for name, fn in legs:
                t = time.time()
                try:
                    out["configs"][name] = fn()
                except Exception as e:  # noqa: BLE001  (one leg's failure must not hide the others)
                    out["configs"][name] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
                out["configs"][name]["wall_s"] = time.time() - t
                torch.cuda.synchronize()
                torch.cuda.empty_cache()
                log(f"{name}: {time.time() - t:.0f} s")
        if rank == 0:
            print(json.dumps(out))
    else:
        fn = {"rmat16": lambda: bench_rmat16(args), "web": lambda: bench_web(args),
              "batch": lambda: bench_batch(args, ws, rank, local),
              "served": lambda: bench_served(args, ws, rank, local)}[args.workload]
        rec = fn()
        if rank == 0:
            print(json.dumps(rec))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
