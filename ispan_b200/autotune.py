"""Autotuner: per graph-shape class, the launch parameters of the pipeline.

Tuned: the push/pull switch of the reachability searches (alpha, beta, gamma:
the reference's own knobs, src/fw_bw.h:576-624, whose defaults 30/200/10 come
from src/bash_one.sh:4), the frontier sizes and vertex degree below which a
search runs asynchronously inside CTAs (async_v, async_e, async_deg), and
the CTAs per SM of the persistent searches (bfs_ctas_per_sm), the work a
warp does per grid round when colouring large WCCs (color_levels: up to
4 * color_levels chunks of 32 frontier entries; less balances the CTAs, more
saves grid barriers) and the pivots of the colouring's first round
(color_pivots).  None of them changes a label; they
only move time between stages.

Method: coordinate descent from the defaults over a small grid per
parameter, two passes, each candidate timed as the median of several runs on
the device (CUDA events inside the captured graph) of the trim, elephant and
mice stages.
The winners are stored per shape class in ``tuning_table.json`` beside this
file; :func:`apply` looks a graph's class up and sets the context.

    python -m ispan_b200.autotune --workloads social,web:0.1,rmat16,batch:0.05
"""
from __future__ import annotations

import argparse
import json
import os
import statistics

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning_table.json")

DEFAULTS = {"alpha": 30, "beta": 200, "gamma": 10, "async_v": 65536, "async_e": 262144, "async_deg": 16,
            "bfs_ctas_per_sm": 0, "color_levels": 32, "color_pivots": 1024}
# switches that are not searched (0 = the library's default; see ispan_tuning)
SWITCHES = {"color_compact": 0, "pair_searches": 0, "tiny_residual": 0, "pdl": 0}
SPACE = {
    "alpha": [5, 10, 30, 100, 300],
    "beta": [50, 200, 1000, 4000],
    "gamma": [3, 5, 10, 30],
    "async_v": [4096, 16384, 65536, 262144],
    "async_e": [16384, 65536, 262144, 1048576],
    "async_deg": [4, 16, 64],
    "bfs_ctas_per_sm": [1, 0],
    "color_levels": [4, 8, 16, 32, 64, 256],
    "color_pivots": [256, 1024, 8192, 65536],
}


def shape_class(V: int, E: int, nseg: int = 1) -> str:
    """Graph-shape class: size (vertices per graph), mean degree, batched or not."""
    per = V / max(nseg, 1)
    size = "s" if per < (1 << 18) else ("m" if per < (1 << 24) else "l")
    d = E / max(V, 1)
    deg = "sparse" if d < 6 else ("mid" if d < 24 else "dense")
    return f"{size}-{deg}-{'batch' if nseg > 1 else 'one'}"


def load_table(path: str = TABLE) -> dict:
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {"classes": {}}
    return {"classes": {}}


def lookup(V: int, E: int, nseg: int = 1, path: str = TABLE) -> dict | None:
    """Tuned parameters of the graph's class, or None if the class was never tuned."""
    ent = load_table(path)["classes"].get(shape_class(V, E, nseg))
    return None if ent is None else {k: ent["params"].get(k, DEFAULTS[k]) for k in DEFAULTS}


def apply(ctx, V: int, E: int, nseg: int = 1, path: str = TABLE, overrides: dict | None = None) -> dict:
    """Set ctx's tunables for the graph's class (then ``overrides``, any of
    DEFAULTS or SWITCHES); returns the parameters to pass to the run (alpha,
    beta, gamma) merged with the launch tunables."""
    p = dict(DEFAULTS)
    p.update(SWITCHES)
    t = lookup(V, E, nseg, path)
    if t:
        p.update(t)
    for k, v in (overrides or {}).items():
        if k not in p:
            raise KeyError(f"unknown tunable {k!r}")
        p[k] = int(v)
    ctx.set_tuning(p["async_v"], p["async_e"], p["async_deg"], p["bfs_ctas_per_sm"], p["color_levels"],
                   p["color_pivots"], p["color_compact"], p["pair_searches"], p["tiny_residual"], p["pdl"])
    return p


def tuned_ms(stage_ms) -> float:
    """The time the tunables act on: the trim, elephant and mice stages
    (reference slots 0, 1 and 2; their sum is the pipeline time)."""
    return stage_ms[0] + stage_ms[1] + stage_ms[2]


def measure(ctx, run, p: dict, reps: int = 5) -> float:
    """Median trim + elephant + mice time (ms, device events) of run(alpha, beta, gamma) under p."""
    ctx.set_tuning(p["async_v"], p["async_e"], p["async_deg"], p["bfs_ctas_per_sm"], p["color_levels"],
                   p["color_pivots"])
    run(p["alpha"], p["beta"], p["gamma"])  # capture the graph for these values
    ts = [tuned_ms(run(p["alpha"], p["beta"], p["gamma"])["stage_ms"]) for _ in range(reps)]
    return statistics.median(ts)


def tune(ctx, run, passes: int = 2, reps: int = 5, log=print) -> tuple[dict, float, float]:
    """Coordinate descent from the defaults; returns (best, best_ms, default_ms)."""
    best = dict(DEFAULTS)
    best_ms = default_ms = measure(ctx, run, best, reps)
    log(f"  default {default_ms:.3f} ms")
    for _ in range(passes):
        improved = False
        for k, vals in SPACE.items():
            for v in vals:
                if v == best[k]:
                    continue
                cand = dict(best, **{k: v})
                ms = measure(ctx, run, cand, reps)
                if ms < best_ms * 0.98:  # keep a change only for a clear gain
                    best, best_ms, improved = cand, ms, True
                    log(f"  {k}={v}: {ms:.3f} ms (new best)")
        if not improved:
            break
    return best, best_ms, default_ms


def _workload(spec: str):
    from . import gen
    name, _, arg = spec.partition(":")
    scale = float(arg) if arg else 1.0
    if name == "social":
        return gen.social(seed=1, scale=scale), None
    if name == "web":
        return gen.web(seed=1, scale=scale), None
    if name == "rmat16":
        return gen.rmat(16, 16, 1), None
    if name == "batch":
        g = gen.batch(nseg=max(2, int(4096 * scale)), seed=1)
        return g, g.vbase
    raise SystemExit(f"unknown workload {spec}")


def main():
    import torch

    from . import Context
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="social,web:0.1,rmat16,batch:0.05")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--passes", type=int, default=2)
    ap.add_argument("--out", default=TABLE)
    args = ap.parse_args()
    table = load_table(args.out)
    for spec in args.workloads.split(","):
        g, vbase = _workload(spec)
        nseg = 1 if vbase is None else len(vbase) - 1
        cls = shape_class(g.V, g.E, nseg)
        print(f"{spec}: V={g.V} E={g.E} class {cls}", flush=True)
        ctx = Context(g.V, g.E)
        lab = torch.empty(max(g.V, 1), dtype=torch.int32, device="cuda")
        fb, fa, bb, ba = g.ptrs

        def run(a, b, c):
            return ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, lab, vbase=vbase, alpha=a, beta=b, gamma=c,
                               stage_times=True)[1]

        best, ms, dms = tune(ctx, run, args.passes, args.reps)
        table["classes"][cls] = {"params": best, "ms": ms, "default_ms": dms, "speedup": dms / ms,
                                 "tuned_on": f"{spec} (V={g.V}, E={g.E})"}
        print(f"  best {best} {ms:.3f} ms vs default {dms:.3f} ms", flush=True)
        ctx.close()
        g.free()
        with open(args.out, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    print(json.dumps(table))


if __name__ == "__main__":
    main()
