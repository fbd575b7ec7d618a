"""Autotuner host logic (no GPU): shape classes, table lookup, and that
apply() hands the class's tunables to the context."""
import json

from ispan_b200 import autotune as AT


class FakeCtx:
    def __init__(self):
        self.calls = []

    def set_tuning(self, *a):
        self.calls.append(a)


def test_shape_classes():
    assert AT.shape_class(41_652_231, 1_470_188_297) == "l-dense-one"
    assert AT.shape_class(65_536, 955_000) == "s-mid-one"
    assert AT.shape_class(700_000_000, 3_300_000_000) == "l-sparse-one"
    assert AT.shape_class(30_000_000, 264_000_000, nseg=204).endswith("-batch")


def test_lookup_and_apply(tmp_path):
    p = tmp_path / "t.json"
    params = dict(AT.DEFAULTS, alpha=100, async_v=4096, bfs_ctas_per_sm=1)
    p.write_text(json.dumps({"classes": {"s-mid-one": {"params": params, "ms": 1.0, "default_ms": 2.0}}}))
    assert AT.lookup(65_536, 955_000, path=str(p)) == params
    assert AT.lookup(41_652_231, 1_470_188_297, path=str(p)) is None
    ctx = FakeCtx()
    got = AT.apply(ctx, 65_536, 955_000, path=str(p))
    assert got["alpha"] == 100 and ctx.calls == [(4096, AT.DEFAULTS["async_e"], AT.DEFAULTS["async_deg"], 1,
                                                  AT.DEFAULTS["color_levels"], AT.DEFAULTS["color_pivots"],
                                                  0, 0, 0, 0)]
    ctx = FakeCtx()
    assert AT.apply(ctx, 10, 10, path=str(p)) == dict(AT.DEFAULTS, **AT.SWITCHES)  # untuned class: defaults
    ctx = FakeCtx()
    got = AT.apply(ctx, 10, 10, path=str(p), overrides={"color_compact": "-1", "alpha": 7})
    assert got["alpha"] == 7 and ctx.calls[0][6] == -1
    try:
        AT.apply(ctx, 10, 10, path=str(p), overrides={"nonsense": 1})
        raise AssertionError("unknown tunable accepted")
    except KeyError:
        pass


def test_descent_keeps_only_clear_gains():
    """tune() on a synthetic cost: the minimum of a separable function."""
    target = {"alpha": 100, "beta": 1000, "async_deg": 64}

    class Ctx(FakeCtx):
        pass

    ctx = Ctx()

    def run(a, b, c):
        t = ctx.calls[-1]
        cost = 10.0 + (a != target["alpha"]) + (b != target["beta"]) + (t[2] != target["async_deg"])
        return {"stage_ms": [cost / 2, cost / 2, 0.0, cost]}

    best, ms, dms = AT.tune(ctx, run, passes=2, reps=1, log=lambda *_: None)
    assert (best["alpha"], best["beta"], best["async_deg"]) == (100, 1000, 64)
    assert ms == 10.0 and dms == 13.0
