"""Host logic of the benchmark (no GPU): the end-to-end record's choice of
input form and the kernel count it reports."""
import bench


def _rec(ms, h):
    return {"value": 1.0 / ms, "unit": "GTEPS", "ms_per_step": ms, "h2d_bytes_per_step": h,
            "d2h_bytes_per_step": 4}


def test_forward_only_where_the_reverse_is_sorted():
    # every copy chunk (an eighth of the edges) below 2^31 edges: the forward CSR alone
    r = bench.e2e_pick(3_300_000_000, _rec(2.0, 10), _rec(3.0, 20))
    assert r["ms_per_step"] == 2.0 and r["h2d_bytes_per_step"] == 10
    assert r["both_directions"]["h2d_bytes_per_step"] == 20 and "forward CSR" in r["input"]


def test_both_directions_beyond_the_sorted_chunks():
    r = bench.e2e_pick(8 * (2**31), _rec(2.0, 10), _rec(3.0, 20))
    assert r["ms_per_step"] == 3.0 and r["h2d_bytes_per_step"] == 20
    assert r["forward_only"]["h2d_bytes_per_step"] == 10 and r["input"] == "both CSRs from pinned host memory"


def test_kernel_count_per_run():
    assert bench.KERNELS_PER_STEP == 27
