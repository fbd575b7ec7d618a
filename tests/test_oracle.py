"""CPU checks of the oracle itself: pinned to the reference's golden outputs
(tests/golden, produced by tests/golden/make_golden.py from the reference's
own CLI) and to the exact SCC partition."""
import glob
import os

import numpy as np
import pytest

import oracle
from ispan_b200 import graphs as G

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load(path):
    z = np.load(path)
    csr = G.CSR(int(z["V"]), int(z["E"]), z["fw_beg"], z["fw_adj"], z["bw_beg"], z["bw_adj"])
    return csr, z


def test_golden_present():
    assert len(GOLD) >= 8


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_tarjan_matches_golden_exact(path):
    csr, z = load(path)
    assert np.array_equal(oracle.tarjan(csr), z["exact"])


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_restatement_is_exact(path):
    csr, z = load(path)
    labels, codes, st = oracle.ispan(csr)
    assert np.array_equal(labels, z["exact"])
    assert st["scc_count"] == oracle.scc_count(z["exact"])


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_restatement_reproduces_reference_codes(path):
    """With the reference's quirks re-enabled, the serial restatement emits the
    reference's own serial scc_id codes bit for bit -- including the inputs
    where the reference's partition is wrong -- or predicts its hang."""
    csr, z = load(path)
    if bool(z["ref_nonterminating"]):
        with pytest.raises(oracle.NonTerminating):
            oracle.ispan(csr, quirks=oracle.QUIRKS_ALL)
        return
    _, codes, _ = oracle.ispan(csr, quirks=oracle.QUIRKS_ALL)
    assert np.array_equal(codes, z["ref_codes_t1"])


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_reference_codes_canonicalise(path):
    csr, z = load(path)
    if bool(z["ref_nonterminating"]):
        pytest.skip("reference does not terminate on this input")
    for t in (1, 4):
        ok = bool(z[f"ref_exact_t{t}"])
        same = np.array_equal(oracle.canon_codes(csr, z[f"ref_codes_t{t}"]), z["exact"])
        assert same == ok


def test_toy_known_answer():
    """graph_converter/toy_edge_list.txt: SCCs {0..4} and {5,6}; the reference
    prints largest 5, trimmed size_2 1, others 1 (the phantom slot V), total 3."""
    csr, z = load(os.path.join(os.path.dirname(__file__), "golden", "toy.npz"))
    assert list(z["exact"]) == [0, 0, 0, 0, 0, 5, 5]
    rep = str(z["ref_report_t1"])
    assert "largest, 5" in rep and "trimmed size_2, 1" in rep and "others, 1" in rep and "total, 3" in rep
    assert oracle.histogram(z["exact"]) == {2: 1, 5: 1}


def test_rmat_reference_exact_wherever_golden_says():
    for p in GOLD:
        if "rmat" in p:
            _, z = load(p)
            assert bool(z["ref_exact_t1"]) and bool(z["ref_exact_t4"])


@pytest.mark.parametrize("seed", range(4))
def test_restatement_vs_tarjan_random(seed):
    for csr in (G.planted(700, seed, giant_frac=0.2), G.rmat(9, 8, seed, permute=True),
                G.random_graph(400, 900, seed)):
        labels, _, _ = oracle.ispan(csr)
        assert np.array_equal(labels, oracle.tarjan(csr))


def test_histogram_and_empty():
    csr = G.from_edges(0, np.zeros((0, 2)))
    assert len(oracle.tarjan(csr)) == 0
    labels, _, st = oracle.ispan(csr)
    assert st["scc_count"] == 0
    csr = G.from_edges(5, np.zeros((0, 2)))
    labels, _, _ = oracle.ispan(csr)
    assert list(labels) == [0, 1, 2, 3, 4]
    assert oracle.histogram(labels) == {1: 5}


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_live_reference_matches_restatement():
    """Where the reference tree was built (oracle/_ref), run it in-process."""
    for csr in (G.rmat(12, 16, 4), G.rmat(10, 16, 5, permute=True)):
        sid, _ = oracle.ref_run(csr, 1)
        _, codes, _ = oracle.ispan(csr, quirks=oracle.QUIRKS_ALL)
        assert np.array_equal(sid, codes)
        sid4, _ = oracle.ref_run(csr, 4)
        assert np.array_equal(oracle.canon_codes(csr, sid4), oracle.tarjan(csr))


# ---- the plain-pipeline small workload at full size: R-MAT scale 16, edge
# factor 16, seeds 1-10, pinned to the reference's own CLI (golden/rmat16/)
RMAT16 = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "rmat16", "s*.npz")))


def rmat16(path):
    """The fixture's graph, regenerated from its seed and checked against the
    digest the fixture recorded."""
    import importlib.util
    z = np.load(path)
    csr = G.rmat(16, 16, int(z["seed"]))
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    assert mg.csr_digest(csr) == str(z["sha256"]), "regenerated graph differs from the fixture's"
    return csr, z


def test_rmat16_fixtures_present():
    assert len(RMAT16) == 10


@pytest.mark.parametrize("path", RMAT16, ids=[os.path.basename(p)[:-4] for p in RMAT16])
def test_rmat16_restatement_and_reference(path):
    csr, z = rmat16(path)
    exact = oracle.tarjan(csr)
    # the serial restatement with the reference's quirks emits its serial codes
    _, codes, _ = oracle.ispan(csr, quirks=oracle.QUIRKS_ALL)
    assert np.array_equal(codes, z["ref_codes_t1"])
    # the reference is exact on these graphs at 1 and 16 threads
    for t in (1, 16):
        assert bool(z[f"ref_exact_t{t}"])
        assert np.array_equal(oracle.canon_codes(csr, z[f"ref_codes_t{t}"]), exact)
    labels, _, _ = oracle.ispan(csr)
    assert np.array_equal(labels, exact)


@pytest.mark.skipif(not (os.path.exists(oracle.REF_LIB) and
                         os.path.exists(os.path.join(os.path.dirname(oracle.__file__), "_ref", "libispan_ref64.so"))),
                    reason="reference builds absent (make -C oracle ref ref64 where the reference tree is)")
@pytest.mark.parametrize("name,csr", [("rmat14", G.rmat(14, 16, 2)), ("planted3000", G.planted(3000, 2))])
def test_wide_reference_build_matches_reference(name, csr):
    """The reference compiled with its 64-bit typedefs (the CPU baseline of
    graphs beyond int32 offsets) emits the same serial codes as its int32
    build."""
    import ref_wide
    narrow, _ = oracle.ref_run(csr, 1)
    wide, _ = ref_wide.run(csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj, 1)
    assert np.array_equal(narrow.astype(np.int64), wide)
