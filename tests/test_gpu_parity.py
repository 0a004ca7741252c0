"""Parity of the GPU build with the reference, through the public C-ABI.

Bit-exact: hit IDs, scores, order (ties included), CIGAR strings, coordinates
and the 8->16 / 16->64 overflow counters.  Ground truth comes from the
reference's own known-answer tests, from golden runs of the reference binary
(tests/golden/cases.json) and from the oracle restatement on seeded inputs.
"""
import os

import numpy as np
import pytest

from helpers import DATA, ROOT, case_inputs, first_fasta_sequence, golden_cases, oracle_search, product_search, \
    product_setup, read_fasta, wide_cases
from kats import KATS, matches
from libssa_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _query(kat):
    kind, val = kat["query"]
    return (first_fasta_sequence(os.path.join(DATA, val)) if kind == "file" else val).encode()


@pytest.mark.parametrize("kat", KATS, ids=[k["source"] for k in KATS])
def test_reference_kats(built_library, kat):
    product_setup(kat["symtype"], kat["matrix"], kat["gap"], kat["chunk"], 2,
                  db_file=os.path.join(DATA, kat["db"]), strands=kat.get("strands", 1),
                  gencode=kat.get("gencode", (1, 1)))
    q = _query(kat)
    for algo, width, align, hits, simd, expected in kat["calls"]:
        import libssa_b200 as L
        L.set_simd_compute_mode(simd)
        res, ovf = product_search(algo, width, align, hits, [q])
        got = [(r[1], r[0], r[2]) for r in res[0]]
        assert matches(expected, got, ovf[0]), (kat["source"], algo, width, simd, got, ovf)


@pytest.mark.parametrize("case", golden_cases(), ids=[c["name"] for c in golden_cases()])
def test_golden_reference_runs(built_library, case):
    queries, records = case_inputs(case)
    product_setup(case["symtype"], case["matrix"], tuple(case["gap"]), case["chunk"], case["simd"], records=records)
    res, ovf = product_search(case["algo"], case["width"], case["align"], case["hits"], queries)
    for qi in range(len(queries)):
        exp = case["expected"][qi]
        assert [list(r) for r in res[qi]] == exp["hits"], (case["name"], qi)
        assert list(ovf[qi]) == [exp["ovf8"], exp["ovf16"]], (case["name"], qi)


@pytest.mark.parametrize("case", wide_cases(), ids=[c["name"] for c in wide_cases()])
@pytest.mark.parametrize("batch", [False, True], ids=["single", "batch"])
def test_wide_value_reference_runs(built_library, case, batch):
    """Scores far outside the int32 range (a matrix file of BLOSUM62 times
    100,000,007): the 64-bit pass runs in int64 and matches the reference's
    full_sw / full_nw (src/algo/64/smith_waterman_63.c:32-98,
    needleman_wunsch_64.c:32-98), at the 64-bit entry and at the end of the
    8/16-bit cascades."""
    queries = [q.encode() for q in case["queries"]]
    records = [r.encode() for r in case["records"]]
    product_setup(case["symtype"], case["matrix"], tuple(case["gap"]), case["chunk"], case["simd"], records=records)
    res, ovf = product_search(case["algo"], case["width"], case["align"], case["hits"], queries + queries[:1] * batch,
                              batch=batch)
    exp = case["expected"][0]
    for r in res:
        assert [list(x) for x in r] == exp["hits"], case["name"]
    if ovf is not None:
        assert list(ovf[0]) == [exp["ovf8"], exp["ovf16"]], case["name"]


def test_alignment_beyond_int32_is_refused(built_library, tmp_path):
    """The traceback kernels compute in int32: an alignment whose values could
    leave that range ends in fatal() with a message (exit status 1, as the
    reference's errors do), never with a wrapped result."""
    import subprocess
    import sys
    case = [c for c in wide_cases() if c["name"] == "wide_sw_64"][0]
    script = f"""
import sys
sys.path.insert(0, {ROOT!r}); sys.path.insert(0, {os.path.join(ROOT, "tests")!r})
import libssa_b200 as L
from helpers import product_setup, product_search
L.load()
case_q = {case["queries"][0]!r}
recs = {case["records"][:20]!r}
product_setup(1, "file:wide_scores.txt", (-11, -1), 1000, 2, records=[r.encode() for r in recs])
product_search("sw", 64, 1, 5, [case_q.encode()])
print("returned")
"""
    r = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=300)
    assert r.returncode == 1, (r.returncode, r.stdout, r.stderr)
    assert "exceeds the supported score range" in r.stderr
    assert "returned" not in r.stdout


@pytest.mark.parametrize("name", ["sw_batched_small", "mixed_sw_8_2", "mixed_nw_8_2"])
def test_requeue_lists_grow_when_a_pass_overflows_them(built_library, monkeypatch, name):
    """The re-queue lists start small (here 2 entries); an entry pass that
    re-queues more pairs runs again with lists of its count, and the answer is
    the reference's."""
    monkeypatch.setenv("SSA_B200_REQUEUE_CAP", "2")
    case = [c for c in golden_cases() if c["name"] == name][0]
    queries, records = case_inputs(case)
    product_setup(case["symtype"], case["matrix"], tuple(case["gap"]), case["chunk"], case["simd"], records=records)
    for batch in (False, True):
        res, ovf = product_search(case["algo"], case["width"], case["align"], case["hits"], queries, batch=batch)
        for qi in range(len(queries)):
            exp = case["expected"][qi]
            assert [list(r) for r in res[qi]] == exp["hits"], (name, qi, batch)
            if ovf is not None:
                assert list(ovf[qi]) == [exp["ovf8"], exp["ovf16"]], (name, qi)
    assert any(e["ovf8"] + e["ovf16"] > 2 for e in case["expected"])


def test_batched_equals_single(built_library):
    """Each query's result is the same alone and inside a batch."""
    case = [c for c in golden_cases() if c["name"] == "sw_batched_small"][0]
    queries, records = case_inputs(case)
    product_setup(case["symtype"], case["matrix"], tuple(case["gap"]), case["chunk"], case["simd"], records=records)
    single, _ = product_search(case["algo"], case["width"], 1, case["hits"], queries)
    batched, _ = product_search(case["algo"], case["width"], 1, case["hits"], queries, batch=True)
    assert single == batched
    for qi in range(len(queries)):
        assert [list(r) for r in batched[qi]] == case["expected"][qi]["hits"]


def _random_case(seed):
    rng = np.random.default_rng(seed)
    nuc = bool(rng.random() < 0.4)
    alpha = W.NT4 if nuc else W.AA20
    q = W.random_residues(rng, int(rng.integers(1, 600)), alpha)
    recs = []
    for _ in range(int(rng.integers(1, 300))):
        r = rng.random()
        if r < 0.15:
            recs.append(W.mutate(rng, q, alpha, 0.05, 0.02, (1, 5)).tobytes())
        elif r < 0.18:
            recs.append(W.mutate(rng, np.tile(q, int(rng.integers(2, 5))), alpha, 0.01, 0.0, (1, 1)).tobytes())
        else:
            recs.append(W.random_residues(rng, int(rng.integers(1, 700)), alpha).tobytes())
    if nuc:
        matrix = ("const", int(rng.integers(1, 8)), -int(rng.integers(1, 8)))
    else:
        matrix = ("builtin", ["blosum62", "blosum45", "pam30", "pam250", "blosum80"][int(rng.integers(0, 5))])
    gap = (-int(rng.integers(0, 20)), -int(rng.integers(0, 4)))
    return dict(algo=["sw", "nw"][int(rng.integers(0, 2))], width=int([8, 16, 64][int(rng.integers(0, 3))]),
                align=1, hits=int(rng.integers(1, 20)), symtype=0 if nuc else 1, matrix=matrix, gap=gap,
                chunk=int([1000, 64, 7][int(rng.integers(0, 3))]), simd=int([2, 1][int(rng.integers(0, 2))]),
                query=q.tobytes(), records=recs)


@pytest.mark.parametrize("seed", range(40))
def test_random_against_oracle(built_library, seed):
    c = _random_case(seed)
    product_setup(c["symtype"], c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    res, ovf = product_search(c["algo"], c["width"], c["align"], c["hits"], [c["query"]])
    exp, eovf = oracle_search(c["algo"], c["width"], c["align"], c["hits"], c["symtype"], c["matrix"], c["gap"],
                              c["chunk"], c["simd"], c["query"], c["records"])
    assert res[0] == exp
    assert tuple(ovf[0]) == tuple(eovf)


def test_long_query_multi_pass(built_library):
    """Queries longer than one 256-row pass and sequences with 8- and 16-bit
    overflow, SW and NW, against the oracle."""
    rng = np.random.default_rng(5)
    q = W.random_residues(rng, 900, W.AA20)
    recs = [W.mutate(rng, q, W.AA20, 0.02, 0.01, (1, 3)).tobytes() for _ in range(3)]
    recs += [W.random_residues(rng, int(rng.integers(50, 1500)), W.AA20).tobytes() for _ in range(40)]
    for algo, width in (("sw", 8), ("sw", 16), ("nw", 16), ("nw", 8)):
        product_setup(1, ("builtin", "blosum62"), (-11, -1), 1000, 2, records=recs)
        res, ovf = product_search(algo, width, 1, 8, [q.tobytes()])
        exp, eovf = oracle_search(algo, width, 1, 8, 1, ("builtin", "blosum62"), (-11, -1), 1000, 2, q.tobytes(),
                                  recs)
        assert res[0] == exp, (algo, width)
        assert tuple(ovf[0]) == tuple(eovf), (algo, width)


def _batch_case(seed):
    rng = np.random.default_rng(1000 + seed)
    nq = int(rng.integers(2, 10))
    qs = [W.random_residues(rng, int(rng.integers(1, 1200)), W.AA20) for _ in range(nq)]
    recs = []
    for _ in range(int(rng.integers(20, 400))):
        r = rng.random()
        src = qs[int(rng.integers(0, nq))]
        if r < 0.08:
            recs.append(W.mutate(rng, src, W.AA20, 0.03, 0.01, (1, 4)).tobytes())
        elif r < 0.1:
            recs.append(W.mutate(rng, np.tile(src, int(rng.integers(2, 4))), W.AA20, 0.01, 0.0, (1, 1)).tobytes())
        elif r < 0.12:
            recs.append(b"")
        else:
            recs.append(W.random_residues(rng, int(rng.integers(1, 900)), W.AA20).tobytes())
    gap = [(-11, -1), (-5, -2), (-10, 0), (0, 0)][int(rng.integers(0, 4))]
    matrix = ("builtin", ["blosum62", "blosum45", "pam30"][int(rng.integers(0, 3))])
    return dict(queries=[q.tobytes() for q in qs], records=recs, gap=gap, matrix=matrix,
                chunk=int([1000, 50, 7][int(rng.integers(0, 3))]), hits=int(rng.integers(1, 15)),
                simd=int([2, 1][int(rng.integers(0, 2))]))


@pytest.mark.parametrize("seed", range(12))
def test_batched_random_against_oracle(built_library, seed):
    """Batches (query pairs share the 16x2 lanes) of 2-9 SW queries, 1-1200
    residues, with overflowing copies and empty records, against the oracle
    query by query."""
    c = _batch_case(seed)
    product_setup(1, c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    batched, _ = product_search("sw", 8, 1, c["hits"], c["queries"], batch=True)
    for qi, q in enumerate(c["queries"]):
        exp, _ = oracle_search("sw", 8, 1, c["hits"], 1, c["matrix"], c["gap"], c["chunk"], c["simd"], q,
                               c["records"])
        assert batched[qi] == exp, (seed, qi, len(q))


@pytest.mark.parametrize("shape", [(16, 4, 4, 0), (20, 4, 4, 0), (24, 4, 4, 0), (28, 4, 4, 0), (20, 5, 2, 0),
                                   (24, 5, 2, 0), (16, 5, 4, 0), (20, 5, 4, 0), (16, 4, 4, 1), (20, 4, 4, 1),
                                   (24, 4, 4, 1), (28, 4, 4, 1), (24, 4, 4, 8), (24, 5, 4, 8)],
                         ids=lambda s: f"R{s[0]}_ctas{s[1]}_cols{s[2]}" + ("_hmax" if s[3] == 1 else
                                                                           "_g8" if s[3] == 8 else ""))
@pytest.mark.parametrize("seed", range(4))
def test_batched_kernel_variants_against_oracle(built_library, monkeypatch, shape, seed):
    """Every variant of the query-pair kernel the shape table can select --
    rows per thread, 4 or 5 resident CTAs per SM, 2 or 4 columns per step,
    the running maximum as integer or fp16x2 max, 4 or 8 threads per sequence
    -- pinned, on batches with
    multi-pass queries, overflowing copies and empty records, against the
    oracle query by query (scores, overflow blocks through the tie order,
    CIGARs)."""
    R, mb, cols, extra = shape
    hm, g8 = extra == 1, extra == 8
    monkeypatch.setenv("SSA_B200_QP_R", str(R))
    monkeypatch.setenv("SSA_B200_QP_MB", str(mb))
    monkeypatch.setenv("SSA_B200_QP_C", str(cols))
    monkeypatch.setenv("SSA_B200_QP_HMAX", str(int(hm)))
    monkeypatch.setenv("SSA_B200_QP_G8", str(int(g8)))
    c = _batch_case(100 + seed)
    product_setup(1, c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    batched, _ = product_search("sw", 8, 1, c["hits"], c["queries"], batch=True)
    import libssa_b200 as L
    used = [u for u in L.tuning_report()["last_call"] if u["kernel"].startswith("sw_qpair")]
    assert used and all(u["R"] == R and u["ctas_per_sm"] == mb for u in used), used
    assert all(u["kernel"] == ("sw_qpair4h" if hm else "sw_qpair4g8" if g8 else "sw_qpair4" if cols == 4
                               else "sw_qpair") for u in used), used
    for qi, q in enumerate(c["queries"]):
        exp, _ = oracle_search("sw", 8, 1, c["hits"], 1, c["matrix"], c["gap"], c["chunk"], c["simd"], q,
                               c["records"])
        assert batched[qi] == exp, (shape, seed, qi, len(q))


FAST_SHAPES = [(G, R, 4) for G in (4, 8, 16, 32) for R in (8, 16, 24) if G * R <= 512] + \
              [(8, 32, 1), (16, 16, 1), (32, 8, 1), (16, 32, 1)]


@pytest.mark.parametrize("shape", FAST_SHAPES, ids=lambda s: f"G{s[0]}_R{s[1]}_cols{s[2]}")
@pytest.mark.parametrize("seed", range(2))
def test_single_query_kernel_variants_against_oracle(built_library, monkeypatch, shape, seed):
    """Every shape of the single-query (sw_align) entry kernels the shape table
    can select -- threads per sequence pair G, rows per thread R, one or four
    columns per step -- pinned, on queries of one to several passes against
    databases with overflowing copies and empty records, against the oracle
    (scores, overflow blocks through the tie order and the counters, CIGARs)."""
    G, R, cols = shape
    monkeypatch.setenv("SSA_B200_FAST_SHAPE", f"{G},{R},{cols}")
    c = _batch_case(300 + seed)
    qs = c["queries"][:3]
    product_setup(1, c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    import libssa_b200 as L
    for q in qs:
        res, ovf = product_search("sw", 8, 1, c["hits"], [q])
        used = [u for u in L.tuning_report()["last_call"] if u["kernel"].startswith("sw_fast")]
        assert used and all(u["kernel"] == ("sw_fast4" if cols == 4 else "sw_fast") and u["G"] == G and
                            u["R"] == R for u in used), used
        exp, eovf = oracle_search("sw", 8, 1, c["hits"], 1, c["matrix"], c["gap"], c["chunk"], c["simd"], q,
                                  c["records"])
        assert res[0] == exp, (shape, seed, len(q))
        assert tuple(ovf[0]) == tuple(eovf), (shape, seed, len(q))


def _nw_batch_case(seed):
    rng = np.random.default_rng(2000 + seed)
    nuc = seed % 2 == 0
    alpha = W.NT4 if nuc else W.AA20
    nq = int(rng.integers(1, 7))
    qs = [W.random_residues(rng, int(rng.integers(1, 900)), alpha) for _ in range(nq)]
    recs = []
    for _ in range(int(rng.integers(20, 250))):
        r = rng.random()
        src = qs[int(rng.integers(0, nq))]
        if r < 0.1:
            recs.append(W.mutate(rng, src, alpha, 0.05, 0.02, (1, 5)).tobytes())
        elif r < 0.14:
            # long enough that some pairs fall outside the exact 16-bit range
            recs.append(W.random_residues(rng, int(rng.integers(3000, 9000)), alpha).tobytes())
        else:
            recs.append(W.random_residues(rng, int(rng.integers(1, 1500)), alpha).tobytes())
    if nuc:
        matrix = ("const", int(rng.integers(1, 6)), -int(rng.integers(1, 6)))
    else:
        matrix = ("builtin", ["blosum62", "pam30"][int(rng.integers(0, 2))])
    gap = [(-5, -2), (-11, -1), (-2, -3), (-40, -4)][int(rng.integers(0, 4))]
    return dict(queries=[q.tobytes() for q in qs], records=recs, gap=gap, matrix=matrix, symtype=0 if nuc else 1,
                chunk=int([1000, 33][int(rng.integers(0, 2))]), hits=int(rng.integers(1, 12)),
                simd=int([2, 1][int(rng.integers(0, 2))]))


@pytest.mark.parametrize("seed", [1, 3])
def test_nw16_redo_list_grows(built_library, monkeypatch, seed):
    """The NW query-pair pass sends sequences beyond its exact range to a redo
    list; with lists starting at 2 entries the pass runs again with room for
    all of them, and the batch still matches the oracle."""
    monkeypatch.setenv("SSA_B200_REQUEUE_CAP", "2")
    c = _nw_batch_case(seed)
    product_setup(c["symtype"], c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    batched, _ = product_search("nw", 16, 1, c["hits"], c["queries"], batch=True)
    for qi, q in enumerate(c["queries"]):
        exp, _ = oracle_search("nw", 16, 1, c["hits"], c["symtype"], c["matrix"], c["gap"], c["chunk"], c["simd"],
                               q, c["records"])
        assert batched[qi] == exp, (seed, qi, len(q))


@pytest.mark.parametrize("cols", [4, 2], ids=lambda c: f"cols{c}")
@pytest.mark.parametrize("seed", range(8))
def test_nw16_batched_against_oracle(built_library, monkeypatch, seed, cols):
    """Needleman-Wunsch at the 16-bit entry through the query-pair kernel
    (single queries and batches; one 4-column block per step, the default, or
    two columns per step, pinned), including multi-pass queries and sequences
    beyond its exact range that go to the lane emulation, against the oracle
    query by query."""
    monkeypatch.setenv("SSA_B200_QP_C", str(cols))
    c = _nw_batch_case(seed)
    product_setup(c["symtype"], c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    batched, _ = product_search("nw", 16, 1, c["hits"], c["queries"], batch=True)
    import libssa_b200 as L
    used = [u for u in L.tuning_report()["last_call"] if u["kernel"].startswith("nw_qpair")]
    assert used and all(u["kernel"] == ("nw_qpair4" if cols == 4 else "nw_qpair") for u in used), used
    single, ovf = product_search("nw", 16, 1, c["hits"], c["queries"][:1])
    for qi, q in enumerate(c["queries"]):
        exp, eovf = oracle_search("nw", 16, 1, c["hits"], c["symtype"], c["matrix"], c["gap"], c["chunk"], c["simd"],
                                  q, c["records"])
        assert batched[qi] == exp, (seed, qi, len(q))
        if qi == 0:
            assert single[0] == exp
            assert tuple(ovf[0]) == tuple(eovf)


from helpers import frame_cases  # noqa: E402


@pytest.mark.parametrize("case", frame_cases(), ids=[c["name"] for c in frame_cases()])
def test_strands_and_translated_frames(built_library, case):
    """Nucleotide queries on one or both strands and translated queries (3 or
    6 frames, several genetic codes): hits, tie order, CIGARs, coordinates,
    the strand and frame fields of every hit and the overflow counters equal
    the reference's, alone and in a batch."""
    queries, records = case_inputs(case)
    product_setup(case["symtype"], case["matrix"], tuple(case["gap"]), case["chunk"], case["simd"], records=records,
                  strands=case["strands"], gencode=tuple(case["gencode"]))
    res, ovf = product_search(case["algo"], case["width"], case["align"], case["hits"], queries, frames=True)
    for qi in range(len(queries)):
        exp = case["expected"][qi]
        assert [list(r) for r in res[qi]] == exp["hits"], (case["name"], qi)
        assert list(ovf[qi]) == [exp["ovf8"], exp["ovf16"]], (case["name"], qi)
    batched, _ = product_search(case["algo"], case["width"], case["align"], case["hits"], queries * 3, batch=True,
                                frames=True)
    assert all(b == res[0] for b in batched)
