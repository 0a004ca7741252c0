"""The oracle restatement (oracle/ssa_oracle.c) pinned against the reference:
its known-answer tests, the golden fixtures made by running the reference
itself, and -- when oracle/_ref/ref_run is built -- fresh reference runs."""
import os

import numpy as np
import pytest

import oracle
from helpers import DATA, case_inputs, first_fasta_sequence, golden_cases, golden_matrices, matrix_table, \
    oracle_search, read_fasta, wide_cases
from kats import KATS, matches


def _query(kat):
    kind, val = kat["query"]
    return (first_fasta_sequence(os.path.join(DATA, val)) if kind == "file" else val).encode()


def _matrix_spec(m) -> str:
    return f"const:{m[1]},{m[2]}" if m[0] == "const" else f"builtin:{m[1]}"


@pytest.mark.parametrize("kat", KATS, ids=[k["source"] for k in KATS])
def test_oracle_reproduces_reference_kats(kat, tmp_path):
    records = read_fasta(os.path.join(DATA, kat["db"]))
    q = _query(kat)
    if kat["symtype"] not in (0, 1) or kat.get("strands", 1) != 1:
        # strands and translated frames are outside the restatement: the KAT
        # pins the reference built from its sources instead
        if not oracle.reference_available():
            pytest.skip("oracle/_ref/ref_run is not built")
        for algo, width, align, hits, simd, expected in kat["calls"]:
            res = oracle.run_reference(os.path.join(DATA, kat["db"]), [q.decode()], algo=algo, width=width,
                                       align=align, hits=hits, symtype=kat["symtype"], strands=kat["strands"],
                                       gencode=kat["gencode"], matrix=_matrix_spec(kat["matrix"]), gap=kat["gap"],
                                       chunk=kat["chunk"], simd=simd, workdir=str(tmp_path))
            got = [(h["score"], h["id"], h["cigar"]) for h in res[0]["hits"]]
            assert matches(expected, got, None), (algo, width, simd, got)
        return
    for algo, width, align, hits, simd, expected in kat["calls"]:
        res, ovf = oracle_search(algo, width, align, hits, kat["symtype"], kat["matrix"], kat["gap"], kat["chunk"],
                                 simd, q, records)
        got = [(r[1], r[0], r[2]) for r in res]
        assert matches(expected, got, ovf), (algo, width, simd, got, ovf)


@pytest.mark.parametrize("case", golden_cases(), ids=[c["name"] for c in golden_cases()])
def test_oracle_matches_golden_reference_runs(case):
    if case["name"] == "sw_plain_full":
        pytest.skip("full-size config covered by the GPU parity test")
    queries, records = case_inputs(case)
    for qi, q in enumerate(queries):
        res, ovf = oracle_search(case["algo"], case["width"], case["align"], case["hits"], case["symtype"],
                                 case["matrix"], case["gap"], case["chunk"], case["simd"], q, records)
        exp = case["expected"][qi]
        assert [list(r) for r in res] == exp["hits"]
        assert [exp["ovf8"], exp["ovf16"]] == list(ovf)


def test_oracle_matrix_parser_matches_reference_tables():
    mats = golden_matrices()
    for name in ("blosum90.txt", "nuc_scoring_matrix.txt"):
        with open(os.path.join(DATA, name)) as f:
            assert (oracle.parse_matrix(f.read()) == np.array(mats["file:" + name])).all()
    assert (oracle.constant_matrix(5, -4) == np.array(mats["const:5,-4"])).all()
    assert (oracle.constant_matrix(127, -128) == np.array(mats["const:127,-128"])).all()


def test_oracle_lane_result_consistent_with_full_search():
    # a sequence alone in a lane reports the same score as the exact kernel
    # whenever it does not overflow
    rng = np.random.default_rng(7)
    cfg = oracle.SearchConfig(algo="sw", matrix=matrix_table(("builtin", "blosum62")))
    for _ in range(20):
        q = rng.integers(1, 24, int(rng.integers(5, 200))).astype(np.uint8)
        d = rng.integers(1, 24, int(rng.integers(5, 300))).astype(np.uint8)
        s, ovf, blocks = oracle.lane_result(cfg, 8, q, d)
        if not ovf:
            assert s == oracle.full_score(cfg, q, d)
            assert blocks == (len(d) + 3) // 4


@pytest.mark.skipif(not oracle.reference_available(), reason="reference binary not built here")
def test_oracle_against_fresh_reference_runs(tmp_path):
    # random small searches: the restatement and the reference agree exactly
    rng = np.random.default_rng(99)
    alpha = np.frombuffer(b"ACGT", np.uint8)
    for trial in range(12):
        algo = ["sw", "nw"][trial % 2]
        width = [8, 16, 64][trial % 3]
        q = alpha[rng.integers(0, 4, int(rng.integers(5, 80)))].tobytes()
        recs = [alpha[rng.integers(0, 4, int(rng.integers(1, 120)))].tobytes() for _ in range(int(rng.integers(5, 90)))]
        db = str(tmp_path / f"db{trial}.sdb")
        oracle.write_sdb(db, seqs=recs)
        ref = oracle.run_reference(db, [q.decode()], algo=algo, width=width, align=1, hits=7, symtype=0,
                                   matrix="const:2,-1", gap=(-2, -1), chunk=13)[0]
        res, ovf = oracle_search(algo, width, 1, 7, 0, "const:2,-1", (-2, -1), 13, 2, q, recs)
        assert [list(r) for r in res] == [[h["id"], h["score"], h["cigar"], h["q_start"], h["q_end"], h["d_start"],
                                           h["d_end"]] for h in ref["hits"]]
        assert (ref["ovf8"], ref["ovf16"]) == ovf


@pytest.mark.parametrize("case", wide_cases(), ids=[c["name"] for c in wide_cases()])
def test_oracle_matches_wide_value_reference_runs(case):
    """64-bit scores far outside the int32 range (a matrix file of BLOSUM62
    times 100,000,007), at the 64-bit entry and through the 8/16-bit cascades
    whose lanes use the truncated table."""
    queries = [q.encode() for q in case["queries"]]
    records = [r.encode() for r in case["records"]]
    for qi, q in enumerate(queries):
        res, ovf = oracle_search(case["algo"], case["width"], case["align"], case["hits"], case["symtype"],
                                 case["matrix"], case["gap"], case["chunk"], case["simd"], q, records)
        exp = case["expected"][qi]
        assert [list(r) for r in res] == exp["hits"]
        assert [exp["ovf8"], exp["ovf16"]] == list(ovf)
        assert max(h[1] for h in exp["hits"]) > 2 ** 31


def test_wide_matrix_file_parses_like_the_reference():
    """The oracle's parser reads the large entries as the reference does
    (int64, unset cells -1)."""
    m = matrix_table("file:wide_scores.txt")
    b62 = np.array(golden_matrices()["blosum62"], dtype=np.int64)
    aa = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ"
    listed = [aa.index(c) for c in "ARNDCQEGHILKMFPSTWYVBZX*"]
    for a in range(32):
        for b in range(32):
            want = b62[(a << 5) + b] * 100_000_007 if a in listed and b in listed else -1
            assert m[(a << 5) + b] == want, (a, b)
