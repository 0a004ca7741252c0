"""Databases larger than their device memory budget (ssa_b200_set_db_memory).

The database is then streamed: segments of its length order take turns on the
device, each segment's entry pass and overflow cascade run while it is
resident, and the hits' sequences are gathered for the traceback.  Every result
must equal the resident database's, bit for bit (the resident path is pinned
against the oracle and the reference by the other parity tests): batched and
single-query Smith-Waterman with the 8 -> 16 -> 64-bit cascade, Needleman-Wunsch
at the 16-bit entry, the exact 64-bit entry, both nucleotide strands, long
pairs, and a sequence longer than a segment.  The server needs a resident
database and refuses a streamed one.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import ROOT, oracle_search, product_search, product_setup
from libssa_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _records(seed: int, n: int, queries: list[np.ndarray], alphabet) -> list[bytes]:
    rng = np.random.default_rng(seed)
    recs = []
    for i in range(n):
        r = rng.random()
        if r < 0.04:
            # near copies: scores beyond 8 and 16 bits take the cascade
            q = queries[int(rng.integers(0, len(queries)))]
            recs.append(W.mutate(rng, np.concatenate([q] * int(rng.integers(1, 4))), alphabet, 0.02, 0.01,
                                 (1, 3)).tobytes())
        elif r < 0.06:
            recs.append(b"")
        else:
            recs.append(W.random_residues(rng, int(rng.integers(10, 1200)), alphabet).tobytes())
    recs.append(W.random_residues(rng, 6000, alphabet).tobytes())      # longer than a segment
    return recs


def _both(search, budget: int):
    """search() with the database resident, then streamed with `budget` bytes."""
    import libssa_b200 as L
    L.set_db_memory(0)
    resident = search()
    assert not L.db_streamed()
    try:
        L.set_db_memory(budget)
        streamed = search()
        assert L.db_streamed()
    finally:
        L.set_db_memory(0)
    return resident, streamed


@pytest.mark.parametrize("budget", [1 << 14, 1 << 17])
def test_streamed_batched_sw_equals_resident(built_library, budget):
    rng = np.random.default_rng(41)
    queries = [W.random_residues(rng, int(rng.integers(30, 900)), W.AA20) for _ in range(9)]
    recs = _records(5, 1500, queries, W.AA20)
    product_setup(1, ("builtin", "blosum62"), (-11, -1), 100, 2, records=recs)
    qb = [q.tobytes() for q in queries]
    resident, streamed = _both(lambda: product_search("sw", 8, 1, 10, qb, batch=True)[0], budget)
    assert streamed == resident
    # and one query against the oracle directly
    want, _ = oracle_search("sw", 8, 1, 10, 1, ("builtin", "blosum62"), (-11, -1), 100, 2, qb[0], recs)
    assert streamed[0] == want


@pytest.mark.parametrize("algo,width", [("sw", 8), ("sw", 16), ("sw", 64), ("nw", 16)])
def test_streamed_single_queries_equal_resident(built_library, algo, width):
    rng = np.random.default_rng(43 + width)
    queries = [W.random_residues(rng, int(rng.integers(40, 600)), W.AA20) for _ in range(3)]
    recs = _records(7, 700, queries, W.AA20)
    product_setup(1, ("builtin", "blosum62"), (-11, -1), 1000, 2, records=recs)
    qb = [q.tobytes() for q in queries]
    resident, streamed = _both(lambda: product_search(algo, width, 1, 7, qb)[0], 1 << 15)
    assert streamed == resident


def test_streamed_nucleotide_both_strands(built_library):
    rng = np.random.default_rng(47)
    queries = [W.random_residues(rng, int(rng.integers(60, 400)), W.NT4) for _ in range(4)]
    recs = _records(9, 600, queries, W.NT4)
    product_setup(0, ("const", 2, -3), (-5, -2), 250, 2, records=recs, strands=3)
    qb = [q.tobytes() for q in queries]
    resident, streamed = _both(lambda: product_search("nw", 16, 1, 5, qb, frames=True)[0], 1 << 15)
    assert streamed == resident


def test_streamed_long_pairs(built_library):
    import libssa_b200 as L
    rng = np.random.default_rng(53)
    queries, recs = [], []
    for _ in range(6):
        a = W.random_residues(rng, int(rng.integers(500, 4000)), W.AA20)
        queries.append(a.tobytes())
        recs.append(W.mutate(rng, a, W.AA20, 0.08, 0.01, (1, 10)).tobytes())
    recs += [W.random_residues(rng, 300, W.AA20).tobytes() for _ in range(200)]
    product_setup(1, ("builtin", "blosum62"), (-11, -1), 1000, 2, records=recs)

    def run():
        qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in queries]
        try:
            out = []
            for algo in (L.SSA_SMITH_WATERMAN, L.SSA_NEEDLEMAN_WUNSCH):
                lists = L.align_pairs(algo, qs, list(range(6)), L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
                out.append([[h.key() for h in lst] for lst in lists])
            return out
        finally:
            for q in qs:
                L.free_sequence(q)

    resident, streamed = _both(run, 1 << 14)
    assert streamed == resident


def test_server_refuses_a_streamed_database(built_library, tmp_path):
    prog = (
        "import libssa_b200 as L\n"
        "L.load(); L.set_output_mode(L.OUTPUT_ERROR)\n"
        "L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)\n"
        "L.init_score_matrix(L.MATRIX_BUILDIN, 'blosum62'); L.init_gap_penalties(-11, -1)\n"
        "L.load_db_memory([b'ACDEFGHIKLMNPQRSTVWY' * 50] * 40)\n"
        "L.set_db_memory(4096)\n"
        "s = L.Server(L.SSA_SMITH_WATERMAN, 3, L.BIT_WIDTH_8, L.COMPUTE_SCORE, slots=2, segments=1)\n"
        "print('server started')\n")
    env = dict(os.environ, PYTHONPATH=ROOT)
    res = subprocess.run([sys.executable, "-c", prog], capture_output=True, text=True, env=env, timeout=300)
    assert res.returncode != 0
    assert "server started" not in res.stdout
    assert "resident" in res.stderr
