"""The serving loop (ssa_server_*): continuous batching over resident slots.

Requests arrive at seeded random times from a client thread while others are
on the GPU; each result must equal, bit for bit, what the same query gets from
sw_align / nw_align alone (hits, scores, tie order, CIGARs, coordinates).  The
mix includes multi-pass queries, sequences that overflow the 8-bit entry, more
requests than slots, a memory budget that admits one request at a time, and
plain searches interleaved with the server's waves.
"""
import threading
import time

import numpy as np
import pytest

from helpers import product_setup
from libssa_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _db(seed: int, n: int, queries: list[np.ndarray]) -> list[bytes]:
    rng = np.random.default_rng(seed)
    recs = []
    for _ in range(n):
        r = rng.random()
        if r < 0.05:
            recs.append(W.mutate(rng, queries[int(rng.integers(0, len(queries)))], W.AA20, 0.03, 0.01,
                                 (1, 3)).tobytes())
        elif r < 0.07:
            recs.append(b"")
        else:
            recs.append(W.random_residues(rng, int(rng.integers(10, 900)), W.AA20).tobytes())
    return recs


def _alone(L, algo: str, qtexts: list[str], hits: int, width: int) -> list:
    out = []
    for t in qtexts:
        q = L.init_sequence_fasta(L.READ_FROM_STRING, t)
        fn = L.sw_align if algo == "sw" else L.nw_align
        out.append([h.key() for h in fn(q, hits, width, L.COMPUTE_ALIGNMENT)])
        L.free_sequence(q)
    return out


def _serve(L, algo: str, qtexts: list[str], hits: int, width: int, slots: int, segments: int, budget: int,
           seed: int, interleave: list[str] | None = None):
    rng = np.random.default_rng(seed)
    delays = rng.exponential(0.01, len(qtexts))
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, t) for t in qtexts]
    server = L.Server(L.SSA_SMITH_WATERMAN if algo == "sw" else L.SSA_NEEDLEMAN_WUNSCH, hits, width,
                      L.COMPUTE_ALIGNMENT, slots=slots, segments=segments, memory_budget=budget)
    tickets = [None] * len(qs)

    def client():
        for i, q in enumerate(qs):
            time.sleep(float(delays[i]))
            tickets[i] = server.submit(q)

    th = threading.Thread(target=client)
    th.start()
    side = _alone(L, algo, interleave, hits, width) if interleave else None
    th.join()
    got, lat = [], []
    for t in tickets:
        h, l = server.wait(t)
        got.append([x.key() for x in h])
        lat.append(l)
    st = server.stats()
    server.stop()
    for q in qs:
        L.free_sequence(q)
    return got, lat, st, side


@pytest.mark.parametrize("slots,segments,budget", [(4, 5, 0), (16, 3, 0), (3, 7, 1)])
def test_served_sw_equals_alone(built_library, slots, segments, budget):
    import libssa_b200 as L
    rng = np.random.default_rng(slots * 100 + segments)
    queries = [W.random_residues(rng, int(rng.integers(20, 700)), W.AA20) for _ in range(14)]
    queries.append(W.random_residues(rng, 1500, W.AA20))          # a multi-pass query
    recs = _db(7 + slots, 600, queries)
    product_setup(L.AMINOACID, ("builtin", "blosum62"), (-11, -1), 100, L.COMPUTE_ON_AVX2, records=recs)
    qtexts = [q.tobytes().decode() for q in queries]
    want = _alone(L, "sw", qtexts, 7, L.BIT_WIDTH_8)
    got, lat, st, _ = _serve(L, "sw", qtexts, 7, L.BIT_WIDTH_8, slots, segments, budget, seed=slots)
    assert got == want
    assert st.completed == len(qtexts) and st.segments == segments
    assert all(x > 0 for x in lat)


def test_served_nw_and_interleaved_searches(built_library):
    import libssa_b200 as L
    rng = np.random.default_rng(3)
    queries = [W.random_residues(rng, int(rng.integers(30, 400)), W.AA20) for _ in range(6)]
    recs = _db(11, 300, queries)
    product_setup(L.AMINOACID, ("builtin", "blosum62"), (-11, -1), 1000, L.COMPUTE_ON_AVX2, records=recs)
    qtexts = [q.tobytes().decode() for q in queries]
    want = _alone(L, "nw", qtexts, 5, L.BIT_WIDTH_16)
    extra = [W.random_residues(rng, 200, W.AA20).tobytes().decode() for _ in range(2)]
    extra_want = _alone(L, "nw", extra, 5, L.BIT_WIDTH_16)
    got, _, _, side = _serve(L, "nw", qtexts, 5, L.BIT_WIDTH_16, 4, 4, 0, seed=5, interleave=extra)
    assert got == want
    assert side == extra_want


def test_server_refuses_queries_beyond_limit(built_library):
    import libssa_b200 as L
    product_setup(L.AMINOACID, ("builtin", "blosum62"), (-11, -1), 1000, L.COMPUTE_ON_AVX2,
                  records=[b"ACDEFGHIKL" * 3])
    server = L.Server(L.SSA_SMITH_WATERMAN, 3, L.BIT_WIDTH_8, L.COMPUTE_SCORE, slots=2, segments=1)
    q = L.init_sequence_fasta(L.READ_FROM_STRING, "A" * (L.SERVE_MAX_QUERY + 1))
    with pytest.raises(ValueError):
        server.submit(q)
    server.stop()
    L.free_sequence(q)
