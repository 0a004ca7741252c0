"""Parity at the full sizes the build is measured on.

Golden runs of the reference itself (tests/golden/scale_*.json, written by
tests/golden/make_scale_golden.py: sw_align/nw_align at 1 thread, AVX2,
chunk 1000, COMPUTE_ALIGNMENT) against the product through its public C-ABI,
on the complete databases and through the same calls the benchmark times:

* 1,024 queries vs 500,000 sequences in ONE ssa_align_batch call (score
  buffer split into sub-batches, every rows-per-thread class, the 16-bit
  cascade of the 8,000-35,000-residue near-copies, multi-warp traceback
  groups), checked on a 64-query sample;
* 64 nucleotide queries vs 200,000 sequences, Needleman-Wunsch, 16-bit
  entry, top 20: every query;
* the 200-request served stream vs 1,000,000 resident sequences through the
  server (all requests in flight together);
* 8 long pairs (5,000-30,000 residues), SW and NW with CIGARs.

Bit-exact: IDs, scores, order (ties included), CIGARs, coordinates and, for
the searches, the per-query 8->16 / 16->64 overflow counters.
"""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN, _digest
from libssa_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _golden(name: str) -> dict:
    with open(os.path.join(GOLDEN, f"scale_{name}.json")) as f:
        return json.load(f)


def _rows(hits) -> list[list]:
    return [[h.id, h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end] for h in hits]


def _setup(L, g: dict, w=None, flat=None, offsets=None):
    s = g["settings"]
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(s["symtype"], L.FORWARD_STRAND, 1, 1)
    kind, arg = s["matrix"].split(":", 1)
    if kind == "const":
        L.init_constant_scores(*map(int, arg.split(",")))
    else:
        L.init_score_matrix(L.MATRIX_BUILDIN, arg)
    L.init_gap_penalties(*s["gap"])
    L.set_chunk_size(s["chunk"])
    L.set_simd_compute_mode(s["simd"])
    L.set_thread_count(1)
    if w is not None:
        L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)


def _batched(L, name: str, w, algo: int, width: int):
    g = _golden(name)
    assert _digest(w.queries, w.db_flat, w.db_offsets) == g["digest"], "workload generator drifted"
    _setup(L, g, w)
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in w.queries]
    try:
        lists = L.align_batch(algo, qs, g["settings"]["hits"], width, L.COMPUTE_ALIGNMENT)
        ovf = L.query_overflows()
    finally:
        for q in qs:
            L.free_sequence(q)
    assert len(ovf) == len(w.queries)
    bad = []
    for i in g["sample"]:
        exp = g["results"][str(i)]
        if _rows(lists[i]) != exp["hits"] or list(ovf[i]) != exp["ovf"]:
            bad.append(i)
    assert not bad, f"{len(bad)} of {len(g['sample'])} sampled queries differ: {bad[:8]}"


def test_sw_batched_1024_queries_full_database(built_library):
    import libssa_b200 as L
    L.load()
    _batched(L, "sw_batched", W.sw_batched(seed=3), L.SSA_SMITH_WATERMAN, L.BIT_WIDTH_8)


def test_nw_nucleotide_64_queries_full_database(built_library):
    import libssa_b200 as L
    L.load()
    _batched(L, "nw_nucleotide", W.nw_nucleotide(seed=2), L.SSA_NEEDLEMAN_WUNSCH, L.BIT_WIDTH_16)


def test_served_200_requests_full_database(built_library):
    import libssa_b200 as L
    L.load()
    g = _golden("sw_served")
    w = W.sw_served_db(seed=g["gen"]["seed"])
    queries = W.served_queries(seed=g["gen"]["query_seed"], n=g["gen"]["queries"])
    assert _digest(queries, w.db_flat, w.db_offsets) == g["digest"], "workload generator drifted"
    _setup(L, g, w)
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in queries]
    server = L.Server(L.SSA_SMITH_WATERMAN, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT, slots=64, segments=8)
    try:
        tickets = [server.submit(q) for q in qs]
        got = [_rows(server.wait(t)[0]) for t in tickets]
    finally:
        server.stop()
        for q in qs:
            L.free_sequence(q)
    bad = [i for i in g["sample"] if got[i] != g["results"][str(i)]["hits"]]
    assert not bad, f"{len(bad)} of {len(g['sample'])} requests differ: {bad[:8]}"


def test_long_pairs_sample(built_library):
    import libssa_b200 as L
    L.load()
    g = _golden("long_pairs")
    pairs = W.long_pairs(seed=g["gen"]["seed"], n_pairs=g["gen"]["n_pairs"])
    import hashlib
    h = hashlib.sha256()
    for a, b in pairs:
        h.update(a + b"\0" + b + b"\0")
    assert h.hexdigest() == g["digest"], "workload generator drifted"
    sample = g["sample"]
    s = g["settings"]
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)
    L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
    L.init_gap_penalties(*s["gap"])
    L.set_chunk_size(s["chunk"])
    L.set_simd_compute_mode(s["simd"])
    L.load_db_memory([pairs[k][1] for k in sample])
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, pairs[k][0].decode()) for k in sample]
    try:
        for algo, name in ((L.SSA_SMITH_WATERMAN, "sw"), (L.SSA_NEEDLEMAN_WUNSCH, "nw")):
            lists = L.align_pairs(algo, qs, list(range(len(sample))), L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
            for j, k in enumerate(sample):
                exp = g["results"][str(k)][name]
                got = _rows(lists[j])
                # the pair's database holds one sequence: its ID there is 0
                assert [[0] + r[1:] for r in got] == exp, (name, k)
    finally:
        for q in qs:
            L.free_sequence(q)
