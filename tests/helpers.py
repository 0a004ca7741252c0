"""Shared helpers of the test suite: fixture access, and one driver per
implementation (the product through its C-ABI, the oracle restatement, the
reference binary) taking the same case description."""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
DATA = os.path.join(GOLDEN, "data")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from libssa_b200 import workloads as W  # noqa: E402


def read_fasta(path: str) -> list[bytes]:
    """Records of a FASTA file, parsed like the database plugin: header lines
    start with '>', sequence lines are concatenated without line breaks."""
    recs: list[bytearray] = []
    with open(path, "rb") as f:
        for line in f:
            if line.startswith(b">"):
                recs.append(bytearray())
            elif recs:
                recs[-1] += line.replace(b"\n", b"").replace(b"\r", b"")
    return [bytes(r) for r in recs]


def first_fasta_sequence(path: str) -> str:
    """The first record of a FASTA file as the reference's query reader sees it."""
    return read_fasta(path)[0].decode()


def golden_matrices() -> dict:
    with open(os.path.join(GOLDEN, "matrices.json")) as f:
        return json.load(f)


def frame_cases() -> list[dict]:
    with open(os.path.join(GOLDEN, "frame_cases.json")) as f:
        return json.load(f)


def golden_cases() -> list[dict]:
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


def wide_cases() -> list[dict]:
    """Score-only searches with a matrix file whose 64-bit values leave the
    int32 range (make_golden.py write_wide_cases)."""
    with open(os.path.join(GOLDEN, "wide_cases.json")) as f:
        return json.load(f)


def matrix_table(spec) -> np.ndarray:
    """spec: ("const", match, mismatch) | ("builtin", name) | ("file", name under golden/data) |
    "const:M,X" | "builtin:name" | "file:name"."""
    if isinstance(spec, str):
        kind, arg = spec.split(":", 1)
        spec = ("const", *map(int, arg.split(","))) if kind == "const" else (kind, arg)
    if spec[0] == "const":
        return oracle.constant_matrix(spec[1], spec[2])
    if spec[0] == "file":
        with open(os.path.join(DATA, spec[1])) as f:
            return oracle.parse_matrix(f.read())
    return np.array(golden_matrices()[spec[1]], dtype=np.int64)


def _digest(queries, flat, offsets) -> str:
    import hashlib
    h = hashlib.sha256()
    for q in queries:
        h.update(q + b"\0")
    h.update(np.ascontiguousarray(offsets, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(flat, dtype=np.uint8).tobytes())
    return h.hexdigest()


def case_inputs(case: dict) -> tuple[list[bytes], list[bytes]]:
    """Queries and records of a golden case, regenerated and checked by hash."""
    if "records" in case:
        return [q.encode() for q in case["queries"]], [r.encode() for r in case["records"]]
    gen = W.CONFIGS[case["workload"]]
    kw = {"seed": case["seed"], "scale": case["scale"]}
    if "n_queries" in case:
        kw["n_queries"] = case["n_queries"]
    w = gen(**kw)
    assert _digest(w.queries, w.db_flat, w.db_offsets) == case["digest"], "workload generator drifted"
    return w.queries, w.db_records()


def lanes(simd: int) -> tuple[int, int]:
    return (32, 16) if simd >= 2 else (16, 8)


# --------------------------------------------------------------------------
# oracle restatement
# --------------------------------------------------------------------------
def oracle_search(algo, width, align, hits, symtype, matrix, gap, chunk, simd, query: bytes, records: list[bytes]):
    nuc = symtype == 0
    l8, l16 = lanes(simd)
    cfg = oracle.SearchConfig(algo=algo, bit_width=width, align_type=align, hitcount=hits, chunk_size=chunk,
                              gap_open=gap[0], gap_extend=gap[1], lanes8=l8, lanes16=l16,
                              matrix=matrix_table(matrix))
    q = oracle.map_codes(query.decode("latin-1"), nuc, True)
    db = [oracle.map_codes(r.decode("latin-1"), nuc, False) for r in records]
    res, ovf = oracle.search(cfg, q, db)
    return [(h.id, h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end) for h in res], ovf


# --------------------------------------------------------------------------
# product (GPU) through the C-ABI
# --------------------------------------------------------------------------
def product_setup(symtype, matrix, gap, chunk, simd, records: list[bytes] | None = None, db_file: str | None = None,
                  strands: int = 1, gencode: tuple[int, int] = (1, 1)):
    """gencode: (query, database) genetic codes."""
    import libssa_b200 as L
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(symtype, strands, gencode[1], gencode[0])
    if isinstance(matrix, str):
        kind, arg = matrix.split(":", 1)
        matrix = ("const", *map(int, arg.split(","))) if kind == "const" else (kind, arg)
    if matrix[0] == "const":
        L.init_constant_scores(matrix[1], matrix[2])
    elif matrix[0] == "file":
        L.init_score_matrix(L.READ_FROM_FILE, os.path.join(DATA, matrix[1]))
    else:
        L.init_score_matrix(L.MATRIX_BUILDIN, matrix[1])
    L.init_gap_penalties(gap[0], gap[1])
    L.set_chunk_size(chunk)
    L.set_simd_compute_mode(simd)
    L.set_thread_count(1)
    if db_file is not None:
        L.init_db(db_file)
    elif records is not None:
        L.load_db_memory(records)


def product_search(algo, width, align, hits, queries: list[bytes], batch: bool = False, frames: bool = False):
    import libssa_b200 as L
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode("latin-1")) for q in queries]
    try:
        if batch:
            lists = L.align_batch(L.SSA_SMITH_WATERMAN if algo == "sw" else L.SSA_NEEDLEMAN_WUNSCH, qs, hits, width,
                                  align)
            ovf = None
        else:
            lists = []
            ovfs = []
            for q in qs:
                fn = L.sw_align if algo == "sw" else L.nw_align
                lists.append(fn(q, hits, width, align))
                st = L.stats()
                ovfs.append((int(st.overflow_8_to_16), int(st.overflow_16_to_64)))
            ovf = ovfs
    finally:
        for q in qs:
            L.free_sequence(q)
    if frames:
        out = [[h.key_frames() for h in lst] for lst in lists]
    else:
        out = [[(h.id, h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end) for h in lst] for lst in lists]
    return out, ovf
