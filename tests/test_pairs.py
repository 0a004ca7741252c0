"""Long-pair batches (ssa_align_pairs): each query against one database
sequence alone.

A pair's list must equal what sw_align / nw_align(query, 1, ...) return for the
query against a database holding only that sequence: the oracle restatement
searched with that one record (score, CIGAR, coordinates; the hit's ID is the
sequence's ID in the full database), the reference binary on a few pairs, pairs
long enough that scores leave 16 bits (the reference's 16 -> 64-bit path),
several queries sharing a sequence, an empty sequence (no hit), and the
traceback split into memory waves with unchanged results.
"""
import numpy as np
import pytest

import oracle
from helpers import oracle_search, product_setup
from libssa_b200 import workloads as W

MATRIX = ("builtin", "blosum62")
GAP = (-11, -1)


def _pairs(seed: int, n: int, lo: int, hi: int) -> tuple[list[bytes], list[bytes], list[int]]:
    """n queries, a database of their partners (related or not) in shuffled
    order plus an empty record and decoys, and each query's partner ID."""
    rng = np.random.default_rng(seed)
    queries, partners = [], []
    for i in range(n):
        a = W.random_residues(rng, int(rng.integers(lo, hi + 1)), W.AA20)
        if i % 4 == 3:
            b = W.random_residues(rng, int(rng.integers(lo, hi + 1)), W.AA20)
        else:
            b = W.mutate(rng, a, W.AA20, 1.0 - rng.uniform(0.85, 0.99), 0.01, (1, 20))
        queries.append(a.tobytes())
        partners.append(b.tobytes())
    records = partners + [b""] + [W.random_residues(rng, 50, W.AA20).tobytes() for _ in range(3)]
    perm = rng.permutation(len(records))
    shuffled = [records[k] for k in perm]
    where = {int(k): pos for pos, k in enumerate(perm)}
    ids = [where[i] for i in range(n)]
    ids[1] = ids[0]                      # two queries share a sequence
    ids[2] = where[n]                    # the empty record: no hit
    return queries, shuffled, ids


def _product(algo: str, width: int, align: int, queries: list[bytes], ids: list[int]):
    import libssa_b200 as L
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in queries]
    try:
        lists = L.align_pairs(L.SSA_SMITH_WATERMAN if algo == "sw" else L.SSA_NEEDLEMAN_WUNSCH, qs, ids, width,
                              align)
    finally:
        for q in qs:
            L.free_sequence(q)
    return [[(h.id, h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end) for h in lst] for lst in lists]


def _oracle(algo: str, width: int, align: int, query: bytes, record: bytes, db_id: int):
    hits, _ = oracle_search(algo, width, align, 1, 1, MATRIX, GAP, 1000, 2, query, [record])
    return [(db_id,) + h[1:] for h in hits]


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["sw", "nw"])
@pytest.mark.parametrize("width,align", [(8, 1), (16, 1), (64, 1), (16, 0)])
def test_pairs_match_oracle(built_library, algo, width, align):
    queries, records, ids = _pairs(11 + width + align, 16, 20, 1400)
    product_setup(1, MATRIX, GAP, 1000, 2, records=records)
    got = _product(algo, width, align, queries, ids)
    for i, q in enumerate(queries):
        assert got[i] == _oracle(algo, width, align, q, records[ids[i]], ids[i]), i
    assert got[2] == []


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["sw", "nw"])
def test_pairs_on_warp_groups_match_oracle(built_library, algo):
    """Pairs of 2,500-4,000 residues: the traceback runs them on groups of 4
    warps (more than 8M cells, up to 16 stripes of 256 query rows, so the
    boundary rows travel through shared memory and the group's global row)."""
    queries, records, ids = _pairs(23, 8, 2500, 4000)
    product_setup(1, MATRIX, GAP, 1000, 2, records=records)
    got = _product(algo, 16, 1, queries, ids)
    for i, q in enumerate(queries):
        assert got[i] == _oracle(algo, 16, 1, q, records[ids[i]], ids[i]), i


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["sw", "nw"])
def test_long_pairs_beyond_16_bits(built_library, algo):
    """Pairs of 9,000 and 14,000 residues: scores above 32767 take the reference's 64-bit path."""
    rng = np.random.default_rng(29)
    queries, records = [], []
    for n in (9000, 14000):
        a = W.random_residues(rng, n, W.AA20)
        queries.append(a.tobytes())
        records.append(W.mutate(rng, a, W.AA20, 0.03, 0.01, (1, 20)).tobytes())
    product_setup(1, MATRIX, GAP, 1000, 2, records=records)
    got16 = _product(algo, 16, 1, queries, [0, 1])
    got64 = _product(algo, 64, 1, queries, [0, 1])
    assert got16 == got64
    for i, q in enumerate(queries):
        want = _oracle(algo, 64, 1, q, records[i], i)
        assert got64[i] == want, i
        if algo == "sw":
            assert want[0][1] > 32767


def _asymmetric_table() -> str:
    """A score table with M[x][y] != M[y][x]: the region passes score
    [query][db] and the search [db][query], so the forward pass's maximum is
    not the score and the pair keeps its separate score pass."""
    aa = "ARNDCQEGHILKMFPSTWYV"
    lines = ["   " + "  ".join(aa)]
    for i, x in enumerate(aa):
        row = [5 if i == j else ((i * 7 + j * 3) % 9) - 6 for j in range(20)]
        lines.append(x + " " + " ".join(f"{v:2d}" for v in row))
    return "\n".join(lines) + "\n"


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["sw", "nw"])
def test_pairs_asymmetric_table(built_library, algo):
    import libssa_b200 as L
    text = _asymmetric_table()
    queries, records, ids = _pairs(31, 10, 100, 2000)
    product_setup(1, MATRIX, GAP, 1000, 2, records=records)
    L.init_score_matrix(L.READ_FROM_STRING, text)
    try:
        got = _product(algo, 16, 1, queries, ids)
    finally:
        L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
    cfg = oracle.SearchConfig(algo=algo, bit_width=16, align_type=1, hitcount=1, gap_open=GAP[0], gap_extend=GAP[1],
                              matrix=oracle.parse_matrix(text))
    for i, q in enumerate(queries):
        hits, _ = oracle.search(cfg, oracle.map_codes(q.decode(), False, True),
                                [oracle.map_codes(records[ids[i]].decode(), False, False)])
        assert got[i] == [(ids[i], h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end) for h in hits], i


@pytest.mark.gpu
def test_pairs_in_memory_waves(built_library):
    import libssa_b200 as L
    queries, records, ids = _pairs(5, 24, 200, 3000)
    product_setup(1, MATRIX, GAP, 1000, 2, records=records)
    whole = _product("sw", 16, 1, queries, ids)
    try:
        L.set_traceback_memory(1 << 20)           # a few hits per wave
        waved = _product("sw", 16, 1, queries, ids)
        waved_nw = _product("nw", 16, 1, queries, ids)
    finally:
        L.set_traceback_memory(0)
    assert waved == whole
    assert waved_nw == _product("nw", 16, 1, queries, ids)


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref/ref_run is not built")
@pytest.mark.parametrize("algo,width", [("sw", 8), ("nw", 16)])
def test_pairs_match_reference_binary(built_library, tmp_path, algo, width):
    queries, records, ids = _pairs(7, 5, 300, 2500)
    product_setup(1, MATRIX, GAP, 1000, 2, records=records)
    got = _product(algo, width, 1, queries, ids)
    for i, q in enumerate(queries):
        db = str(tmp_path / f"pair{i}.sdb")
        oracle.write_sdb(db, seqs=[records[ids[i]]])
        ref = oracle.run_reference(db, [q.decode()], algo=algo, width=width, align=1, hits=1, symtype=1,
                                   matrix="builtin:blosum62", gap=GAP, workdir=str(tmp_path))[0]
        want = [(ids[i], h["score"], h["cigar"], h["q_start"], h["q_end"], h["d_start"], h["d_end"])
                for h in ref["hits"]]
        assert got[i] == want, i


@pytest.mark.gpu
def test_pairs_refuse_unknown_ids(built_library):
    import libssa_b200 as L
    product_setup(1, MATRIX, GAP, 1000, 2, records=[b"ACDEFGHIKL"])
    q = L.init_sequence_fasta(L.READ_FROM_STRING, "ACDEF")
    try:
        with pytest.raises(ValueError):
            L.align_pairs(L.SSA_SMITH_WATERMAN, [q], [1], 16, L.COMPUTE_SCORE)
    finally:
        L.free_sequence(q)


def test_pairs_refuse_truncating_settings(built_library):
    """Settings whose narrow lanes would truncate (here gapO + gapE below the
    int8 range at the 8-bit entry) are refused before any device work."""
    import libssa_b200 as L
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)
    L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
    L.init_gap_penalties(-100, -100)
    L.load_db_memory([b"ACDEFGHIKL"])
    q = L.init_sequence_fasta(L.READ_FROM_STRING, "ACDEF")
    try:
        with pytest.raises(ValueError):
            L.align_pairs(L.SSA_SMITH_WATERMAN, [q], [0], L.BIT_WIDTH_8, L.COMPUTE_SCORE)
    finally:
        L.free_sequence(q)
        L.init_gap_penalties(-11, -1)


def test_pairs_refuse_two_strand_setups(built_library):
    """A pair is one query sequence against one database sequence; setups that
    search several strands or frames per query are refused before any device
    work."""
    import libssa_b200 as L
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.NUCLEOTIDE, L.BOTH_STRANDS, 1, 1)
    L.init_constant_scores(2, -3)
    L.init_gap_penalties(-5, -2)
    L.load_db_memory([b"ACGTACGTAC"])
    q = L.init_sequence_fasta(L.READ_FROM_STRING, "ACGTA")
    try:
        with pytest.raises(ValueError):
            L.align_pairs(L.SSA_NEEDLEMAN_WUNSCH, [q], [0], L.BIT_WIDTH_16, L.COMPUTE_SCORE)
    finally:
        L.free_sequence(q)
        L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)
        L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
        L.init_gap_penalties(-11, -1)
