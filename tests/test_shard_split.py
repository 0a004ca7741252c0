"""The database-sharded split: contiguous record ranges per rank, a gather of
the per-record results (score, blocks of the entry-width lane, blocks of the
16-bit lane) to one rank, and that rank's replay of the reference's lane
schedule and heap (ssa_b200_replay_gathered).

On the CPU the per-record results come from the oracle's lane emulation
(test data standing in for each rank's GPU pass); what is checked is the
product's gather layout and replay: the replayed lists must equal a whole
search of the database -- the oracle restatement's, which is pinned to the
reference -- with the same hits, scores, tie order and overflow counters.  Two
gloo ranks run the split as processes.  The GPU test runs the shards'
entry passes on the device (ssa_b200_shard_scores) and compares with
sw_align/nw_align, CIGARs included.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from helpers import ROOT, lanes, matrix_table, oracle_search, product_setup
from libssa_b200 import workloads as W


def _case(seed: int):
    rng = np.random.default_rng(seed)
    nuc = bool(seed % 3 == 2)
    alpha = W.NT4 if nuc else W.AA20
    qs = [W.random_residues(rng, int(rng.integers(20, 400)), alpha) for _ in range(3)]
    recs = []
    for _ in range(int(rng.integers(150, 400))):
        r = rng.random()
        if r < 0.12:
            recs.append(W.mutate(rng, qs[int(rng.integers(0, 3))], alpha, 0.05, 0.02, (1, 4)))
        elif r < 0.16:
            recs.append(W.mutate(rng, np.tile(qs[int(rng.integers(0, 3))], 3), alpha, 0.01, 0.0, (1, 1)))
        elif r < 0.18:
            recs.append(np.zeros(0, np.uint8))
        else:
            recs.append(W.random_residues(rng, int(rng.integers(1, 500)), alpha))
    algo = ["sw", "nw"][seed % 2]
    width = [8, 16, 64, 8][seed % 4]
    matrix = "const:3,-2" if nuc else "builtin:" + ["blosum62", "blosum50"][seed % 2]
    return dict(algo=algo, width=width, hits=int(rng.integers(3, 15)), symtype=0 if nuc else 1, matrix=matrix,
                gap=(-int(rng.integers(3, 12)), -int(rng.integers(1, 3))), chunk=[1000, 50, 13][seed % 3],
                simd=[2, 1][seed % 2], queries=[q.tobytes() for q in qs], records=[r.tobytes() for r in recs])


def oracle_triples(c: dict, lo: int, hi: int):
    """Per (query, record in [lo, hi)): final score, blocks of the overflowing
    entry-width lane, blocks of the overflowing 16-bit lane (-1: the lane
    reported) -- what each rank's passes produce."""
    l8, l16 = lanes(c["simd"])
    cfg = oracle.SearchConfig(algo=c["algo"], bit_width=c["width"], align_type=0, hitcount=c["hits"],
                              chunk_size=c["chunk"], gap_open=c["gap"][0], gap_extend=c["gap"][1], lanes8=l8,
                              lanes16=l16, matrix=matrix_table(c["matrix"]))
    nuc = c["symtype"] == 0
    qcodes = [oracle.map_codes(q.decode(), nuc, True) for q in c["queries"]]
    dcodes = [oracle.map_codes(r.decode(), nuc, False) for r in c["records"][lo:hi]]
    n = len(qcodes)
    sc = np.zeros((n, hi - lo), np.int64)
    be = np.full((n, hi - lo), -1, np.int32)
    b16 = np.full((n, hi - lo), -1, np.int32)
    for qi, q in enumerate(qcodes):
        for k, d in enumerate(dcodes):
            if len(d) == 0:
                continue
            w = c["width"]
            while True:
                s, ovf, nb = oracle.lane_result(cfg, w, q, d)
                if w == 64 or not ovf:
                    sc[qi, k] = s
                    break
                if w == c["width"]:
                    be[qi, k] = nb
                else:
                    b16[qi, k] = nb
                w = 16 if w == 8 else 64
    return sc, be, b16


def _product_replay(c: dict, sc, be, b16, align: int = 0):
    import libssa_b200 as L
    L.load()
    product_setup(c["symtype"], c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in c["queries"]]
    try:
        algo = L.SSA_SMITH_WATERMAN if c["algo"] == "sw" else L.SSA_NEEDLEMAN_WUNSCH
        lists = L.replay_gathered(algo, qs, c["hits"], c["width"], align, sc, be, b16)
        ovf = L.query_overflows()
    finally:
        for q in qs:
            L.free_sequence(q)
    return [[(h.id, h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end) for h in lst] for lst in lists], ovf


def _expected(c: dict):
    out = []
    for q in c["queries"]:
        res, ovf = oracle_search(c["algo"], c["width"], 0, c["hits"], c["symtype"], c["matrix"], c["gap"],
                                 c["chunk"], c["simd"], q, c["records"])
        out.append((res, tuple(ovf)))
    return out


def _bounds(n: int, parts: int) -> list[int]:
    return [round(i * n / parts) for i in range(parts + 1)]


@pytest.mark.parametrize("seed", range(8))
@pytest.mark.parametrize("parts", [1, 3])
def test_gathered_replay_equals_whole_search(built_library, seed, parts):
    c = _case(seed)
    n = len(c["records"])
    b = _bounds(n, parts)
    pieces = [oracle_triples(c, b[i], b[i + 1]) for i in range(parts)]
    sc, be, b16 = (np.concatenate([p[k] for p in pieces], axis=1) for k in range(3))
    got, ovf = _product_replay(c, sc, be, b16)
    for qi, (res, eovf) in enumerate(_expected(c)):
        assert got[qi] == res, (seed, qi)
        assert tuple(ovf[qi]) == eovf, (seed, qi)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, seed: int, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        c = _case(seed)
        b = _bounds(len(c["records"]), world)
        part = oracle_triples(c, b[rank], b[rank + 1])          # this rank's contiguous record range
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(part, gathered, dst=0)
        if rank == 0:
            sc, be, b16 = (np.concatenate([p[k] for p in gathered], axis=1) for k in range(3))
            got, ovf = _product_replay(c, sc, be, b16)
            out.put((got, [tuple(o) for o in ovf], [tuple(x.shape) for x in (sc, be, b16)]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("seed", [0, 3])
def test_two_gloo_ranks_gather_to_the_replaying_rank(built_library, seed):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, seed, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, ovf, shapes = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    c = _case(seed)
    assert shapes == [(len(c["queries"]), len(c["records"]))] * 3
    for qi, (res, eovf) in enumerate(_expected(c)):
        assert got[qi] == res, qi
        assert ovf[qi] == eovf, qi


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(6))
def test_device_shards_replayed_equal_plain_search(built_library, seed):
    """Three record ranges scored on the device one after the other (as three
    ranks would), gathered, replayed with alignments: equal to the plain
    sw_align/nw_align lists, CIGARs included."""
    import libssa_b200 as L
    c = _case(seed)
    product_setup(c["symtype"], c["matrix"], c["gap"], c["chunk"], c["simd"], records=c["records"])
    algo = L.SSA_SMITH_WATERMAN if c["algo"] == "sw" else L.SSA_NEEDLEMAN_WUNSCH
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in c["queries"]]
    try:
        b = _bounds(len(c["records"]), 3)
        pieces = [L.shard_scores(algo, qs, c["width"], b[i], b[i + 1]) for i in range(3)]
        sc, be, b16 = (np.concatenate([p[k] for p in pieces], axis=1) for k in range(3))
        want_triples = oracle_triples(c, 0, len(c["records"]))
        for k in range(3):
            assert np.array_equal((sc, be, b16)[k], want_triples[k]), k
        got = L.replay_gathered(algo, qs, c["hits"], c["width"], L.COMPUTE_ALIGNMENT, sc, be, b16)
        fn = L.sw_align if c["algo"] == "sw" else L.nw_align
        want = [fn(q, c["hits"], c["width"], L.COMPUTE_ALIGNMENT) for q in qs]
    finally:
        for q in qs:
            L.free_sequence(q)
    key = lambda lst: [(h.id, h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end) for h in lst]  # noqa: E731
    assert [key(x) for x in got] == [key(x) for x in want]


def test_bench_record_ranges_cover_the_database_in_chunks():
    """The benchmark's --split db layout: contiguous ranges, together the whole
    database, cut at multiples of 1,000 records, about equal residues."""
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(3)
    lens = W.gamma_lengths(rng, 23_456, 350.0, 20, 35_000)
    for parts in (1, 2, 3, 8):
        b = bench.record_ranges(lens, parts)
        assert b[0] == 0 and b[-1] == len(lens) and len(b) == parts + 1
        assert all(b[i] <= b[i + 1] for i in range(parts))
        assert all(x % 1000 == 0 for x in b[1:-1])
        res = [int(lens[b[i]:b[i + 1]].sum()) for i in range(parts)]
        assert max(res) - min(res) <= 2 * 1000 * 35_000 / 10 + lens.sum() * 0.1
