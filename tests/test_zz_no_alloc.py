"""Allocation-free scoring, ssa_b200_score64_noalloc(), through the C-ABI.

Each call must return exactly the scores of the regular BIT_WIDTH_64 search
(sw_align / nw_align, same matrix, gaps and database), also on back-to-back
calls that reuse its fixed device buffers.  The file sorts last so that the
calls also run after everything else in the suite has used the device.
"""
import numpy as np
import pytest

from helpers import product_setup

pytestmark = pytest.mark.gpu

AA = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", dtype=np.uint8)


def _protein(rng, n: int) -> bytes:
    return AA[rng.integers(0, len(AA), size=n)].tobytes()


def _records(seed: int, n: int, max_len: int) -> list[bytes]:
    rng = np.random.default_rng(seed)
    lens = rng.integers(1, max_len + 1, size=n)
    lens[::37] = 0                                   # empty records score 0 and are never hits
    lens[5] = max_len
    return [_protein(rng, int(k)) for k in lens]


def _regular_scores(algo: str, query: bytes, n_nonempty: int) -> dict[int, int]:
    import libssa_b200 as L
    q = L.init_sequence_fasta(L.READ_FROM_STRING, query.decode())
    try:
        fn = L.sw_align if algo == "sw" else L.nw_align
        hits = fn(q, n_nonempty, L.BIT_WIDTH_64, L.COMPUTE_SCORE)
    finally:
        L.free_sequence(q)
    return {h.id: h.score for h in hits}


def _device_db(torch, records: list[bytes]):
    import oracle
    codes = [oracle.map_codes(r.decode(), False, False) for r in records]
    lens = np.array([len(c) for c in codes], dtype=np.int32)
    offs = np.zeros(len(codes), dtype=np.int64)
    offs[1:] = np.cumsum(lens[:-1])
    flat = np.concatenate([c for c in codes if len(c)]).astype(np.uint8)
    dev = torch.device("cuda:0")
    return (torch.from_numpy(flat).to(dev), torch.from_numpy(offs).to(dev), torch.from_numpy(lens).to(dev),
            int(lens.max()))


def _noalloc(torch, algo: str, query: bytes, db, n: int) -> np.ndarray:
    import libssa_b200 as L
    import oracle
    d_codes, d_offs, d_lens, max_len = db
    qc = torch.from_numpy(oracle.map_codes(query.decode(), False, True)).to("cuda:0")
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda:0")
    rc = L.score64_noalloc(L.SSA_SMITH_WATERMAN if algo == "sw" else L.SSA_NEEDLEMAN_WUNSCH, qc.data_ptr(),
                           qc.numel(), d_codes.data_ptr(), d_offs.data_ptr(), d_lens.data_ptr(), n, max_len,
                           out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == L.NOALLOC_OK
    return out.cpu().numpy()


@pytest.mark.parametrize("algo", ["sw", "nw"])
def test_noalloc_matches_regular_search(built_library, algo):
    torch = pytest.importorskip("torch")
    import libssa_b200 as L
    records = _records(11 if algo == "sw" else 12, 300, 1500)
    product_setup(L.AMINOACID, ("builtin", "blosum62"), (-11, -1), 1000, L.COMPUTE_ON_AVX2, records=records)
    nonempty = [i for i, r in enumerate(records) if r]
    queries = [_protein(np.random.default_rng(21), 700), _protein(np.random.default_rng(22), 97)]
    db = _device_db(torch, records)
    results = []
    for query in queries + queries[:1]:              # two different calls in a row, then a repeat
        want = _regular_scores(algo, query, len(nonempty))
        got = _noalloc(torch, algo, query, db, len(records))
        assert sorted(want) == nonempty
        assert all(int(got[i]) == want[i] for i in nonempty), algo
        assert all(int(got[i]) == 0 for i, r in enumerate(records) if not r)
        results.append(got)
    assert np.array_equal(results[0], results[2])


def test_noalloc_rejects_sizes_beyond_limits(built_library):
    torch = pytest.importorskip("torch")
    import libssa_b200 as L
    product_setup(L.AMINOACID, ("builtin", "blosum62"), (-11, -1), 1000, L.COMPUTE_ON_AVX2)
    buf = torch.zeros(16, dtype=torch.int64, device="cuda:0")
    p = buf.data_ptr()
    sw = L.SSA_SMITH_WATERMAN
    assert L.score64_noalloc(sw, p, L.NOALLOC_MAX_QUERY + 1, p, p, p, 1, 10, p) == L.NOALLOC_ETOOBIG
    assert L.score64_noalloc(sw, p, 10, p, p, p, 1, L.NOALLOC_MAX_SEQ_LEN + 1, p) == L.NOALLOC_ETOOBIG
    assert L.score64_noalloc(sw, p, 10, p, p, p, L.NOALLOC_MAX_SEQS + 1, 10, p) == L.NOALLOC_ETOOBIG
    assert L.score64_noalloc(7, p, 10, p, p, p, 1, 10, p) == L.NOALLOC_EINVAL
