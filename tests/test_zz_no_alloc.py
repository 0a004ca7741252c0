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


def _noalloc_rc(torch, algo: str, query: bytes, db, n: int, max_len: int | None = None):
    import libssa_b200 as L
    import oracle
    d_codes, d_offs, d_lens, longest = db
    qc = torch.from_numpy(oracle.map_codes(query.decode(), False, True)).to("cuda:0")
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda:0")
    rc = L.score64_noalloc(L.SSA_SMITH_WATERMAN if algo == "sw" else L.SSA_NEEDLEMAN_WUNSCH, qc.data_ptr(),
                           qc.numel(), d_codes.data_ptr(), d_offs.data_ptr(), d_lens.data_ptr(), n,
                           longest if max_len is None else max_len, out.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    return rc, out.cpu().numpy()


def _noalloc(torch, algo: str, query: bytes, db, n: int) -> np.ndarray:
    import libssa_b200 as L
    rc, out = _noalloc_rc(torch, algo, query, db, n)
    assert rc == L.NOALLOC_OK
    return out


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


def test_noalloc_sequence_longer_than_its_bound(built_library):
    """A caller that passes max_seq_len 4096 but holds a longer sequence gets
    SSA_B200_NOALLOC_ESEQLEN (the per-warp boundary rows of a multi-pass query
    hold 4096 columns), and every other sequence's score is still right."""
    torch = pytest.importorskip("torch")
    import libssa_b200 as L
    records = _records(13, 60, 900)
    records[7] = _protein(np.random.default_rng(14), 5000)
    product_setup(L.AMINOACID, ("builtin", "blosum62"), (-11, -1), 1000, L.COMPUTE_ON_AVX2, records=records)
    nonempty = [i for i, r in enumerate(records) if r]
    query = _protein(np.random.default_rng(23), 600)           # three 256-row passes
    want = _regular_scores("sw", query, len(nonempty))
    db = _device_db(torch, records)
    rc, got = _noalloc_rc(torch, "sw", query, db, len(records), max_len=L.NOALLOC_MAX_SEQ_LEN)
    assert rc == L.NOALLOC_ESEQLEN
    assert all(int(got[i]) == want[i] for i in nonempty if i != 7)


_NO_GROWTH_SCRIPT = r"""
import sys
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
import numpy as np
import torch
import libssa_b200 as L
import test_zz_no_alloc as T
from helpers import product_setup
L.load()
records = T._records(15, 200, 1200)
product_setup(L.AMINOACID, ("builtin", "blosum62"), (-11, -1), 1000, L.COMPUTE_ON_AVX2)
db = T._device_db(torch, records)
d_codes, d_offs, d_lens, longest = db
qs = [torch.from_numpy(np.frombuffer(T._protein(np.random.default_rng(s), n), np.uint8) % 20 + 1).to("cuda:0")
      for s, n in ((31, 300), (32, 700))]
outs = [torch.zeros(len(records), dtype=torch.int32, device="cuda:0") for _ in range(4)]
stream = torch.cuda.current_stream().cuda_stream
def call(algo, q, out):
    rc = L.score64_noalloc(algo, q.data_ptr(), q.numel(), d_codes.data_ptr(), d_offs.data_ptr(), d_lens.data_ptr(),
                           len(records), longest, out.data_ptr(), stream)
    assert rc == L.NOALLOC_OK, rc
torch.cuda.synchronize()
call(L.SSA_SMITH_WATERMAN, qs[0], outs[0])          # set-up call: Smith-Waterman only
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
for k in range(3):
    call(L.SSA_SMITH_WATERMAN, qs[k % 2], outs[1])
    call(L.SSA_NEEDLEMAN_WUNSCH, qs[k % 2], outs[2])
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
print("free", free0, free1)
assert free1 == free0, (free0, free1)
"""


def test_noalloc_calls_after_setup_allocate_nothing(built_library, tmp_path):
    """In a fresh process: after one Smith-Waterman set-up call, repeated
    Smith-Waterman and Needleman-Wunsch calls leave the device's free memory
    unchanged -- the set-up loaded every kernel a call launches, so none is
    loaded (and allocated for) later."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    script = tmp_path / "no_growth.py"
    script.write_text(_NO_GROWTH_SCRIPT)
    r = subprocess.run([sys.executable, str(script), os.path.dirname(here), here], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
