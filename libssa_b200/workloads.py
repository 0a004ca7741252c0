"""Seeded synthetic database-search workloads.

No public benchmark database is available offline (the reference's own
Swiss-Prot / Rfam files are not distributed with it), so every workload is
generated from a fixed ``numpy.random.default_rng`` seed with the shapes,
length distributions and residue distributions of the five configurations the
B200 build is measured on:

1. ``sw_plain``   -- 1 protein query of 375 residues vs 10,000 sequences,
   lengths gamma(shape 2, mean 350) clipped to [20, 5000]; BLOSUM62, gaps
   11/1, 8-bit entry, top 10 with CIGAR.
2. ``nw_nucleotide`` -- 64 queries U[150, 600] over ACGT vs 200,000 sequences
   U[100, 1500]; 5% are mutated copies of a query (10% substitutions, 2% indel
   events of length 1-5); match 2 / mismatch -3, gaps 5/2, 16-bit entry,
   top 20 with CIGAR.
3. ``sw_batched`` -- 1,024 queries, lognormal(median 300, sigma 0.7) clipped
   to [30, 5000], vs 500,000 sequences gamma(2, mean 350) clipped to
   [20, 35000]; 1% of the sequences are 8,000-35,000 residue copies of a query
   (the query tiled to that length) at 98% identity.  BLOSUM62, gaps 11/1,
   8-bit entry, top 10 with CIGAR.
4. ``sw_served``  -- 1,000,000 sequences gamma(2, mean 350) clipped to
   [20, 5000]; queries lognormal(median 300, sigma 0.8) clipped to [30, 5000]
   arriving as a Poisson process.
5. ``long_pairs`` -- pairs of U[5000, 30000]-residue sequences and a mutated
   copy (85-99% identity, 1% indel events of length 1-20).

Residues are i.i.d. uniform over the 20 standard amino acids or ACGT.
``scale`` shrinks the counts for parity tests (same distributions).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

AA20 = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", dtype=np.uint8)
NT4 = np.frombuffer(b"ACGT", dtype=np.uint8)


@dataclass
class Workload:
    name: str
    algo: str                      # "sw" or "nw"
    bit_width: int
    hitcount: int
    align_type: int
    symtype: int                   # 1 amino acid, 0 nucleotide
    matrix: str                    # "builtin:blosum62" or "const:M,X"
    gap: tuple[int, int]
    queries: list[bytes]
    db_flat: np.ndarray            # ASCII residues, all records back to back
    db_offsets: np.ndarray         # uint64, n + 1
    meta: dict = field(default_factory=dict)

    @property
    def n_db(self) -> int:
        return len(self.db_offsets) - 1

    def db_record(self, i: int) -> bytes:
        return self.db_flat[self.db_offsets[i]:self.db_offsets[i + 1]].tobytes()

    def db_records(self) -> list[bytes]:
        return [self.db_record(i) for i in range(self.n_db)]

    def cells(self) -> int:
        """Sum over queries of query length x database residues."""
        res = int(self.db_offsets[-1])
        return sum(len(q) for q in self.queries) * res


def gamma_lengths(rng, n, mean=350.0, lo=20, hi=5000):
    return np.clip(np.rint(rng.gamma(2.0, mean / 2.0, n)), lo, hi).astype(np.int64)


def lognormal_lengths(rng, n, median=300.0, sigma=0.7, lo=30, hi=5000):
    return np.clip(np.rint(np.exp(np.log(median) + sigma * rng.standard_normal(n))), lo, hi).astype(np.int64)


def random_residues(rng, n, alphabet) -> np.ndarray:
    return alphabet[rng.integers(0, len(alphabet), n)]


def mutate(rng, seq: np.ndarray, alphabet, sub_rate: float, indel_rate: float, indel_len: tuple[int, int]):
    """Substitutions at sub_rate per residue, indel events at indel_rate per
    residue (insertion or deletion with equal odds, length uniform in
    indel_len)."""
    n = len(seq)
    out = seq.copy()
    subs = rng.random(n) < sub_rate
    out[subs] = random_residues(rng, int(subs.sum()), alphabet)
    ev = np.flatnonzero(rng.random(n) < indel_rate)
    if len(ev) == 0:
        return out
    pieces = []
    prev = 0
    for pos in ev:
        if pos < prev:
            continue
        length = int(rng.integers(indel_len[0], indel_len[1] + 1))
        pieces.append(out[prev:pos])
        if rng.random() < 0.5:
            pieces.append(random_residues(rng, length, alphabet))   # insertion
            prev = pos
        else:
            prev = min(n, pos + length)                             # deletion
    pieces.append(out[prev:])
    return np.concatenate(pieces)


def _pack(records: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    offsets = np.zeros(len(records) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([len(r) for r in records])
    flat = np.concatenate(records).astype(np.uint8) if records else np.zeros(0, np.uint8)
    return flat, offsets


def sw_plain(seed: int = 1, scale: float = 1.0) -> Workload:
    rng = np.random.default_rng(seed)
    q = random_residues(rng, 375, AA20)
    n = max(1, int(round(10_000 * scale)))
    lens = gamma_lengths(rng, n)
    flat = random_residues(rng, int(lens.sum()), AA20)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    return Workload("sw_plain", "sw", 8, 10, 1, 1, "builtin:blosum62", (-11, -1), [q.tobytes()], flat, offsets,
                    {"seed": seed, "scale": scale})


def nw_nucleotide(seed: int = 2, scale: float = 1.0, n_queries: int = 64) -> Workload:
    rng = np.random.default_rng(seed)
    nq = n_queries
    queries = [random_residues(rng, int(rng.integers(150, 601)), NT4) for _ in range(nq)]
    n = max(1, int(round(200_000 * scale)))
    records = []
    for _ in range(n):
        if rng.random() < 0.05:
            src = queries[int(rng.integers(0, nq))]
            records.append(mutate(rng, src, NT4, 0.10, 0.02, (1, 5)))
        else:
            records.append(random_residues(rng, int(rng.integers(100, 1501)), NT4))
    flat, offsets = _pack(records)
    return Workload("nw_nucleotide", "nw", 16, 20, 1, 0, "const:2,-3", (-5, -2), [q.tobytes() for q in queries],
                    flat, offsets, {"seed": seed, "scale": scale})


def sw_batched(seed: int = 3, scale: float = 1.0, n_queries: int = 1024, n_db: int = 500_000) -> Workload:
    rng = np.random.default_rng(seed)
    nq = max(1, int(round(n_queries * scale))) if scale < 1 else n_queries
    qlens = lognormal_lengths(rng, nq, 300.0, 0.7)
    queries = [random_residues(rng, int(L), AA20) for L in qlens]
    n = max(1, int(round(n_db * scale)))
    lens = gamma_lengths(rng, n, 350.0, 20, 35000)
    is_copy = rng.random(n) < 0.01
    flat_parts = []
    records_lens = np.zeros(n, dtype=np.int64)
    bulk = random_residues(rng, int(lens[~is_copy].sum()), AA20)
    pos = 0
    copy_src = {}                  # record -> index of the query it copies
    for i in range(n):
        if is_copy[i]:
            copy_src[i] = int(rng.integers(0, nq))
            src = queries[copy_src[i]]
            target = int(rng.integers(8000, 35001))
            tiled = np.tile(src, target // len(src) + 1)[:target]
            rec = mutate(rng, tiled, AA20, 0.02, 0.0, (1, 1))
        else:
            rec = bulk[pos:pos + lens[i]]
            pos += int(lens[i])
        flat_parts.append(rec)
        records_lens[i] = len(rec)
    flat, offsets = _pack(flat_parts)
    return Workload("sw_batched", "sw", 8, 10, 1, 1, "builtin:blosum62", (-11, -1), [q.tobytes() for q in queries],
                    flat, offsets, {"seed": seed, "scale": scale, "long_copies": int(is_copy.sum()), "copy_src": copy_src})


def sw_served_db(seed: int = 4, scale: float = 1.0) -> Workload:
    rng = np.random.default_rng(seed)
    n = max(1, int(round(1_000_000 * scale)))
    lens = gamma_lengths(rng, n)
    flat = random_residues(rng, int(lens.sum()), AA20)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    return Workload("sw_served", "sw", 8, 10, 1, 1, "builtin:blosum62", (-11, -1), [], flat, offsets,
                    {"seed": seed, "scale": scale})


def served_queries(seed: int, n: int) -> list[bytes]:
    rng = np.random.default_rng(seed)
    lens = lognormal_lengths(rng, n, 300.0, 0.8)
    return [random_residues(rng, int(L), AA20).tobytes() for L in lens]


def poisson_arrivals(seed: int, rate: float, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def long_pairs(seed: int = 5, n_pairs: int = 4096, lo: int = 5000, hi: int = 30000) -> list[tuple[bytes, bytes]]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_pairs):
        a = random_residues(rng, int(rng.integers(lo, hi + 1)), AA20)
        ident = rng.uniform(0.85, 0.99)
        b = mutate(rng, a, AA20, 1.0 - ident, 0.01, (1, 20))
        out.append((a.tobytes(), b.tobytes()))
    return out


CONFIGS = {
    "sw_plain": sw_plain,
    "nw_nucleotide": nw_nucleotide,
    "sw_batched": sw_batched,
    "sw_served": sw_served_db,
}
