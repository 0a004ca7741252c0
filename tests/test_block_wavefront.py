"""The 4-column block wavefront of the query-pair entry kernels
(libssa_b200/csrc/sw_qpair_kernel.cu: sw_qpair4_kernel, nw_qpair4_kernel), modelled on the CPU.

A group of G threads computes one database sequence against the rows of one pass: thread k owns R consecutive
rows, and at step s it computes the 4-column block b = s - k.  Inside a block the four chains (chain j: column
4b + j) run skewed by one row, so iteration `it` holds cell (it - j, 4b + j) of every chain.  E is one value per
row shared by the chains (chain j reads what chain j - 1 wrote one iteration earlier), H per row holds the
block's last column (chain 3), the top row of a block comes from thread k - 1's last row of the step before
(a shuffle), and thread 0 takes the top row from the closed-form boundary (Needleman-Wunsch) or the bias (Smith-
Waterman) in the first pass, and from the row thread G - 1 left in the pass before in later passes.  The
Needleman-Wunsch kernel stages that row through a 3-slot shared-memory ring filled by cp.async two blocks ahead
(one commit group per block, `cp.async.wait_group 1` before a block's slot is read).

This model runs that dataflow step by step in exact integer arithmetic and checks, against the oracle's lane
(the reference's 8-bit Smith-Waterman and 16-bit / exact Needleman-Wunsch lanes) on random queries of one to
several passes and database sequences that end anywhere in their last block:

* Smith-Waterman: the running maximum (the score) where no cell reaches 255, else the first block in which one
  does (the kernel re-queues the pair with that block + 1 as the lane's spent blocks);
* Needleman-Wunsch: H at the query's last row in the sequence's last column;
* the ring: every block's slot holds that block's boundary row when it is read, and its copy group is complete.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from helpers import matrix_table
from libssa_b200 import workloads as W

G = 4            # threads per database sequence
C = 4            # columns per block (chains per thread)
AHEAD = 2        # ring: blocks copied ahead
SLOTS = AHEAD + 1


class Ring:
    """The boundary ring of one group's thread 0: slot contents and the cp.async commit groups in flight."""

    def __init__(self):
        self.slot = [None] * SLOTS      # (block, row) written by the copy of that block
        self.groups = []                # commit groups in order: the block copied, or None (empty group)
        self.complete = 0               # groups [0, complete) are known complete

    def copy(self, block, row):
        self.slot[block % SLOTS] = (block, row)

    def commit(self, block):
        self.groups.append(block)

    def wait(self, pending):
        """cp.async.wait_group pending: all but the newest `pending` groups complete."""
        self.complete = max(self.complete, len(self.groups) - pending)

    def read(self, block):
        # the group that copied this block is among the complete ones
        idx = self.groups.index(block)
        assert idx < self.complete, (block, idx, self.complete)
        held = self.slot[block % SLOTS]
        assert held is not None and held[0] == block, (block, held)
        return held[1]


def run_wavefront(algo, prof, L, passes, R, go, ge, q_last=None):
    """One database sequence of L columns through `passes` passes of G x R rows.

    prof[row][col]: the profile score at query row `row` (pad rows included) and database column `col` (pad
    columns of the last block included).  Returns (maximum, first block reaching 255) for Smith-Waterman, and
    H at (q_last, L - 1) for Needleman-Wunsch."""
    nw = algo == "nw"
    nb = (L + 3) // 4
    GR = G * R
    goe = go + ge
    left_h = lambda i: go + (i + 1) * ge            # H(i, -1)
    left_e = lambda i: 2 * go + (i + 2) * ge        # E entering column 0
    top_h = lambda j: 0 if j < 0 else go + (j + 1) * ge    # H(-1, j)
    top_f = lambda c: 2 * go + (c + 2) * ge         # F entering row 0
    scratch = {}                                    # block -> (out_h, out_f) of the previous pass
    best, cross, captured = 0, None, None
    for pas in range(passes):
        last_pass = pas + 1 == passes
        row0 = [pas * GR + k * R for k in range(G)]
        if nw:
            H = [[left_h(row0[k] + r) for r in range(R)] for k in range(G)]
            E = [[left_e(row0[k] + r) for r in range(R)] for k in range(G)]
            diag = [0 if row0[k] == 0 else left_h(row0[k] - 1) for k in range(G)]
        else:
            H = [[0] * R for _ in range(G)]
            E = [[0] * R for _ in range(G)]
            diag = [0] * G
        out_h = [[0] * C for _ in range(G)]
        out_f = [[0] * C for _ in range(G)]
        ring = Ring()
        if pas > 0:
            for x in range(AHEAD):
                if x < nb:
                    ring.copy(x, scratch[x])
                ring.commit(x if x < nb else None)
        for s in range(nb + G - 1):
            prev_h = [row[:] for row in out_h]      # the shuffle reads the step before
            prev_f = [row[:] for row in out_f]
            for k in range(G):
                b = s - k
                if b < 0 or b >= nb:
                    continue
                if k > 0:
                    up_h, up_f = prev_h[k - 1][:], prev_f[k - 1][:]
                elif pas > 0:
                    ring.wait(AHEAD - 1)
                    up_h, up_f = (list(v) for v in ring.read(b))
                    nxt = b + AHEAD
                    if nxt < nb:
                        ring.copy(nxt, scratch[nxt])
                    ring.commit(nxt if nxt < nb else None)
                elif nw:
                    up_h = [top_h(4 * b + j) for j in range(C)]
                    up_f = [top_f(4 * b + j) for j in range(C)]
                else:
                    up_h, up_f = [0] * C, [0] * C
                f = up_f[:]
                hv = [[None] * R for _ in range(C)]
                Hk, Ek = H[k], E[k]
                for it in range(R + C - 1):
                    for j in range(C):
                        r = it - j
                        if r < 0 or r >= R:
                            continue
                        v = prof[row0[k] + r][4 * b + j]
                        if r == 0:
                            hd = diag[k] if j == 0 else up_h[j - 1]
                        else:
                            hd = Hk[r - 1] if j == 0 else hv[j - 1][r - 1]
                        t = max(Ek[r], f[j]) if nw else max(Ek[r], f[j], 0)
                        h = max(hd + v, t)
                        hg = h + goe
                        f[j] = max(f[j] + ge, hg)
                        Ek[r] = max(Ek[r] + ge, hg)
                        hv[j][r] = h
                        if j == C - 1:
                            Hk[r] = h
                        if nw:
                            if row0[k] + r == q_last and 4 * b + j == L - 1:
                                captured = h
                        else:
                            # a thread's running maximum per pass, checked after every block: the
                            # first block in which it reaches 255, the minimum over threads and passes
                            best = max(best, h)
                            if h >= 255 and (cross is None or b < cross):
                                cross = b
                diag[k] = up_h[C - 1]
                out_h[k] = [hv[j][R - 1] for j in range(C)]
                out_f[k] = f[:]
                if k == G - 1 and not last_pass:
                    scratch[b] = (out_h[k][:], out_f[k][:])
    return captured if nw else (best, cross)


def _profile(algo, matrix, q, d, rows, nb):
    """The profile words the kernels read, as integers: the entry width's truncation of the score of database
    code d[col] against query code q[row]; rows past the query score -128 (Smith-Waterman 8-bit: never raises a
    maximum) or 0 (Needleman-Wunsch: rows below the query do not feed back into it); columns past the sequence,
    up to its last block's end, hold the record's pad code 0."""
    pad_row = -128 if algo == "sw" else 0
    dtype = np.int8 if algo == "sw" else np.int16
    table = np.asarray(matrix, dtype=np.int64).astype(dtype).astype(np.int64)
    cols = np.zeros(4 * nb, dtype=np.int64)
    cols[:len(d)] = d
    P = np.full((rows, 4 * nb), pad_row, dtype=np.int64)
    for i, qc in enumerate(q):
        P[i, :] = table[(cols << 5) + int(qc)]
    return P.tolist()


def _codes(rng, n, alpha, nucleotide):
    return oracle.map_codes(W.random_residues(rng, n, alpha).tobytes().decode(), nucleotide, True)


def _sw_case(seed):
    rng = np.random.default_rng(7100 + seed)
    q = _codes(rng, int(rng.integers(1, 70)), W.AA20, False)
    r = rng.random()
    if r < 0.35:
        # a near-copy of the query, long enough to reach 255 in some cases
        reps = int(rng.integers(1, 3))
        d = np.tile(q, reps)[:int(rng.integers(1, 2 * len(q) * reps + 2))].copy()
        flip = rng.random(len(d)) < 0.05
        d[flip] = _codes(rng, int(flip.sum()), W.AA20, False) if flip.any() else d[flip]
    else:
        d = _codes(rng, int(rng.integers(1, 45)), W.AA20, False)
    gap = [(-11, -1), (-5, -2), (-2, -3), (-3, -1)][int(rng.integers(0, 4))]
    return q, d, gap


@pytest.mark.parametrize("R", [1, 2, 4])
@pytest.mark.parametrize("seed", range(14))
def test_smith_waterman_block_wavefront(R, seed):
    q, d, (go, ge) = _sw_case(seed)
    matrix = matrix_table(("builtin", "blosum62"))
    passes = max(1, -(-len(q) // (G * R)))
    nb = (len(d) + 3) // 4
    prof = _profile("sw", matrix, q, d, passes * G * R, nb)
    # the 8-bit lane adds the int8 truncation of gapO + gapE
    goe8 = int(np.int8(go + ge))
    best, cross = run_wavefront("sw", prof, len(d), passes, R, goe8 - ge, ge)
    cfg = oracle.SearchConfig(algo="sw", bit_width=8, gap_open=go, gap_extend=ge, matrix=matrix)
    score, overflow, blocks = oracle.lane_result(cfg, 8, q, d)
    if cross is None:
        assert not overflow and best == score, (seed, R, best, score, overflow)
    else:
        assert overflow and blocks == cross + 1, (seed, R, cross, blocks, overflow)


def _nw_case(seed):
    rng = np.random.default_rng(7300 + seed)
    nuc = seed % 2 == 0
    alpha = W.NT4 if nuc else W.AA20
    q = _codes(rng, int(rng.integers(1, 70)), alpha, nuc)
    d = _codes(rng, int(rng.integers(1, 45)), alpha, nuc)
    matrix = matrix_table(("const", 2, -3) if nuc else ("builtin", "blosum62"))
    gap = [(-5, -2), (-11, -1), (-2, -3), (-40, -4)][int(rng.integers(0, 4))]
    return q, d, matrix, gap, nuc


@pytest.mark.parametrize("R", [1, 2, 4])
@pytest.mark.parametrize("seed", range(14))
def test_needleman_wunsch_block_wavefront(R, seed):
    q, d, matrix, (go, ge), nuc = _nw_case(seed)
    passes = max(1, -(-len(q) // (G * R)))
    nb = (len(d) + 3) // 4
    prof = _profile("nw", matrix, q, d, passes * G * R, nb)
    got = run_wavefront("nw", prof, len(d), passes, R, go, ge, q_last=len(q) - 1)
    cfg = oracle.SearchConfig(algo="nw", bit_width=16, gap_open=go, gap_extend=ge, matrix=matrix)
    assert got == oracle.full_score(cfg, q, d), (seed, R, len(q), len(d))


def test_ring_slot_reuse_is_caught():
    """The ring's checks fire when a slot is overwritten before it is read (a planted mistake in the model's
    accounting, not in the kernel): a copy three blocks ahead lands in the slot of the block being read next."""
    ring = Ring()
    ring.copy(0, "row0")
    ring.commit(0)
    ring.copy(3, "row3")            # slot 0 again: block 0's row is gone
    ring.commit(3)
    ring.wait(0)
    with pytest.raises(AssertionError):
        ring.read(0)
