"""The schedule of the stripe pipeline (libssa_b200/csrc/stripe_pipeline.cuh), modelled on the CPU.

A group of W warps shares one alignment: stripe i of query rows runs on warp
i % W, the group advances one chunk (32 wavefront steps) per group barrier, a
warp starts its next stripe when its previous one is done and the stripe above
started at least 2 steps earlier (4 when the stripe above is the last of a
super-pass of W stripes), and all running stripes cut at the group's column
limit published in the step before.  Lane 31 of a stripe writes the stripe's
bottom row at column c in step c + 31 (counted from the stripe's start, 32
steps per chunk); the stripe below reads it through a shared-memory ring of 256
columns (double-buffered by super-pass parity) or, across a super-pass, through
a global row that warp 0 reads 32 columns ahead.

This model replays that schedule step by step and checks, for every stripe and
column, that the value read was written in an earlier step and that neither the
ring slot nor the global row was overwritten before the read, for groups of 1,
2, 4 and 8 warps, fixed stripe lengths, lengths fixed at start from a limit that
shrinks, and cuts applied to running stripes.
"""
import pytest

RING = 256


def _chunk(step: int) -> int:
    return step // 32


def _schedule(W: int, n: int, B: int, start_len=None, cut=None):
    """Start step and length (chunks) of every stripe, as run_stripes runs them."""
    nc_full = (B + 31 + 31) // 32
    started = [(-1, 0)] * W          # per warp: (stripe, start step)
    nxt = list(range(W))
    active = [False] * W
    S, L = [0] * W, [0] * W
    starts, lens = {}, {}
    T = 0
    while True:
        snap = list(started)         # values written in earlier steps
        for w in range(W):
            if not active[w] and nxt[w] < n:
                i = nxt[w]
                ok = i == 0
                if not ok:
                    st = snap[(w - 1) % W]
                    lag = 4 if i % W == 0 else 2
                    ok = st[0] == i - 1 and st[1] <= T - lag
                if ok:
                    active[w], S[w] = True, T
                    L[w] = start_len(i, T) if start_len else nc_full
                    starts[i], lens[i] = T, L[w]
                    started[w] = (i, T)
        for w in range(W):
            if active[w]:
                c = T - S[w]
                if cut is not None:
                    L[w] = min(L[w], max(c + 1, cut(T)))
                    lens[nxt[w]] = L[w]
                if c + 1 >= L[w]:
                    active[w] = False
                    nxt[w] += W
        if all(not active[w] and nxt[w] >= n for w in range(W)):
            return starts, lens, T + 1
        T += 1
        assert T < n * (nc_full + 2 * W + 8) + 64, "the step bound of run_stripes would be reached"


def _check(W: int, n: int, B: int, start_len=None, cut=None):
    starts, lens, _ = _schedule(W, n, B, start_len, cut)
    cols = {i: min(B, lens[i] * 32 - 31) for i in lens}     # columns a stripe processes
    for q in range(1, n):
        p = q - 1
        for x in range(max(0, cols[q])):
            assert x < cols[p], f"stripe {q} needs column {x} beyond stripe {p}"
            write = starts[p] + _chunk(x + 31)
            if q % W == 0:   # global row, read 32 columns ahead
                read = starts[q] + (0 if x < 32 else _chunk(x) - 1)
            else:            # shared-memory ring, read at the column's step
                read = starts[q] + _chunk(x)
            assert write < read, f"W{W} n{n} B{B}: column {x} of stripe {q} read before it was written"
            if q % W == 0:
                nxt = p + W
                if nxt != q and nxt < n and x < cols[nxt]:
                    assert starts[nxt] + _chunk(x + 31) > read, "global row overwritten before it was read"
            else:
                if x + RING < cols[p]:
                    assert starts[p] + _chunk(x + RING + 31) > read, "ring slot overwritten by the same stripe"
                p2 = p + 2 * W
                if p2 < n:
                    for xx in range(x % RING, cols[p2], RING):
                        assert starts[p2] + _chunk(xx + 31) > read, "ring slot overwritten two super-passes later"


SIZES = [1, 2, 31, 32, 33, 64, 65, 257, 289, 600, 2100]


@pytest.mark.parametrize("W", [1, 2, 4, 8])
@pytest.mark.parametrize("n", [1, 2, 4, 5, 9, 17])
def test_fixed_lengths(W, n):
    for B in SIZES:
        _check(W, n, B)


@pytest.mark.parametrize("W", [1, 2, 4, 8])
@pytest.mark.parametrize("n", [2, 5, 9])
def test_lengths_from_a_shrinking_limit(W, n):
    for B in SIZES:
        def start_len(i, T, B=B):
            lim = max(0, B - 1 - 7 * T)
            return min((B + 62) // 32, (lim + 63) // 32)
        _check(W, n, B, start_len=start_len)


@pytest.mark.parametrize("W", [1, 2, 4, 8])
@pytest.mark.parametrize("drop", [0, 3, 11, 40])
def test_cuts_applied_to_running_stripes(W, drop):
    for n in (2, 5, 9):
        for B in SIZES:
            def cut(T, B=B, drop=drop):
                lim = B - 1 if T < drop else max(0, (B - 1) // 3)
                return (lim + 63) // 32
            _check(W, n, B, cut=cut)
