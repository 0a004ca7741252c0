"""Measures the entry-pass shape table of the current GPU.

    python -m libssa_b200.tune [--out libssa_b200/tuning/b200.tune] [--reps 3]

The reference searches with one fixed tile: 4-column blocks and 32 or 16
lanes per vector (src/algo/8/search_8_util.h:25-27, src/algo/8/search_8.c:
41-56).  The B200 entry kernels have free shape parameters instead, and this
script times every candidate, per database bucket, on seeded synthetic data:

* the query-pair Smith-Waterman kernel (batches): rows per thread
  R in {16, 20, 24, 28} x resident CTAs per SM in {4, 5} x columns per step
  in {2, 4} (column-strip width: two or four dependency chains per thread),
  the 4-column kernel with its running maximum in fp16x2, and (R = 24) the
  4-column kernel with 8 threads of 12 rows per sequence, on 64 queries of
  exactly two passes (2 x 4R rows); cost = entry-pass device time per
  (query pair x pass x database column);
* the single-query kernels (sw_align): with one column per step, threads
  per sequence pair G in {8, 16, 32} x rows per thread R in {8, 16, 24, 32};
  with one 4-column block per step, G in {4, 8, 16, 32} x R in {8, 16, 24};
  G x R <= 512, on one query of two passes (2 x G x R rows); cost =
  entry-pass device time per (pass x database column).

Database buckets (the engine's db_bucket): mean sequence length below 250,
below 1,000 or longer, times fewer or more than 50,000 sequences; each gets a
gamma(2)-length database of that kind.  The engine picks, per query, the shape
with the smallest passes x cost of the searched database's bucket.  Costs are
written in picoseconds, one line per (kernel, bucket, shape); the file is
committed, and the library reads it from libssa_b200/tuning/b200.tune next to
its build (or from $SSA_B200_TUNING).
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tuning", "b200.tune")

# (mean length, clip low, clip high) per length bucket; sequence counts per size bucket
LENGTHS = [(150.0, 20, 600), (350.0, 20, 5000), (1500.0, 100, 20000)]
COUNTS = [10_000, 200_000]
QPAIR_R = (16, 20, 24, 28)
# (resident CTAs per SM, columns per step, running maximum in fp16x2, 8 threads per sequence)
QPAIR_VARIANTS = ((4, 2, 0, 0), (5, 2, 0, 0), (4, 4, 0, 0), (5, 4, 0, 0), (4, 4, 1, 0), (4, 4, 0, 1), (5, 4, 0, 1))
FAST_G = (8, 16, 32)
FAST_R = (8, 16, 24, 32)
FAST4_G = (4, 8, 16, 32)
FAST4_R = (8, 16, 24)
KINDS = ("qpair", "fast")


def bucket_db(length_b: int, size_b: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    mean, lo, hi = LENGTHS[length_b]
    rng = np.random.default_rng(seed)
    n = COUNTS[size_b]
    lens = W.gamma_lengths(rng, n, mean, lo, hi)
    flat = W.random_residues(rng, int(lens.sum()), W.AA20)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    return flat, offsets


def _setup(L):
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)
    L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
    L.init_gap_penalties(-11, -1)
    L.set_chunk_size(1000)
    L.set_simd_compute_mode(L.COMPUTE_ON_AVX2)


def _entry_seconds(L, fn, reps: int) -> float:
    fn()                                   # warm-up (and buffer growth)
    best = float("inf")
    for _ in range(reps):
        fn()
        best = min(best, L.stats().entry_seconds)
    return best


def _fast_candidates():
    for G in FAST_G:
        for R in FAST_R:
            if G * R <= 512:
                yield "fast", G, R, 1
    for G in FAST4_G:
        for R in FAST4_R:
            if G * R <= 512:
                yield "fast4", G, R, 4


def tune(reps: int = 3, log=print, kinds=KINDS) -> list[str]:
    """Times the candidates of the kernels in `kinds` ("qpair": the batched
    query-pair kernel; "fast": the single-query kernels) on every bucket."""
    import libssa_b200 as L
    L.load()
    _setup(L)
    rng = np.random.default_rng(77)
    lines = []
    for size_b in range(len(COUNTS)):
        for length_b in range(len(LENGTHS)):
            bucket = length_b + 3 * size_b
            flat, offsets = bucket_db(length_b, size_b, 1000 + bucket)
            L.load_db_memory(flat=flat, offsets=offsets)
            cols = int(np.sum((np.diff(offsets).astype(np.int64) + 3) // 4 * 4))
            t0 = time.time()
            # query-pair kernel: 32 pairs of queries of exactly two passes
            for R in (QPAIR_R if "qpair" in kinds else ()):
                rows = 2 * 4 * R
                qs = [L.init_sequence_fasta(L.READ_FROM_STRING,
                                            W.random_residues(rng, rows, W.AA20).tobytes().decode())
                      for _ in range(64)]
                for mb, c, hm, g8 in QPAIR_VARIANTS:
                    if g8 and R != 24:
                        continue
                    os.environ["SSA_B200_QP_R"] = str(R)
                    os.environ["SSA_B200_QP_MB"] = str(mb)
                    os.environ["SSA_B200_QP_C"] = str(c)
                    os.environ["SSA_B200_QP_HMAX"] = str(hm)
                    os.environ["SSA_B200_QP_G8"] = str(g8)
                    try:
                        t = _entry_seconds(L, lambda: L.align_batch(L.SSA_SMITH_WATERMAN, qs, 10,
                                                                    L.BIT_WIDTH_8, L.COMPUTE_SCORE), reps)
                    finally:
                        for v in ("SSA_B200_QP_R", "SSA_B200_QP_MB", "SSA_B200_QP_C", "SSA_B200_QP_HMAX",
                                  "SSA_B200_QP_G8"):
                            del os.environ[v]
                    ps = t / (32 * 2 * cols) * 1e12
                    kind = "qpair4g8" if g8 else "qpair4h" if hm else "qpair4" if c == 4 else "qpair"
                    lines.append(f"{kind} {bucket} {R} {mb} {ps:.4f}")
                for q in qs:
                    L.free_sequence(q)
            # single-query kernels: one query of exactly two passes
            for kind, G, R, C in (_fast_candidates() if "fast" in kinds else ()):
                q = L.init_sequence_fasta(L.READ_FROM_STRING,
                                          W.random_residues(rng, 2 * G * R, W.AA20).tobytes().decode())
                os.environ["SSA_B200_FAST_SHAPE"] = f"{G},{R},{C}"
                try:
                    t = _entry_seconds(L, lambda: L.sw_align(q, 10, L.BIT_WIDTH_8, L.COMPUTE_SCORE), reps)
                finally:
                    del os.environ["SSA_B200_FAST_SHAPE"]
                L.free_sequence(q)
                ps = t / (2 * cols) * 1e12
                lines.append(f"{kind} {bucket} {G} {R} {ps:.4f}")
            log(f"bucket {bucket}: {COUNTS[size_b]} sequences, mean length {LENGTHS[length_b][0]:.0f}, "
                f"{time.time() - t0:.1f} s")
    return lines


def device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except Exception:  # noqa: BLE001
        pass
    return "unknown"


def write(lines: list[str], path: str, version: int) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        f.write("# libssa B200 entry-pass shape table, written by python -m libssa_b200.tune\n")
        f.write("# qpair <bucket> <R> <CTAs per SM> <ps per query pair, pass and database column>\n")
        f.write("# qpair4 <bucket> <R> <CTAs per SM> <ps ...>  (4 columns per step)\n")
        f.write("# qpair4h <bucket> <R> <CTAs per SM> <ps ...>  (4 columns, running maximum in fp16x2)\n")
        f.write("# qpair4g8 <bucket> 24 <CTAs per SM> <ps ...>  (4 columns, 8 threads of 12 rows per sequence)\n")
        f.write("# fast <bucket> <G> <R> <ps per pass and database column>\n")
        f.write("# fast4 <bucket> <G> <R> <ps ...>  (4 columns per step)\n")
        f.write("# bucket = length bucket (mean <250, <1000, longer) + 3 x size bucket (<50,000 sequences, more)\n")
        f.write(f"version {version}\n")
        f.write(f"device {device_name()}\n")
        for ln in lines:
            f.write(ln + "\n")


def kept_entries(path: str, kinds) -> list[str]:
    """The entries of an existing table that a run measuring only `kinds`
    keeps: every cost line of the other kernels ("qpair*" lines belong to
    "qpair", "fast*" lines to "fast")."""
    if not os.path.exists(path):
        return []
    kept = []
    with open(path) as f:
        for ln in f:
            ln = ln.split("#", 1)[0].strip()
            if not ln or ln.split()[0] in ("version", "device"):
                continue
            if not ln.split()[0].startswith(tuple(kinds)):
                kept.append(ln)
    return kept


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--version", type=int, default=int(time.strftime("%Y%m%d")))
    ap.add_argument("--kernels", default="all", choices=["all", *KINDS],
                    help="measure only these kernels and keep the other entries of the existing table")
    args = ap.parse_args()
    kinds = KINDS if args.kernels == "all" else (args.kernels,)
    kept = kept_entries(args.out, kinds) if args.kernels != "all" else []
    os.environ["SSA_B200_TUNING"] = "builtin"     # measure with nothing pinned by an older table
    lines = kept + tune(args.reps, kinds=kinds)
    write(lines, args.out, args.version)
    print(f"wrote {args.out} ({len(lines)} entries)")


if __name__ == "__main__":
    main()
