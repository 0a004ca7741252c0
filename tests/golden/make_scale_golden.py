"""Generates the full-size golden runs under tests/golden/ from the reference.

    python tests/golden/make_scale_golden.py [--jobs N] [--only NAME ...]

The fixtures of make_golden.py are small; these cover the workloads the
build is measured on at their full sizes, so that paths which only appear at
scale (sub-batches of the score buffer, every rows-per-thread class, the
16-bit cascade of the 8,000-35,000-residue near-copies, multi-warp traceback
groups, hundreds of chunks of schedule replay) meet the reference.

Needs ``oracle/_ref/ref_run`` (``make -C oracle ref REF=<reference tree>``).
Every query runs through the reference's ``sw_align``/``nw_align`` at 1 thread
(the only setting whose tie order is deterministic), AVX2 lanes, chunk size
1000, COMPUTE_ALIGNMENT; queries are spread over ``--jobs`` processes.  Each
fixture stores the workload generator's arguments and input digest, the
sampled query indices and, per query, the reference's hits (ID, score, CIGAR,
coordinates) and its 8->16 / 16->64 overflow counts.

Samples:

* ``scale_sw_batched.json``: 1,024 queries vs 500,000 sequences (seed 3):
  48 queries at evenly spaced length quantiles and the 16 queries owning the
  longest near-copies (those go through the 16-bit pass and the widest
  traceback groups);
* ``scale_nw_nucleotide.json``: all 64 queries vs 200,000 sequences (seed 2);
* ``scale_sw_served.json``: the 200-request served stream (query seed 40)
  vs 1,000,000 sequences (seed 4);
* ``scale_long_pairs.json``: 8 of the 4,096 long pairs (seed 5) at stratified
  sizes, each aligned by SW and NW against a database of its one partner.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from libssa_b200 import workloads as W  # noqa: E402

SERVED_SAMPLE = 200
SERVED_QUERY_SEED = 40
PAIR_SAMPLE = 8


def digest(queries: list[bytes], flat: np.ndarray, offsets: np.ndarray) -> str:
    h = hashlib.sha256()
    for q in queries:
        h.update(q + b"\0")
    h.update(np.ascontiguousarray(offsets, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(flat, dtype=np.uint8).tobytes())
    return h.hexdigest()


def hit_rows(res: dict) -> list[list]:
    return [[h["id"], h["score"], h["cigar"], h["q_start"], h["q_end"], h["d_start"], h["d_end"]]
            for h in res["hits"]]


def run_parallel(db: str, queries: dict[int, bytes], jobs: int, **kw) -> dict[int, dict]:
    """Reference runs of {index: query} at 1 thread, longest queries first,
    dealt round-robin to `jobs` processes."""
    order = sorted(queries, key=lambda i: -len(queries[i]))
    shards = [order[k::jobs] for k in range(jobs)]

    def one(shard):
        if not shard:
            return {}
        res = oracle.run_reference(db, [queries[i].decode() for i in shard], threads=1, simd=2, chunk=1000,
                                   **kw)
        return {i: {"ovf": [r["ovf8"], r["ovf16"]], "hits": hit_rows(r)} for i, r in zip(shard, res)}

    out: dict[int, dict] = {}
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for part in ex.map(one, shards):
            out.update(part)
    return out


def batched_sample(w: W.Workload) -> list[int]:
    lens = np.array([len(q) for q in w.queries])
    order = np.argsort(lens, kind="stable")
    pick = [int(order[int((i + 0.5) * len(order) / 48)]) for i in range(48)]
    copies = sorted(w.meta["copy_src"].items(), key=lambda kv: -int(w.db_offsets[kv[0] + 1] - w.db_offsets[kv[0]]))
    for _, q in copies:
        if len(pick) >= 64:
            break
        if q not in pick:
            pick.append(q)
    return pick


def write(name: str, payload: dict) -> None:
    path = os.path.join(HERE, f"scale_{name}.json")
    with open(path, "w") as f:
        json.dump(payload, f, separators=(",", ":"))
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)", flush=True)


def make_batched(jobs: int, td: str) -> None:
    w = W.sw_batched(seed=3)
    sample = batched_sample(w)
    db = os.path.join(td, "sw_batched.sdb")
    oracle.write_sdb(db, flat=w.db_flat, lengths=np.diff(w.db_offsets))
    res = run_parallel(db, {i: w.queries[i] for i in sample}, jobs, algo="sw", width=8, align=1, hits=10,
                       symtype=1, matrix="builtin:blosum62", gap=(-11, -1))
    write("sw_batched", {
        "workload": "sw_batched", "gen": {"seed": 3}, "digest": digest(w.queries, w.db_flat, w.db_offsets),
        "settings": {"algo": "sw", "width": 8, "hits": 10, "matrix": "builtin:blosum62", "gap": [-11, -1],
                     "chunk": 1000, "simd": 2, "symtype": 1},
        "sample": sample, "results": {str(i): res[i] for i in sample}})


def make_nw(jobs: int, td: str) -> None:
    w = W.nw_nucleotide(seed=2)
    sample = list(range(len(w.queries)))
    db = os.path.join(td, "nw_nucleotide.sdb")
    oracle.write_sdb(db, flat=w.db_flat, lengths=np.diff(w.db_offsets))
    res = run_parallel(db, {i: w.queries[i] for i in sample}, jobs, algo="nw", width=16, align=1, hits=20,
                       symtype=0, matrix="const:2,-3", gap=(-5, -2))
    write("nw_nucleotide", {
        "workload": "nw_nucleotide", "gen": {"seed": 2}, "digest": digest(w.queries, w.db_flat, w.db_offsets),
        "settings": {"algo": "nw", "width": 16, "hits": 20, "matrix": "const:2,-3", "gap": [-5, -2],
                     "chunk": 1000, "simd": 2, "symtype": 0},
        "sample": sample, "results": {str(i): res[i] for i in sample}})


def make_served(jobs: int, td: str) -> None:
    w = W.sw_served_db(seed=4)
    queries = W.served_queries(seed=SERVED_QUERY_SEED, n=SERVED_SAMPLE)
    sample = list(range(len(queries)))
    db = os.path.join(td, "sw_served.sdb")
    oracle.write_sdb(db, flat=w.db_flat, lengths=np.diff(w.db_offsets))
    res = run_parallel(db, {i: queries[i] for i in sample}, jobs, algo="sw", width=8, align=1, hits=10,
                       symtype=1, matrix="builtin:blosum62", gap=(-11, -1))
    write("sw_served", {
        "workload": "sw_served", "gen": {"seed": 4, "query_seed": SERVED_QUERY_SEED, "queries": SERVED_SAMPLE},
        "digest": digest(queries, w.db_flat, w.db_offsets),
        "settings": {"algo": "sw", "width": 8, "hits": 10, "matrix": "builtin:blosum62", "gap": [-11, -1],
                     "chunk": 1000, "simd": 2, "symtype": 1},
        "sample": sample, "results": {str(i): res[i] for i in sample}})


def pair_sample(pairs) -> list[int]:
    sizes = np.array([len(a) * len(b) for a, b in pairs])
    order = np.argsort(sizes, kind="stable")
    return [int(order[int((i + 0.5) * (len(order) - 1) / PAIR_SAMPLE)]) for i in range(PAIR_SAMPLE)]


def make_pairs(jobs: int, td: str) -> None:
    pairs = W.long_pairs(seed=5)
    sample = pair_sample(pairs)
    h = hashlib.sha256()
    for a, b in pairs:
        h.update(a + b"\0" + b + b"\0")

    def one(k):
        a, b = pairs[k]
        db = os.path.join(td, f"pair{k}.sdb")
        oracle.write_sdb(db, seqs=[b])
        out = {}
        for algo in ("sw", "nw"):
            r = oracle.run_reference(db, [a.decode()], algo=algo, width=16, align=1, hits=1, symtype=1,
                                     matrix="builtin:blosum62", gap=(-11, -1), chunk=1000, threads=1, simd=2)[0]
            out[algo] = hit_rows(r)
        return k, out

    res = {}
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for k, out in ex.map(one, sample):
            res[k] = out
    write("long_pairs", {
        "workload": "long_pairs", "gen": {"seed": 5, "n_pairs": len(pairs)}, "digest": h.hexdigest(),
        "settings": {"width": 16, "hits": 1, "matrix": "builtin:blosum62", "gap": [-11, -1], "chunk": 1000,
                     "simd": 2, "symtype": 1},
        "sample": sample, "results": {str(k): res[k] for k in sample}})


MAKERS = {"sw_batched": make_batched, "nw_nucleotide": make_nw, "sw_served": make_served, "long_pairs": make_pairs}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", nargs="*", choices=sorted(MAKERS), default=sorted(MAKERS))
    args = ap.parse_args()
    if not oracle.reference_available():
        sys.exit("oracle/_ref/ref_run is not built (make -C oracle ref REF=<reference tree>)")
    with tempfile.TemporaryDirectory() as td:
        for name in args.only:
            t0 = time.time()
            MAKERS[name](args.jobs, td)
            print(f"{name}: {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main()
