"""Benchmark of the libssa B200 build on the batched Smith-Waterman workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--scale S]

Workload (``sw_batched``, synthetic, seeded): 1,024 protein queries with
lognormal(median 300, sigma 0.7) lengths clipped to [30, 5000] against a
500,000-sequence database (gamma(2, mean 350) lengths clipped to [20, 35000],
1% near-identical 8,000-35,000 residue copies of a query); BLOSUM62, gaps
11/1, 8-bit cascade entry, top 10 hits with CIGAR.  One step is one batched
search of all 1,024 queries through ``ssa_align_batch`` (COMPUTE_ALIGNMENT).

Metric: GCUPS = sum over queries of query length x database residues / time.
* ``value``: device time of the search kernels (entry pass, overflow passes,
  traceback; CUDA events on the library's streams), database resident in HBM;
* ``e2e``: wall time of the public C-ABI call with host buffers (query upload,
  result download, host schedule/heap replay and list building included);
* ``parity``: the last timed step's lists of a 64-query sample (IDs, scores,
  order, CIGARs, coordinates, overflow counters) against the reference's own
  answers at 1 thread (tests/golden/scale_sw_batched.json);
* ``roofline``: the entry-pass kernel against the measured integer ALU-pipe
  ceiling of the same device (fused 16x2 add-max: an add and a max per 16-bit
  half), 9 integer operations per cell;
* ``cpu_baseline``: the reference libssa (built from its sources into
  oracle/_ref) on the host cores, all threads on a 16-query length-stratified
  sample and 1 thread on 4 of them, against the full database;
* ``plain_gpu``: the same queries one ``sw_align`` call each (16-query sample);
* ``config1`` / ``config2`` / ``config5``: 1 x 375 vs 10,000 sequences
  (sw_align), 64 nucleotide queries vs 200,000 (NW, batched), 4,096 long
  pairs (SW and NW with CIGARs), each with its parity check;
* ``served``: the 200-request stream of the served workload at Poisson rates
  50-2,000/s into the request loop (``ssa_server_*``) over a resident
  1,000,000-sequence database: GCUPS, p50/p99 latency, admission counts and
  parity against the reference per rate.  ``--workload sw_served`` prints
  that leg alone as its own line.

With N > 1 (torchrun) every rank searches its own seeded 1,024-query batch
against the full database (weak scaling, no collective on the data path);
``value`` is all ranks' cells over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GCUPS (batched SW search, 1,024 queries vs 500k sequences, top 10 with CIGAR)"
ALGO_OPS_PER_CELL = 9          # 4 saturating adds + 5 maxes of the reference's ALIGNCORE


# --------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------
class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def _reduce(pg, x: float, op) -> float:
    if pg is None:
        return x
    import torch
    device = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(pg, x: float) -> float:
    """Max over ranks (the job's time is the slowest rank's)."""
    return _reduce(pg, x, pg.ReduceOp.MAX) if pg is not None else x


def reduce_sum(pg, x: float) -> float:
    """Sum over ranks (all ranks' cells)."""
    return _reduce(pg, x, pg.ReduceOp.SUM) if pg is not None else x


def job_throughput(pg, cells_per_step: float, steps: int, seconds: float) -> float:
    """GCUPS of the whole job: every rank's cells over the slowest rank's time."""
    return reduce_sum(pg, float(cells_per_step)) * steps / reduce_max(pg, seconds) / 1e9


def barrier(pg):
    if pg is not None:
        pg.barrier()


def make_workload(scale: float, query_seed: int, kind: str = "sw_batched", n_queries: int | None = None):
    from libssa_b200 import workloads as W
    if kind == "sw_plain":
        # a 10,000-sequence database and n_queries queries of 375
        import numpy as np
        w = W.sw_plain(seed=1, scale=scale)
        rng = np.random.default_rng(2000 + query_seed)
        w.queries = [W.random_residues(rng, 375, W.AA20).tobytes() for _ in range(n_queries or 1)]
        return w
    w = W.sw_batched(seed=3, scale=scale)
    if query_seed != 3:
        # a rank's own query batch of the same length distribution
        import numpy as np
        rng = np.random.default_rng(1000 + query_seed)
        lens = W.lognormal_lengths(rng, len(w.queries), 300.0, 0.7)
        w.queries = [W.random_residues(rng, int(L), W.AA20).tobytes() for L in lens]
    if n_queries:
        # a length-stratified subset of the batch (small profiling cases)
        w.queries = [w.queries[i] for i in sorted(stratified([len(q) for q in w.queries], n_queries))]
    return w


def rank_workload(args, rank: int):
    """A rank's shard of the job: its own seeded query batch (rank 0 the
    canonical one) against the full database, which every rank holds."""
    return make_workload(args.scale, 3 if rank == 0 else 3 + rank, args.workload, args.queries)


def load_traffic() -> float | None:
    """DRAM bytes per cell of the entry pass, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "sw_qpair4_kernel_32q.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_cell:"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


# --------------------------------------------------------------------------
# parity of timed outputs against the reference's golden runs
# --------------------------------------------------------------------------
GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name: str) -> dict | None:
    try:
        with open(os.path.join(GOLDEN, f"scale_{name}.json")) as f:
            return json.load(f)
    except OSError:
        return None


def hit_rows(hits) -> list[list]:
    return [[h.id, h.score, h.cigar, h.q_start, h.q_end, h.d_start, h.d_end] for h in hits]


def parity(name: str, lists: dict, overflows: dict | None = None) -> dict:
    """Compares {query index: hit list} (and {index: (ovf8, ovf16)}) with the
    reference's answers stored in tests/golden/scale_<name>.json."""
    g = golden(name)
    if g is None:
        return {"sample": 0, "mismatches": None, "source": f"tests/golden/scale_{name}.json missing"}
    bad = []
    for i in g["sample"]:
        exp = g["results"][str(i)]
        if i not in lists or hit_rows(lists[i]) != exp["hits"]:
            bad.append(i)
        elif overflows is not None and list(overflows[i]) != exp["ovf"]:
            bad.append(i)
    return {"sample": len(g["sample"]), "mismatches": len(bad), "mismatched": bad[:8],
            "checked": "IDs, scores, order, CIGARs, coordinates" + (", overflow counters" if overflows else ""),
            "source": f"tests/golden/scale_{name}.json (the reference's sw_align/nw_align, 1 thread, AVX2)"}


# --------------------------------------------------------------------------
# CPU baseline: the reference built from its sources (oracle/_ref/ref_run)
# --------------------------------------------------------------------------
def stratified(lengths, n: int) -> list[int]:
    """n indices at evenly spaced length quantiles."""
    import numpy as np
    order = np.argsort(np.asarray(lengths), kind="stable")
    return [int(order[int((i + 0.5) * len(order) / n)]) for i in range(n)]


def reference_run(w, pick: list[int], threads: int, db_path: str | None = None) -> tuple[int, float]:
    """(cells, seconds of the align calls) of the reference on queries `pick`
    against the full database of workload w."""
    import oracle
    if not oracle.reference_available():
        raise RuntimeError("oracle/_ref/ref_run is not built")
    import numpy as np
    qs = [w.queries[i].decode() for i in pick]
    with tempfile.TemporaryDirectory() as td:
        db = db_path
        if db is None:
            db = os.path.join(td, "db.sdb")
            oracle.write_sdb(db, flat=w.db_flat, lengths=np.diff(w.db_offsets))
        res = oracle.run_reference(db, qs, algo="sw", width=8, align=1, hits=10, symtype=1,
                                   matrix="builtin:blosum62", gap=(-11, -1), chunk=1000, threads=threads, simd=2,
                                   timing=True)
    return sum(len(q) for q in qs) * int(w.db_offsets[-1]), sum(r["seconds"] for r in res)


REF_POOL = 16          # length-stratified queries the reference is timed on
REF_PER_STEP = 4       # of them per step of the reference arm, in rotation


def cpu_baselines(w) -> dict:
    """The reference on this host: all threads on the 16-query pool, 1 thread
    on 4 of its queries (every 4th length quantile)."""
    import oracle
    import numpy as np
    threads = os.cpu_count() or 1
    pool = stratified([len(q) for q in w.queries], REF_POOL)
    with tempfile.TemporaryDirectory() as td:
        db = os.path.join(td, "db.sdb")
        oracle.write_sdb(db, flat=w.db_flat, lengths=np.diff(w.db_offsets))
        cells, secs = reference_run(w, pool, threads, db)
        one = pool[1::4]
        cells1, secs1 = reference_run(w, one, 1, db)
    lens = sorted(len(w.queries[i]) for i in pool)
    return {"value": round(cells / secs / 1e9, 3), "unit": "GCUPS", "cores": threads, "kind": "reference",
            "sample": f"{REF_POOL} length-stratified queries (lengths {lens}) vs the full {w.n_db}-sequence database, "
                      f"sw_align COMPUTE_ALIGNMENT, 8-bit entry, AVX2, {threads} threads; cells / summed call time",
            "seconds": round(secs, 2),
            "one_thread": {"value": round(cells1 / secs1 / 1e9, 3), "unit": "GCUPS", "cores": 1,
                           "sample": f"{len(one)} of those queries (lengths "
                                     f"{sorted(len(w.queries[i]) for i in one)}), 1 thread",
                           "seconds": round(secs1, 2)}}


def pairs_reference_sample(pairs, n_pairs: int, threads: int) -> tuple[float, float, str]:
    """(GCUPS, seconds, description) of the reference on a sample of long pairs:
    per pair a database of the one partner sequence and sw_align + nw_align
    with COMPUTE_ALIGNMENT at the 16-bit entry, as a reference caller aligns a
    pair."""
    import oracle
    if not oracle.reference_available():
        raise RuntimeError("oracle/_ref/ref_run is not built")
    import numpy as np
    sizes = np.array([len(a) * len(b) for a, b in pairs])
    order = np.argsort(sizes)
    # pairs at the 10th, 30th, ... size percentiles up to the median
    pick = [int(order[int((0.1 + 0.2 * i) * (len(order) - 1))]) for i in range(n_pairs)]
    secs, cells = 0.0, 0
    with tempfile.TemporaryDirectory() as td:
        for k in pick:
            a, b = pairs[k]
            db = os.path.join(td, f"pair{k}.sdb")
            oracle.write_sdb(db, seqs=[b])
            for algo in ("sw", "nw"):
                res = oracle.run_reference(db, [a.decode()], algo=algo, width=16, align=1, hits=1, symtype=1,
                                           matrix="builtin:blosum62", gap=(-11, -1), chunk=1000, threads=threads,
                                           simd=2, timing=True)
                secs += sum(r["seconds"] for r in res)
                cells += len(a) * len(b)
    desc = (f"{n_pairs} pairs of the workload ({sorted(int(sizes[k]) for k in pick)} cells), each against a "
            f"database of its one partner, sw_align and nw_align COMPUTE_ALIGNMENT, 16-bit entry, AVX2, "
            f"{threads} threads")
    return cells / secs / 1e9, secs, desc


def run_reference_arm(args):
    """The reference's own CPU path on this host's cores: every step runs 4
    queries of a 16-query length-stratified pool (in rotation, so the timed
    steps cover the whole pool) against the full database; the value is all
    timed steps' cells over their summed align-call time."""
    import oracle
    import numpy as np
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return 0
    w = make_workload(args.scale, 3)
    threads = os.cpu_count() or 1
    pool = stratified([len(q) for q in w.queries], REF_POOL)
    cells_t, secs_t, step_s = 0, 0.0, []
    covered = set()
    with tempfile.TemporaryDirectory() as td:
        db = os.path.join(td, "db.sdb")
        oracle.write_sdb(db, flat=w.db_flat, lengths=np.diff(w.db_offsets))
        for i in range(args.warmup + args.steps):
            # every 4th quantile of the pool: each step spans the length range
            k0 = i % (REF_POOL // REF_PER_STEP)
            pick = pool[k0::REF_POOL // REF_PER_STEP]
            cells, secs = reference_run(w, pick, threads, db)
            if i >= args.warmup:
                cells_t += cells
                secs_t += secs
                step_s.append(secs)
                covered.update(pick)
    value = cells_t / secs_t / 1e9
    desc = (f"{len(covered)} of a {REF_POOL}-query length-stratified pool (lengths "
            f"{sorted(len(w.queries[i]) for i in pool)}), {REF_PER_STEP} per step (every 4th length quantile, "
            f"in rotation), vs the full "
            f"{w.n_db}-sequence database, sw_align COMPUTE_ALIGNMENT, 8-bit entry, AVX2, {threads} threads; "
            "cells over summed call time")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * statistics.median(step_s), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8/int16/int64", "data": "synthetic (seeded)",
        "config": {"workload": "sw_batched", "queries": len(w.queries), "db_sequences": w.n_db,
                   "db_residues": int(w.db_offsets[-1]), "scale": args.scale},
        "cpu_baseline": {"value": round(value, 3), "unit": "GCUPS", "cores": threads, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# the B200 arm
# --------------------------------------------------------------------------
def set_search(L, matrix: str = "blosum62", gap=(-11, -1), symtype=None):
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.AMINOACID if symtype is None else symtype, L.FORWARD_STRAND, 1, 1)
    if matrix.startswith("const:"):
        L.init_constant_scores(*map(int, matrix[6:].split(",")))
    else:
        L.init_score_matrix(L.MATRIX_BUILDIN, matrix)
    L.init_gap_penalties(*gap)
    L.set_chunk_size(1000)
    L.set_simd_compute_mode(L.COMPUTE_ON_AVX2)
    L.set_thread_count(1)


def run_ours(args):
    world, rank, local, pg = dist_setup()
    os.environ["SSA_B200_DEVICE"] = str(local)
    import libssa_b200 as L
    if not L.libraries_built():
        from libssa_b200 import build
        build.build()
    L.load()
    w = rank_workload(args, rank)
    set_search(L)
    L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)
    if args.db_memory:
        L.set_db_memory(args.db_memory)     # below the packed size: the database is streamed
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in w.queries]
    cells = sum(len(q) for q in w.queries) * int(w.db_offsets[-1])

    def step():
        return L.align_batch(L.SSA_SMITH_WATERMAN, qs, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT)

    for _ in range(args.warmup):
        step()
    peak_lane_ops, peak_ipc = L.int_peak()
    barrier(pg)
    launches0 = L.stats().kernel_launches_total
    sampler = ClockSampler(local)
    sampler.start()
    wall, dev, entry, h2d, d2h = [], [], [], [], []
    lists = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        lists = step()
        wall.append(time.perf_counter() - t0)
        st = L.stats()
        dev.append(st.kernel_seconds)
        entry.append(st.entry_seconds)
        h2d.append(st.h2d_bytes)
        d2h.append(st.d2h_bytes)
    clocks = sampler.stop()
    launches = L.stats().kernel_launches_total - launches0
    ovf = L.query_overflows()
    tuning = L.tuning_report()
    barrier(pg)
    t_wall = reduce_max(pg, sum(wall))
    t_dev = reduce_max(pg, sum(dev))
    total_cells = reduce_sum(pg, float(cells)) * args.steps
    value = total_cells / t_dev / 1e9
    e2e = total_cells / t_wall / 1e9

    if rank != 0:
        return 0
    # roofline of the entry pass: algorithmic lane operations per launch over
    # its device time
    t_entry = statistics.median(entry)
    achieved = cells * ALGO_OPS_PER_CELL / t_entry / 1e12
    peak = peak_lane_ops / 1e12
    traffic_per_cell = load_traffic()
    plain = args.workload == "sw_plain"
    metric = (f"GCUPS (plain SW search, {len(w.queries)} quer{'y' if len(w.queries) == 1 else 'ies'} of 375 vs "
              f"10,000 sequences, top 10 with CIGAR)" if plain else METRIC)
    line = {
        "metric": metric, "value": round(value, 2), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t_dev / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int16x2 (8-bit lane semantics), int32",
        "data": ("synthetic (seeded: queries of 375 vs 10,000 gamma-length sequences)" if plain else
                 "synthetic (seeded: 1,024 lognormal-length queries vs 500,000 gamma-length sequences)"),
        "config": {"workload": args.workload, "queries_per_gpu": len(w.queries), "db_sequences": w.n_db,
                   "db_residues": int(w.db_offsets[-1]), "cells_per_step_per_gpu": cells,
                   "matrix": "blosum62", "gap": [-11, -1], "bit_width": 8, "hits": 10,
                   "align_type": "COMPUTE_ALIGNMENT", "scale": args.scale,
                   "l2": "inputs larger than L2 (database codes %.2f GB)" % (int(w.db_offsets[-1]) / 1e9),
                   "parallelism": f"{world} x independent query batch vs full database",
                   "db_streamed": bool(L.db_streamed())},
        "e2e": {"value": round(e2e, 2), "unit": "GCUPS", "h2d_bytes_per_step": int(statistics.median(h2d)),
                "d2h_bytes_per_step": int(statistics.median(d2h))},
        "roofline": {"bound": "alu", "achieved": round(achieved, 3), "peak": round(peak, 3),
                     "unit": "Top/s", "frac": round(achieved / peak, 4),
                     "traffic": (round(traffic_per_cell * cells) if traffic_per_cell else None),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per cell of an entry-pass "
                                       "launch on a small case (32 queries vs 250,000 sequences), scaled by cells "
                                       "(profiles/sw_qpair4_kernel_32q.md)",
                     "kernel": ("sw_qpair4_kernel / sw_qpair_kernel (entry pass, all rows-per-thread classes)"
                                if len(w.queries) > 1 else "sw_fast_kernel (entry pass)"),
                     "peak_source": "measured on this device: integer ALU pipe running fused 16x2 add-max "
                                    f"({peak_ipc:.2f} warp-inst/clk/SM, an add and a max per 16-bit half); "
                                    "9 integer ops per cell (4 adds, 5 maxes); neither HBM nor tensor cores "
                                    "bound this integer max-plus recurrence"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "timing": {"device_seconds": round(t_dev, 4), "wall_seconds": round(t_wall, 4),
                   "entry_seconds_median": round(t_entry, 4)},
        "tuning": {"table": os.path.relpath(tuning["source"], ROOT) if os.path.isabs(tuning["source"])
                   else tuning["source"], "version": tuning["version"], "device": tuning["device"],
                   "shapes_last_call": tuning["last_call"]},
    }
    if not plain and args.scale == 1.0 and not args.queries and rank == 0 and lists is not None:
        line["parity"] = parity("sw_batched", dict(enumerate(lists)), dict(enumerate(ovf)))
    if args.plain_queries > 0:
        # the plain one-query-per-call path on a length-stratified query sample
        pick = stratified([len(q) for q in w.queries], args.plain_queries)
        sample = [qs[i] for i in pick]
        L.sw_align(sample[0], 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT)
        t_plain, d_plain = 0.0, 0.0
        for q in sample:
            t0 = time.perf_counter()
            L.sw_align(q, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT)
            t_plain += time.perf_counter() - t0
            d_plain += L.stats().kernel_seconds
        cells_plain = sum(len(w.queries[i]) for i in pick) * int(w.db_offsets[-1])
        plain_e2e = cells_plain / t_plain / 1e9
        line["plain_gpu"] = {"value": round(plain_e2e, 2), "unit": "GCUPS",
                             "device": round(cells_plain / d_plain / 1e9, 2),
                             "batched_over_plain": {"e2e": round(e2e / plain_e2e, 2),
                                                    "device": round(value / (cells_plain / d_plain / 1e9), 2)},
                             "sample": f"{args.plain_queries} length-stratified queries, one sw_align call each "
                                       "(COMPUTE_ALIGNMENT); value: wall time of the calls (like e2e), device: "
                                       "device time of their kernels (like value)"}
    for q in qs:
        L.free_sequence(q)
    if world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baselines(w)
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": "GCUPS", "cores": os.cpu_count() or 1,
                                    "kind": "reference", "sample": f"unavailable: {e}"}
    if world == 1 and not plain and args.scale == 1.0 and not args.queries and not args.no_legs:
        del w
        line["config1"] = config1_leg(L)
        line["config2"] = config2_leg(L)
        line["config5"] = config5_leg(L, args)
    if world == 1 and args.served_requests > 0:
        line["served"] = served_sweep(args, L)
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# --split db: the database-sharded layout (one record range per GPU)
# --------------------------------------------------------------------------
def record_ranges(lengths, parts: int, chunk: int = 1000) -> list[int]:
    """Bounds of `parts` contiguous record ranges holding about equal residues,
    cut at multiples of the reference's chunk of 1,000 records."""
    import numpy as np
    n = len(lengths)
    cum = np.concatenate([[0], np.cumsum(np.asarray(lengths, dtype=np.int64))])
    bounds = [0]
    for r in range(1, parts):
        target = cum[-1] * r / parts
        i = int(np.searchsorted(cum, target))
        i = min(n, max(bounds[-1], int(round(i / chunk)) * chunk))
        bounds.append(i)
    bounds.append(n)
    return bounds


def run_db_split(args):
    """Every rank loads the whole database through the plugin; rank r scores
    the queries against its contiguous record range on its GPU
    (ssa_b200_shard_scores), the per-record results (score, blocks of the
    overflowing entry-width and 16-bit lanes) go to rank 0 in one gather, and
    rank 0 replays the reference's lane schedule and heap and traces the hits
    back (ssa_b200_replay_gathered).  The same 1,024 queries on every rank:
    total work fixed as N grows (strong scaling)."""
    import numpy as np
    world, rank, local, pg = dist_setup()
    os.environ["SSA_B200_DEVICE"] = str(local)
    import libssa_b200 as L
    L.load()
    w = make_workload(args.scale, 3)
    set_search(L)
    L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in w.queries]
    lens = np.diff(w.db_offsets).astype(np.int64)
    bounds = record_ranges(lens, world)
    lo, hi = bounds[rank], bounds[rank + 1]
    cells_rank = sum(len(q) for q in w.queries) * int(lens[lo:hi].sum())
    cells = sum(len(q) for q in w.queries) * int(w.db_offsets[-1])

    def step():
        t0 = time.perf_counter()
        sc, be, b16 = L.shard_scores(L.SSA_SMITH_WATERMAN, qs, L.BIT_WIDTH_8, lo, hi)
        dev = L.stats().entry_seconds
        t1 = time.perf_counter()
        if pg is not None:
            import torch
            wmax = max(bounds[i + 1] - bounds[i] for i in range(world))
            parts = []
            for a in (sc, be.astype(np.int64), b16.astype(np.int64)):
                t = torch.full((len(qs), wmax), -1, dtype=torch.int64, device="cuda")
                t[:, :a.shape[1]] = torch.from_numpy(a).cuda()
                lst = [torch.empty_like(t) for _ in range(world)] if rank == 0 else None
                pg.gather(t, lst, dst=0)
                if rank == 0:
                    parts.append(np.concatenate([lst[i][:, :bounds[i + 1] - bounds[i]].cpu().numpy()
                                                 for i in range(world)], axis=1))
            if rank == 0:
                sc, be, b16 = parts[0], parts[1].astype(np.int32), parts[2].astype(np.int32)
        lists = None
        if rank == 0:
            lists = L.replay_gathered(L.SSA_SMITH_WATERMAN, qs, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT, sc, be, b16)
            dev += L.stats().kernel_seconds
        return lists, time.perf_counter() - t0, dev, t1 - t0

    for _ in range(args.warmup):
        step()
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    wall, dev, shard_wall = 0.0, 0.0, 0.0
    lists = None
    for _ in range(args.steps):
        barrier(pg)
        lists, t_wall, t_dev, t_shard = step()
        wall += t_wall
        dev += t_dev
        shard_wall += t_shard
    clocks = sampler.stop()
    barrier(pg)
    t_wall = reduce_max(pg, wall)
    t_dev = reduce_max(pg, dev)
    if rank == 0:
        line = {"metric": METRIC + ", database-sharded", "value": round(cells * args.steps / t_dev / 1e9, 2),
                "unit": "GCUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(1e3 * t_dev / args.steps, 3), "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "int16x2 (8-bit lane semantics), int32",
                "data": "synthetic (seeded: 1,024 lognormal-length queries vs 500,000 gamma-length sequences)",
                "config": {"workload": "sw_batched", "split": "database records", "ranges": bounds,
                           "cells_per_step": cells, "cells_rank0": cells_rank, "scale": args.scale},
                "e2e": {"value": round(cells * args.steps / t_wall / 1e9, 2), "unit": "GCUPS"},
                "clocks": clocks,
                "timing": "value: max over ranks of (shard entry + cascade device time, and on rank 0 the "
                          "traceback); e2e: wall time of the step incl. the gather and the host replay"}
        if args.scale == 1.0 and lists is not None:
            line["parity"] = parity("sw_batched", dict(enumerate(lists)), dict(enumerate(L.query_overflows())))
        print(json.dumps(line), flush=True)
    for q in qs:
        L.free_sequence(q)
    return 0


# --------------------------------------------------------------------------
# the other configurations, measured in the same run
# --------------------------------------------------------------------------
def config1_leg(L) -> dict:
    """1 query of 375 residues vs 10,000 sequences through sw_align (8-bit
    entry, top 10 with CIGAR): per-call wall and device time over 20 calls."""
    from libssa_b200 import workloads as W
    w = W.sw_plain(seed=1)
    set_search(L)
    L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)
    q = L.init_sequence_fasta(L.READ_FROM_STRING, w.queries[0].decode())
    for _ in range(3):
        hits = L.sw_align(q, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT)
    wall, dev, entry = [], [], []
    for _ in range(20):
        t0 = time.perf_counter()
        hits = L.sw_align(q, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT)
        wall.append(time.perf_counter() - t0)
        st = L.stats()
        dev.append(st.kernel_seconds)
        entry.append(st.entry_seconds)
    ovf = L.query_overflows()[0]
    L.free_sequence(q)
    cells = w.cells()
    # golden: the reference's answer on this exact input (tests/golden/cases.json, sw_plain_full)
    par = {"sample": 1, "mismatches": None}
    try:
        with open(os.path.join(GOLDEN, "cases.json")) as f:
            case = [c for c in json.load(f) if c["name"] == "sw_plain_full"][0]
        exp = case["expected"][0]
        ok = hit_rows(hits) == exp["hits"] and list(ovf) == [exp["ovf8"], exp["ovf16"]]
        par = {"sample": 1, "mismatches": 0 if ok else 1, "source": "tests/golden/cases.json sw_plain_full"}
    except (OSError, IndexError, KeyError):
        pass
    return {"metric": "GCUPS (plain SW, 1 query of 375 vs 10,000 sequences, top 10 with CIGAR)",
            "value": round(cells / statistics.median(dev) / 1e9, 2), "unit": "GCUPS",
            "e2e": round(cells / statistics.median(wall) / 1e9, 2),
            "ms_per_call": {"wall_median": round(1e3 * statistics.median(wall), 3),
                            "device_median": round(1e3 * statistics.median(dev), 3),
                            "entry_median": round(1e3 * statistics.median(entry), 3)},
            "calls": 20, "parity": par,
            "timing": "value: device time of the call's kernels (median of 20 calls); e2e: wall time of sw_align"}


def config2_leg(L) -> dict:
    """64 nucleotide queries vs 200,000 sequences, Needleman-Wunsch, 16-bit
    entry, constant scores 2/-3, gaps 5/2, top 20 with CIGAR, one batched call
    per step."""
    from libssa_b200 import workloads as W
    w = W.nw_nucleotide(seed=2)
    set_search(L, "const:2,-3", (-5, -2), symtype=L.NUCLEOTIDE)
    L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in w.queries]
    cells = w.cells()
    L.align_batch(L.SSA_NEEDLEMAN_WUNSCH, qs, 20, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
    dev, wall = 0.0, 0.0
    steps = 3
    for _ in range(steps):
        t0 = time.perf_counter()
        lists = L.align_batch(L.SSA_NEEDLEMAN_WUNSCH, qs, 20, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
        wall += time.perf_counter() - t0
        dev += L.stats().kernel_seconds
    ovf = L.query_overflows()
    for q in qs:
        L.free_sequence(q)
    return {"metric": "GCUPS (batched NW nucleotide search, 64 queries vs 200,000 sequences, top 20 with CIGAR)",
            "value": round(cells * steps / dev / 1e9, 2), "unit": "GCUPS",
            "e2e": round(cells * steps / wall / 1e9, 2), "steps": steps,
            "ms_per_step": round(1e3 * dev / steps, 2), "cells_per_step": cells,
            "parity": parity("nw_nucleotide", dict(enumerate(lists)), dict(enumerate(ovf)))}


def config5_leg(L, args) -> dict:
    """4,096 long pairs (5,000-30,000 residues, a query and its mutated copy),
    SW and NW with CIGARs through ssa_align_pairs, one timed step after one
    warm-up."""
    from libssa_b200 import workloads as W
    pairs = W.long_pairs(seed=5)
    set_search(L, gap=(-11, -1))
    L.load_db_memory([b for _, b in pairs])
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, a.decode()) for a, _ in pairs]
    ids = list(range(len(pairs)))
    cells = 2 * sum(len(a) * len(b) for a, b in pairs)
    algos = (L.SSA_SMITH_WATERMAN, L.SSA_NEEDLEMAN_WUNSCH)
    for algo in algos:
        L.align_pairs(algo, qs, ids, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
    dev, wall = 0.0, 0.0
    out = {}
    for algo in algos:
        t0 = time.perf_counter()
        out[algo] = L.align_pairs(algo, qs, ids, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
        wall += time.perf_counter() - t0
        dev += L.stats().gpu_seconds
    for q in qs:
        L.free_sequence(q)
    g = golden("long_pairs")
    par = {"sample": 0, "mismatches": None}
    if g is not None:
        bad = []
        for k in g["sample"]:
            for algo, name in ((algos[0], "sw"), (algos[1], "nw")):
                got = [[0] + r[1:] for r in hit_rows(out[algo][k])]   # the reference's one-sequence database: ID 0
                if got != g["results"][str(k)][name]:
                    bad.append((k, name))
        par = {"sample": len(g["sample"]), "mismatches": len(bad), "mismatched": bad[:8],
               "source": "tests/golden/scale_long_pairs.json (the reference, one-sequence databases, 1 thread)"}
    return {"metric": "GCUPS (4,096 long-pair SW and NW alignments with CIGAR, 5k-30k residues per side)",
            "value": round(cells / dev / 1e9, 2), "unit": "GCUPS", "e2e": round(cells / wall / 1e9, 2),
            "ms_per_step": round(1e3 * dev, 1), "cells_per_step": cells, "parity": par}


# --------------------------------------------------------------------------
# served: Poisson arrivals into the request loop (ssa_server_*)
# --------------------------------------------------------------------------
SERVED_RATES = (50, 100, 200, 500, 1000, 2000)


def served_once(L, texts, qs, residues, rate: float, seed: int, slots: int, segments: int) -> tuple[dict, list]:
    """One Poisson stream of the queries `qs` at `rate`/s into a fresh server."""
    import numpy as np
    from libssa_b200 import workloads as W
    arrivals = W.poisson_arrivals(seed=seed, rate=rate, n=len(qs))
    server = L.Server(L.SSA_SMITH_WATERMAN, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT, slots=slots, segments=segments)
    tickets = [None] * len(qs)
    t0 = time.perf_counter()

    def client():
        for i, q in enumerate(qs):
            delay = t0 + float(arrivals[i]) - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            tickets[i] = server.submit(q)

    th = threading.Thread(target=client)
    th.start()
    th.join()
    lat, results = [], []
    for t in tickets:
        hits, latency = server.wait(t)
        lat.append(latency)
        results.append(hits)
    wall = time.perf_counter() - t0
    st = server.stats()
    server.stop()
    cells = sum(len(t) for t in texts) * residues
    lat_ms = np.array(lat) * 1e3
    return ({"rate_qps": rate, "value": round(cells / wall / 1e9, 2), "unit": "GCUPS",
             "latency_ms": {"p50": round(float(np.percentile(lat_ms, 50)), 1),
                            "p99": round(float(np.percentile(lat_ms, 99)), 1),
                            "max": round(float(lat_ms.max()), 1)},
             "requests": len(qs), "queued": int(st.queued), "admitted_at_once": len(qs) - int(st.queued),
             "max_waiting": int(st.max_pending), "max_slots_used": int(st.max_occupied),
             "mean_slots_used": round(st.slot_waves / max(1, st.waves), 1), "waves": int(st.waves),
             "device_seconds": round(st.device_seconds, 3), "wall_seconds": round(wall, 3)}, results)


def served_sweep(args, L) -> dict:
    """A resident 1,000,000-sequence database; the 200-request stream of the
    served workload arrives as a Poisson process at each rate into a fresh
    server.  GCUPS over the wall time from the first arrival to the last
    result, submit-to-result latency, admission counts, and every result
    against the reference's answer for that request."""
    from libssa_b200 import workloads as W
    w = W.sw_served_db(seed=4, scale=args.served_scale)
    set_search(L)
    L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)
    g = golden("sw_served") if args.served_scale == 1.0 else None
    n = g["gen"]["queries"] if g else args.served_requests
    texts = [q.decode() for q in W.served_queries(seed=40, n=n)][:args.served_requests]
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, t) for t in texts]
    residues = int(w.db_offsets[-1])
    rates = [args.served_rate] if args.served_rate else list(SERVED_RATES)
    per_rate = []
    for k, rate in enumerate(rates):
        res, results = served_once(L, texts, qs, residues, rate, 41 + k, args.served_slots, args.served_segments)
        if g is not None:
            res["parity"] = parity("sw_served", {i: results[i] for i in range(len(results))})
        per_rate.append(res)
    for q in qs:
        L.free_sequence(q)
    return {"per_rate": per_rate, "unit": "GCUPS",
            "config": {"workload": "sw_served", "db_sequences": w.n_db, "db_residues": residues,
                       "requests_per_rate": len(qs), "slots": args.served_slots, "segments": args.served_segments,
                       "hits": 10, "align_type": "COMPUTE_ALIGNMENT",
                       "queries": "the served stream's first requests (query seed 40), lognormal(300, 0.8) lengths"},
            "timing": "wall time from the first arrival to the last completion; latency = submit to result"}


def run_nw_arm(args):
    import libssa_b200 as L
    L.load()
    leg = config2_leg(L)
    line = {"metric": leg["metric"], "value": leg["value"], "unit": "GCUPS", "n_gpus": 1, "steps": leg["steps"],
            "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int16 lanes (16-bit entry), int32",
            "data": "synthetic (seeded: 64 nucleotide queries of 150-600 vs 200,000 sequences of 100-1,500)",
            "config": {"workload": "nw_nucleotide", "cells_per_step": leg["cells_per_step"]},
            "e2e": {"value": leg["e2e"], "unit": "GCUPS"}, "parity": leg["parity"]}
    print(json.dumps(line), flush=True)
    return 0


def run_pairs_arm(args):
    """Long pairs, each a query of 5,000-30,000 residues and a mutated
    copy of it (85-99% identity, 1% indel events of length 1-20), BLOSUM62, gaps
    11/1, 16-bit entry.  One step aligns every pair with Smith-Waterman and with
    Needleman-Wunsch through ssa_align_pairs (query i against database sequence
    i alone); --pair-align score times the score-only calls."""
    import libssa_b200 as L
    from libssa_b200 import workloads as W
    L.load()
    pairs = W.long_pairs(seed=5, n_pairs=args.pairs, lo=args.pair_lo, hi=args.pair_hi)
    set_search(L)
    L.load_db_memory([b for _, b in pairs])
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, a.decode()) for a, _ in pairs]
    ids = list(range(len(pairs)))
    cells_one = sum(len(a) * len(b) for a, b in pairs)
    cells = 2 * cells_one
    align = L.COMPUTE_SCORE if args.pair_align == "score" else L.COMPUTE_ALIGNMENT
    algos = (L.SSA_SMITH_WATERMAN, L.SSA_NEEDLEMAN_WUNSCH)
    for _ in range(args.warmup):
        for algo in algos:
            L.align_pairs(algo, qs, ids, L.BIT_WIDTH_16, align)
    dev, wall = 0.0, 0.0
    per_algo = {0: 0.0, 1: 0.0}
    h2d = d2h = 0
    for _ in range(args.steps):
        for algo in algos:
            t0 = time.perf_counter()
            L.align_pairs(algo, qs, ids, L.BIT_WIDTH_16, align)
            wall += time.perf_counter() - t0
            st = L.stats()
            dev += st.gpu_seconds
            per_algo[algo] += st.gpu_seconds
            h2d += int(st.h2d_bytes)
            d2h += int(st.d2h_bytes)
    line = {"metric": "GCUPS (long-pair SW and NW alignments" + (" with CIGAR" if align else ", scores only") +
                      ", 5k-30k residues per side)",
            "value": round(cells * args.steps / dev / 1e9, 2), "unit": "GCUPS", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dev / args.steps * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded: query / mutated-copy pairs of 5,000-30,000 residues)",
            "config": {"workload": "long_pairs", "pairs": len(pairs), "query_lengths": [args.pair_lo, args.pair_hi],
                       "algorithms": ["sw", "nw"], "align": args.pair_align,
                       "cells_per_step": cells, "bit_width": 16,
                       "l2": "inputs and direction matrices far larger than L2"},
            "e2e": {"value": round(cells * args.steps / wall / 1e9, 2), "unit": "GCUPS",
                    "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps},
            "timing": {"device_seconds": round(dev, 4), "wall_seconds": round(wall, 4),
                       "sw_seconds": round(per_algo[0], 4), "nw_seconds": round(per_algo[1], 4)}}
    if not args.no_cpu_baseline and align:
        import multiprocessing
        threads = multiprocessing.cpu_count()
        try:
            g, secs, desc = pairs_reference_sample(pairs, 3, threads)
            line["cpu_baseline"] = {"value": round(g, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
                                    "sample": desc, "seconds": round(secs, 2)}
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"unavailable": str(e)}
    print(json.dumps(line), flush=True)
    for q in qs:
        L.free_sequence(q)
    return 0


def run_served_arm(args):
    import libssa_b200 as L
    L.load()
    res = served_sweep(args, L)
    best = max(res["per_rate"], key=lambda r: r["value"])
    line = {"metric": "GCUPS (served SW search, 1,000,000 resident sequences, Poisson arrivals, top 10 with CIGAR)",
            "value": best["value"], "unit": "GCUPS", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int16x2 (8-bit lane semantics), int32",
            "data": "synthetic (seeded: 1,000,000 resident sequences, Poisson arrivals)", **res}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--split", default="queries", choices=["queries", "db"],
                    help="with N GPUs: each rank its own query batch vs the whole database (queries), or the "
                         "same queries vs one record range per rank, gathered and replayed on rank 0 (db)")
    ap.add_argument("--scale", type=float, default=1.0, help="database and query count scale (1.0 = full)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-legs", action="store_true", help="skip the config-1, -2 and -5 legs")
    ap.add_argument("--plain-queries", type=int, default=16,
                    help="queries timed through the plain one-query-per-call path (0 = skip)")
    ap.add_argument("--served-requests", type=int, default=200,
                    help="requests per arrival rate of the served leg (1,000,000-sequence database; 0 = skip)")
    ap.add_argument("--served-rate", type=float, default=0.0,
                    help="one Poisson arrival rate for the served leg, 1/s (0 = the sweep 50-2,000/s)")
    ap.add_argument("--served-slots", type=int, default=64, help="resident query slots of the server")
    ap.add_argument("--served-segments", type=int, default=8, help="database segments per scan turn")
    ap.add_argument("--served-scale", type=float, default=1.0, help="served database scale (1.0 = 1M sequences)")
    ap.add_argument("--workload", default="sw_batched", choices=["sw_batched", "sw_plain", "sw_served", "nw_nucleotide", "long_pairs"],
                    help="sw_plain: a 10,000-sequence database with --queries queries of 375")
    ap.add_argument("--queries", type=int, default=None,
                    help="query count: --workload sw_plain (queries of 375), or a length-stratified subset of the "
                         "1,024-query batch")
    ap.add_argument("--db-memory", type=int, default=0,
                    help="device memory for the database in bytes (0 = automatic; smaller streams it)")
    ap.add_argument("--pairs", type=int, default=4096, help="pair count for --workload long_pairs")
    ap.add_argument("--pair-lo", type=int, default=5000, help="shortest query of --workload long_pairs")
    ap.add_argument("--pair-hi", type=int, default=30000, help="longest query of --workload long_pairs")
    ap.add_argument("--pair-align", default="alignment", choices=["alignment", "score"],
                    help="--workload long_pairs: COMPUTE_ALIGNMENT or COMPUTE_SCORE")
    args = ap.parse_args()
    if args.impl == "reference":
        sys.exit(run_reference_arm(args))
    if args.workload == "sw_served":
        sys.exit(run_served_arm(args))
    if args.workload == "nw_nucleotide":
        sys.exit(run_nw_arm(args))
    if args.workload == "long_pairs":
        sys.exit(run_pairs_arm(args))
    if args.split == "db":
        sys.exit(run_db_split(args))
    sys.exit(run_ours(args))


if __name__ == "__main__":
    main()
