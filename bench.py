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
* ``roofline``: the entry-pass kernel against the measured integer ALU-pipe
  ceiling of the same device (fused 16x2 add-max: an add and a max per 16-bit
  half), 9 integer operations per cell;
* ``cpu_baseline``: the reference libssa (built from its sources into
  oracle/_ref) on the host cores, on a sample of the same workload;
* ``served``: 64 requests arriving as a Poisson process (50/s) into
  the request loop (``ssa_server_*``) over a resident 1,000,000-sequence
  database: GCUPS over first arrival to last result, p50/p99 latency.
  ``--workload sw_served`` prints that leg alone as its own line.

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
    return w


def rank_workload(args, rank: int):
    """A rank's shard of the job: its own seeded query batch (rank 0 the
    canonical one) against the full database, which every rank holds."""
    return make_workload(args.scale, 3 if rank == 0 else 3 + rank, args.workload, args.queries)


def load_traffic() -> float | None:
    """DRAM bytes per cell of the entry pass, from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "sw_qpair_kernel_traffic_scale05.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_cell:"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


# --------------------------------------------------------------------------
# CPU baseline: the reference built from its sources (oracle/_ref/ref_run)
# --------------------------------------------------------------------------
def reference_sample(w, n_queries: int, threads: int, repeat: int = 1) -> tuple[float, float, str]:
    """(GCUPS, seconds, description) of the reference on a query sample."""
    import oracle
    if not oracle.reference_available():
        raise RuntimeError("oracle/_ref/ref_run is not built")
    import numpy as np
    lens = np.array([len(q) for q in w.queries])
    # a representative sample: queries at evenly spaced length quantiles
    order = np.argsort(lens)
    pick = [int(order[int((i + 0.5) * len(order) / n_queries)]) for i in range(n_queries)]
    qs = [w.queries[i].decode() for i in pick]
    with tempfile.TemporaryDirectory() as td:
        db = os.path.join(td, "db.sdb")
        oracle.write_sdb(db, flat=w.db_flat, lengths=np.diff(w.db_offsets))
        res = oracle.run_reference(db, qs, algo="sw", width=8, align=1, hits=10, symtype=1,
                                   matrix="builtin:blosum62", gap=(-11, -1), chunk=1000, threads=threads, simd=2,
                                   timing=True, repeat=repeat)
    residues = int(w.db_offsets[-1])
    secs = sum(r["seconds"] for r in res)
    cells = sum(len(q) for q in qs) * residues
    desc = (f"{n_queries} queries (lengths {sorted(len(q) for q in qs)}) of the workload vs the full "
            f"{w.n_db}-sequence database, sw_align COMPUTE_ALIGNMENT, 8-bit entry, AVX2, {threads} threads")
    return cells / secs / 1e9, secs, desc


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
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return 0
    w = make_workload(args.scale, 3)
    threads = os.cpu_count() or 1
    vals = []
    desc = ""
    for i in range(args.warmup + args.steps):
        g, secs, desc = reference_sample(w, args.ref_queries, threads)
        if i >= args.warmup:
            vals.append((g, secs))
    value = statistics.median(v[0] for v in vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GCUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * statistics.median(v[1] for v in vals), 3), "higher_is_better": True,
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
def run_ours(args):
    world, rank, local, pg = dist_setup()
    os.environ["SSA_B200_DEVICE"] = str(local)
    import libssa_b200 as L
    if not L.libraries_built():
        from libssa_b200 import build
        build.build()
    L.load()
    w = rank_workload(args, rank)
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)
    L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
    L.init_gap_penalties(-11, -1)
    L.set_chunk_size(1000)
    L.set_simd_compute_mode(L.COMPUTE_ON_AVX2)
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
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        wall.append(time.perf_counter() - t0)
        st = L.stats()
        dev.append(st.kernel_seconds)
        entry.append(st.entry_seconds)
        h2d.append(st.h2d_bytes)
        d2h.append(st.d2h_bytes)
    clocks = sampler.stop()
    launches = L.stats().kernel_launches_total - launches0
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
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the entry-pass launches "
                                       "at half scale, scaled by cells (profiles/sw_qpair_kernel_traffic_scale05.md)",
                     "kernel": ("sw_qpair_kernel (entry pass, all rows-per-thread classes)" if len(w.queries) > 1
                                else "sw_fast_kernel (entry pass)"),
                     "peak_source": "measured on this device: integer ALU pipe running fused 16x2 add-max "
                                    f"({peak_ipc:.2f} warp-inst/clk/SM, an add and a max per 16-bit half); "
                                    "9 integer ops per cell (4 adds, 5 maxes); neither HBM nor tensor cores "
                                    "bound this integer max-plus recurrence"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "timing": {"device_seconds": round(t_dev, 4), "wall_seconds": round(t_wall, 4),
                   "entry_seconds_median": round(t_entry, 4)},
    }
    if args.plain_queries > 0:
        # the plain one-query-per-call path on a length-stratified query sample
        import numpy as np
        lens = np.array([len(q) for q in w.queries])
        order = np.argsort(lens)
        pick = [int(order[int((i + 0.5) * len(order) / args.plain_queries)]) for i in range(args.plain_queries)]
        sample = [qs[i] for i in pick]
        L.sw_align(sample[0], 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT)
        t0 = time.perf_counter()
        for q in sample:
            L.sw_align(q, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT)
        t_plain = time.perf_counter() - t0
        cells_plain = sum(len(w.queries[i]) for i in pick) * int(w.db_offsets[-1])
        line["plain_gpu"] = {"value": round(cells_plain / t_plain / 1e9, 2), "unit": "GCUPS",
                             "sample": f"{args.plain_queries} length-stratified queries, one sw_align call each "
                                       "(COMPUTE_ALIGNMENT), wall time"}
    if world == 1 and not args.no_cpu_baseline:
        try:
            g, secs, desc = reference_sample(w, args.ref_queries, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": round(g, 3), "unit": "GCUPS", "cores": os.cpu_count() or 1,
                                    "kind": "reference", "sample": desc}
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": "GCUPS", "cores": os.cpu_count() or 1,
                                    "kind": "reference", "sample": f"unavailable: {e}"}
    for q in qs:
        L.free_sequence(q)
    if world == 1 and args.served_queries > 0:
        line["served"] = served_leg(args, L)
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# served: Poisson arrivals into the request loop (ssa_server_*)
# --------------------------------------------------------------------------
def served_leg(args, L) -> dict:
    """A resident 1,000,000-sequence database, queries arriving as a
    Poisson process into the server; GCUPS over the wall time from the first
    arrival to the last completion, and the submit-to-result latencies."""
    import numpy as np
    from libssa_b200 import workloads as W
    w = W.sw_served_db(seed=4, scale=args.served_scale)
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)
    L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
    L.init_gap_penalties(-11, -1)
    L.set_chunk_size(1000)
    L.set_simd_compute_mode(L.COMPUTE_ON_AVX2)
    L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)
    texts = [q.decode() for q in W.served_queries(seed=40, n=args.served_queries)]
    arrivals = W.poisson_arrivals(seed=41, rate=args.served_rate, n=len(texts))
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, t) for t in texts]
    server = L.Server(L.SSA_SMITH_WATERMAN, 10, L.BIT_WIDTH_8, L.COMPUTE_ALIGNMENT, slots=args.served_slots,
                      segments=args.served_segments)
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
    lat = []
    for t in tickets:
        _, latency = server.wait(t)
        lat.append(latency)
    wall = time.perf_counter() - t0
    st = server.stats()
    server.stop()
    for q in qs:
        L.free_sequence(q)
    residues = int(w.db_offsets[-1])
    cells = sum(len(t) for t in texts) * residues
    lat_ms = np.array(lat) * 1e3
    return {"value": round(cells / wall / 1e9, 2), "unit": "GCUPS",
            "latency_ms": {"p50": round(float(np.percentile(lat_ms, 50)), 1),
                           "p99": round(float(np.percentile(lat_ms, 99)), 1),
                           "max": round(float(lat_ms.max()), 1)},
            "config": {"workload": "sw_served", "db_sequences": w.n_db, "db_residues": residues,
                       "queries": len(texts), "arrival_rate_qps": args.served_rate, "slots": args.served_slots,
                       "segments": int(st.segments), "waves": int(st.waves), "hits": 10,
                       "align_type": "COMPUTE_ALIGNMENT"},
            "device_seconds": round(st.device_seconds, 3), "wall_seconds": round(wall, 3),
            "timing": "wall time from the first arrival to the last completion; latency = submit to result"}


def run_nw_arm(args):
    """64 nucleotide queries vs 200,000 sequences, Needleman-Wunsch,
    16-bit entry, constant scores 2/-3, gaps 5/2, top 20 with CIGAR; one step is
    one batched search (ssa_align_batch)."""
    import libssa_b200 as L
    from libssa_b200 import workloads as W
    L.load()
    w = W.nw_nucleotide(seed=2, scale=args.scale, n_queries=64)
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.NUCLEOTIDE, L.FORWARD_STRAND, 1, 1)
    L.init_constant_scores(2, -3)
    L.init_gap_penalties(-5, -2)
    L.set_chunk_size(1000)
    L.set_simd_compute_mode(L.COMPUTE_ON_AVX2)
    L.load_db_memory(flat=w.db_flat, offsets=w.db_offsets)
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, q.decode()) for q in w.queries]
    cells = sum(len(q) for q in w.queries) * int(w.db_offsets[-1])
    for _ in range(args.warmup):
        L.align_batch(L.SSA_NEEDLEMAN_WUNSCH, qs, 20, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
    dev, wall = 0.0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        L.align_batch(L.SSA_NEEDLEMAN_WUNSCH, qs, 20, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
        wall += time.perf_counter() - t0
        dev += L.stats().kernel_seconds
    st = L.stats()
    line = {"metric": "GCUPS (batched NW nucleotide search, 64 queries vs 200k sequences, top 20 with CIGAR)",
            "value": round(cells * args.steps / dev / 1e9, 2), "unit": "GCUPS", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int16 lanes (16-bit entry), int32", "data": "synthetic (seeded: 64 nucleotide queries of 150-600 vs 200,000 sequences of 100-1,500)",
            "config": {"workload": "nw_nucleotide", "queries": len(qs), "db_sequences": w.n_db,
                       "db_residues": int(w.db_offsets[-1]), "cells_per_step": cells, "scale": args.scale},
            "e2e": {"value": round(cells * args.steps / wall / 1e9, 2), "unit": "GCUPS"},
            "timing": {"device_seconds": round(dev, 4), "wall_seconds": round(wall, 4),
                       "entry_seconds_last": round(st.entry_seconds, 4),
                       "overflow_16_to_64_last": int(st.overflow_16_to_64)}}
    print(json.dumps(line), flush=True)
    for q in qs:
        L.free_sequence(q)
    return 0


def run_pairs_arm(args):
    """Long pairs, each a query of 5,000-30,000 residues and a mutated
    copy of it (85-99% identity, 1% indel events of length 1-20), BLOSUM62, gaps
    11/1, 16-bit entry, full CIGAR.  One step aligns every pair with
    Smith-Waterman and with Needleman-Wunsch through ssa_align_pairs (query i
    against database sequence i alone)."""
    import libssa_b200 as L
    from libssa_b200 import workloads as W
    L.load()
    pairs = W.long_pairs(seed=5, n_pairs=args.pairs, lo=args.pair_lo, hi=args.pair_hi)
    L.set_output_mode(L.OUTPUT_SILENT)
    L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)
    L.init_score_matrix(L.MATRIX_BUILDIN, "blosum62")
    L.init_gap_penalties(-11, -1)
    L.set_chunk_size(1000)
    L.set_simd_compute_mode(L.COMPUTE_ON_AVX2)
    L.load_db_memory([b for _, b in pairs])
    qs = [L.init_sequence_fasta(L.READ_FROM_STRING, a.decode()) for a, _ in pairs]
    ids = list(range(len(pairs)))
    cells_one = sum(len(a) * len(b) for a, b in pairs)
    cells = 2 * cells_one
    algos = (L.SSA_SMITH_WATERMAN, L.SSA_NEEDLEMAN_WUNSCH)
    for _ in range(args.warmup):
        for algo in algos:
            L.align_pairs(algo, qs, ids, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
    dev, wall = 0.0, 0.0
    per_algo = {0: 0.0, 1: 0.0}
    h2d = d2h = 0
    for _ in range(args.steps):
        for algo in algos:
            t0 = time.perf_counter()
            L.align_pairs(algo, qs, ids, L.BIT_WIDTH_16, L.COMPUTE_ALIGNMENT)
            wall += time.perf_counter() - t0
            st = L.stats()
            dev += st.gpu_seconds
            per_algo[algo] += st.gpu_seconds
            h2d += int(st.h2d_bytes)
            d2h += int(st.d2h_bytes)
    line = {"metric": "GCUPS (long-pair SW and NW alignments with CIGAR, 5k-30k residues per side)",
            "value": round(cells * args.steps / dev / 1e9, 2), "unit": "GCUPS", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dev / args.steps * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded: 4,096 query / mutated-copy pairs of 5,000-30,000 residues)",
            "config": {"workload": "long_pairs", "pairs": len(pairs), "query_lengths": [args.pair_lo, args.pair_hi],
                       "algorithms": ["sw", "nw"],
                       "cells_per_step": cells, "bit_width": 16,
                       "l2": "inputs and direction matrices far larger than L2"},
            "e2e": {"value": round(cells * args.steps / wall / 1e9, 2), "unit": "GCUPS",
                    "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps},
            "timing": {"device_seconds": round(dev, 4), "wall_seconds": round(wall, 4),
                       "sw_seconds": round(per_algo[0], 4), "nw_seconds": round(per_algo[1], 4)}}
    if not args.no_cpu_baseline:
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
    res = served_leg(args, L)
    line = {"metric": "GCUPS (served SW search, 1,000,000 resident sequences, Poisson arrivals, top 10 with CIGAR)",
            "value": res["value"], "unit": "GCUPS", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int16x2 (8-bit lane semantics), int32", "data": "synthetic (seeded: 1,000,000 resident sequences, Poisson arrivals)",
            **{k: v for k, v in res.items() if k not in ("value", "unit")}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="database and query count scale (1.0 = full)")
    ap.add_argument("--ref-queries", type=int, default=4, help="queries in the reference CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-queries", type=int, default=16,
                    help="queries timed through the plain one-query-per-call path (0 = skip)")
    ap.add_argument("--served-queries", type=int, default=64,
                    help="requests of the served leg (1,000,000-sequence database; 0 = skip)")
    ap.add_argument("--served-rate", type=float, default=50.0, help="Poisson arrival rate of the served leg, 1/s")
    ap.add_argument("--served-slots", type=int, default=64, help="resident query slots of the server")
    ap.add_argument("--served-segments", type=int, default=8, help="database segments per scan turn")
    ap.add_argument("--served-scale", type=float, default=1.0, help="served database scale (1.0 = 1M sequences)")
    ap.add_argument("--workload", default="sw_batched", choices=["sw_batched", "sw_plain", "sw_served", "nw_nucleotide", "long_pairs"],
                    help="sw_plain: a 10,000-sequence database with --queries queries of 375")
    ap.add_argument("--queries", type=int, default=None, help="query count for --workload sw_plain")
    ap.add_argument("--db-memory", type=int, default=0,
                    help="device memory for the database in bytes (0 = automatic; smaller streams it)")
    ap.add_argument("--pairs", type=int, default=4096, help="pair count for --workload long_pairs")
    ap.add_argument("--pair-lo", type=int, default=5000, help="shortest query of --workload long_pairs")
    ap.add_argument("--pair-hi", type=int, default=30000, help="longest query of --workload long_pairs")
    args = ap.parse_args()
    if args.impl == "reference":
        sys.exit(run_reference_arm(args))
    if args.workload == "sw_served":
        sys.exit(run_served_arm(args))
    if args.workload == "nw_nucleotide":
        sys.exit(run_nw_arm(args))
    if args.workload == "long_pairs":
        sys.exit(run_pairs_arm(args))
    sys.exit(run_ours(args))


if __name__ == "__main__":
    main()
