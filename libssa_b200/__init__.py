"""Python mirror of the libssa C API, backed by the B200 build.

The functions below have the names, arguments and behaviour of the C entry
points in ``include/libssa.h`` (the reference's ``src/libssa.h``), bound with
ctypes to ``_lib/libssa.so``.  The database is served by ``_lib/libsdb_b200.so``,
the plugin implementing ``libssa_extern_db.h``; ``load_db_memory`` feeds it
sequences straight from Python.

The shared libraries must have been built (``python -m libssa_b200.build``);
importing this package fails loudly otherwise.  All searching runs on the GPU.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libssa.so")
PLUGIN_PATH = os.path.join(LIB_DIR, "libsdb_b200.so")

# constants of libssa.h (reference: src/libssa.h:29-72)
NUCLEOTIDE, AMINOACID, TRANS_QUERY, TRANS_DB, TRANS_BOTH = 0, 1, 2, 3, 4
FORWARD_STRAND, COMPLEMENTARY_STRAND, BOTH_STRANDS = 1, 2, 3
BIT_WIDTH_8, BIT_WIDTH_16, BIT_WIDTH_64 = 8, 16, 64
OUTPUT_SILENT, OUTPUT_ERROR, OUTPUT_WARNING, OUTPUT_INFO = 0, 1, 2, 3
COMPUTE_SCORE, COMPUTE_ALIGNMENT = 0, 1
READ_FROM_FILE, READ_FROM_STRING, MATRIX_BUILDIN = 0, 1, 2
COMPUTE_ON_SSE2, COMPUTE_ON_SSE41, COMPUTE_ON_AVX2 = 0, 1, 2
SSA_SMITH_WATERMAN, SSA_NEEDLEMAN_WUNSCH = 0, 1

EXPORTED = [
    "set_output_mode", "set_simd_compute_mode", "set_chunk_size", "set_thread_count", "init_score_matrix",
    "init_constant_scores", "init_gap_penalties", "init_symbol_translation", "init_db", "init_sequence_fasta",
    "free_sequence", "sw_align", "nw_align", "free_alignment", "ssa_exit", "ssa_align_batch", "ssa_get_stats",
    "ssa_query_length", "ssa_db_refresh", "ssa_b200_int_peak", "ssa_b200_score64_noalloc",
    "ssa_server_start", "ssa_server_submit", "ssa_server_wait", "ssa_server_get_stats", "ssa_server_stop",
    "ssa_b200_translation_table", "ssa_align_pairs", "ssa_b200_set_traceback_memory", "ssa_b200_set_db_memory",
    "ssa_b200_db_streamed",
]

# allocation-free scoring (include/libssa_b200.h)
NOALLOC_MAX_QUERY, NOALLOC_MAX_SEQ_LEN, NOALLOC_MAX_SEQS = 4096, 4096, 262144
NOALLOC_OK, NOALLOC_EINVAL, NOALLOC_ETOOBIG, NOALLOC_ECUDA, NOALLOC_ESEQLEN = 0, 1, 2, 3, 4


class DbSeq(ctypes.Structure):
    _fields_ = [("seq", ctypes.c_void_p), ("len", ctypes.c_size_t), ("ID", ctypes.c_size_t),
                ("strand", ctypes.c_int), ("frame", ctypes.c_int)]


class QSeq(ctypes.Structure):
    _fields_ = [("seq", ctypes.c_void_p), ("len", ctypes.c_size_t), ("strand", ctypes.c_int),
                ("frame", ctypes.c_int)]


class Alignment(ctypes.Structure):
    _fields_ = [("db_seq", DbSeq), ("query", QSeq), ("alignment", ctypes.c_char_p),
                ("alignment_len", ctypes.c_size_t), ("score", ctypes.c_long), ("align_q_start", ctypes.c_size_t),
                ("align_q_end", ctypes.c_size_t), ("align_d_start", ctypes.c_size_t),
                ("align_d_end", ctypes.c_size_t)]


class AlignmentList(ctypes.Structure):
    _fields_ = [("alignments", ctypes.POINTER(ctypes.POINTER(Alignment))), ("len", ctypes.c_size_t)]


class Stats(ctypes.Structure):
    _fields_ = [("overflow_8_to_16", ctypes.c_uint64), ("overflow_16_to_64", ctypes.c_uint64),
                ("cells", ctypes.c_uint64), ("gpu_seconds", ctypes.c_double),
                ("kernel_launches_total", ctypes.c_uint64), ("entry_seconds", ctypes.c_double),
                ("kernel_seconds", ctypes.c_double), ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64)]


P_LIST = ctypes.POINTER(AlignmentList)

_lib = None
_plugin = None


def libraries_built() -> bool:
    return os.path.exists(LIB_PATH) and os.path.exists(PLUGIN_PATH)


def load():
    """Loads the plugin and the library (RTLD_GLOBAL so libssa.so resolves
    the ssa_db_* imports against the plugin)."""
    global _lib, _plugin
    if _lib is not None:
        return _lib
    if not libraries_built():
        raise RuntimeError("libssa_b200 is not built: run `python -m libssa_b200.build` (the GPU library has "
                           "no CPU fallback)")
    _plugin = ctypes.CDLL(PLUGIN_PATH, mode=ctypes.RTLD_GLOBAL)
    lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
    lib.set_output_mode.argtypes = [ctypes.c_int]
    lib.set_simd_compute_mode.argtypes = [ctypes.c_int]
    lib.set_chunk_size.argtypes = [ctypes.c_size_t]
    lib.set_thread_count.argtypes = [ctypes.c_size_t]
    lib.init_score_matrix.argtypes = [ctypes.c_int, ctypes.c_char_p]
    lib.init_constant_scores.argtypes = [ctypes.c_int8, ctypes.c_int8]
    lib.init_gap_penalties.argtypes = [ctypes.c_int8, ctypes.c_int8]
    lib.init_symbol_translation.argtypes = [ctypes.c_int] * 4
    lib.init_db.argtypes = [ctypes.c_char_p]
    lib.init_sequence_fasta.argtypes = [ctypes.c_int, ctypes.c_char_p]
    lib.init_sequence_fasta.restype = ctypes.c_void_p
    lib.free_sequence.argtypes = [ctypes.c_void_p]
    for fn in (lib.sw_align, lib.nw_align):
        fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
        fn.restype = P_LIST
    lib.free_alignment.argtypes = [P_LIST]
    lib.ssa_exit.argtypes = []
    lib.ssa_align_batch.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t,
                                    ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P_LIST)]
    lib.ssa_align_batch.restype = ctypes.c_int
    lib.ssa_align_pairs.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                                    ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P_LIST)]
    lib.ssa_align_pairs.restype = ctypes.c_int
    lib.ssa_b200_set_traceback_memory.argtypes = [ctypes.c_size_t]
    lib.ssa_b200_set_db_memory.argtypes = [ctypes.c_size_t]
    lib.ssa_b200_db_streamed.restype = ctypes.c_int
    lib.ssa_get_stats.argtypes = [ctypes.POINTER(Stats)]
    lib.ssa_b200_query_overflows.restype = ctypes.c_size_t
    lib.ssa_b200_query_overflows.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                             ctypes.c_size_t]
    lib.ssa_db_refresh.argtypes = []
    lib.ssa_b200_int_peak.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.ssa_b200_simd_rate.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.ssa_b200_shard_scores.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t,
                                          ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]
    lib.ssa_b200_replay_gathered.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t,
                                             ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(P_LIST)]
    lib.ssa_b200_tuning_report.restype = ctypes.c_size_t
    lib.ssa_b200_tuning_report.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.ssa_b200_int_peak.restype = ctypes.c_int
    lib.ssa_query_length.argtypes = [ctypes.c_void_p]
    lib.ssa_query_length.restype = ctypes.c_size_t
    lib.ssa_b200_score64_noalloc.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_void_p, ctypes.c_void_p]
    lib.ssa_b200_score64_noalloc.restype = ctypes.c_int
    lib.ssa_server_start.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                     ctypes.c_size_t, ctypes.c_size_t]
    lib.ssa_server_start.restype = ctypes.c_void_p
    lib.ssa_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.ssa_server_submit.restype = ctypes.c_longlong
    lib.ssa_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double)]
    lib.ssa_server_wait.restype = P_LIST
    lib.ssa_server_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ServerStats)]
    lib.ssa_server_stop.argtypes = [ctypes.c_void_p]
    lib.ssa_b200_translation_table.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_uint8)]
    lib.ssa_b200_translation_table.restype = ctypes.c_int
    _plugin.ssa_db_b200_load_memory.argtypes = [ctypes.c_size_t, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)]
    _plugin.ssa_db_b200_load_memory.restype = ctypes.c_int
    _plugin.ssa_db_get_sequence_count.restype = ctypes.c_size_t
    _lib = lib
    return lib


# --------------------------------------------------------------------------
# libssa.h mirror
# --------------------------------------------------------------------------
def set_output_mode(mode: int) -> None:
    load().set_output_mode(mode)


def set_simd_compute_mode(mode: int) -> None:
    load().set_simd_compute_mode(mode)


def set_chunk_size(size: int) -> None:
    load().set_chunk_size(size)


def set_thread_count(count: int) -> None:
    load().set_thread_count(count)


def init_score_matrix(mode: int, matrix: str) -> None:
    load().init_score_matrix(mode, matrix.encode())


def init_constant_scores(match: int, mismatch: int) -> None:
    load().init_constant_scores(match, mismatch)


def init_gap_penalties(gap_open: int, gap_extend: int) -> None:
    load().init_gap_penalties(gap_open, gap_extend)


def init_symbol_translation(symtype: int, strands: int, db_gencode: int, q_gencode: int) -> None:
    load().init_symbol_translation(symtype, strands, db_gencode, q_gencode)


def init_db(path: str) -> None:
    load().init_db(path.encode())


def init_sequence_fasta(mode: int, text: str):
    """Returns an opaque query handle (int) or None when the reference would
    return NULL."""
    q = load().init_sequence_fasta(mode, text.encode("latin-1"))
    return q or None


def free_sequence(q) -> None:
    if q:
        load().free_sequence(q)


@dataclass
class Hit:
    id: int
    score: int
    cigar: str | None
    q_start: int
    q_end: int
    d_start: int
    d_end: int
    dlen: int
    qlen: int
    db_seq: bytes = b""
    strand: int = 0      # alignment_t.db_seq.strand
    frame: int = 0       # alignment_t.db_seq.frame
    qstrand: int = 0     # alignment_t.query.strand
    qframe: int = 0      # alignment_t.query.frame

    def key(self):
        return (self.id, self.score, self.cigar, self.q_start, self.q_end, self.d_start, self.d_end)

    def key_frames(self):
        return self.key() + (self.strand, self.frame, self.qstrand, self.qframe)


def _read_list(lp) -> list[Hit]:
    out = []
    lst = lp.contents
    for i in range(lst.len):
        a = lst.alignments[i].contents
        cig = a.alignment.decode() if a.alignment is not None else None
        seq = ctypes.string_at(a.db_seq.seq, a.db_seq.len) if a.db_seq.seq else b""
        out.append(Hit(int(a.db_seq.ID), int(a.score), cig, int(a.align_q_start), int(a.align_q_end),
                       int(a.align_d_start), int(a.align_d_end), int(a.db_seq.len), int(a.query.len), seq,
                       int(a.db_seq.strand), int(a.db_seq.frame), int(a.query.strand), int(a.query.frame)))
    return out


def sw_align(q, hitcount: int, bit_width: int, align_type: int) -> list[Hit]:
    lib = load()
    lp = lib.sw_align(q, hitcount, bit_width, align_type)
    try:
        return _read_list(lp)
    finally:
        lib.free_alignment(lp)


def nw_align(q, hitcount: int, bit_width: int, align_type: int) -> list[Hit]:
    lib = load()
    lp = lib.nw_align(q, hitcount, bit_width, align_type)
    try:
        return _read_list(lp)
    finally:
        lib.free_alignment(lp)


def ssa_exit() -> None:
    load().ssa_exit()


# --------------------------------------------------------------------------
# libssa_b200.h extensions
# --------------------------------------------------------------------------
def align_batch(algorithm: int, queries: list, hitcount: int, bit_width: int, align_type: int) -> list[list[Hit]]:
    """Batched search of several query handles; one hit list per query."""
    lib = load()
    n = len(queries)
    qarr = (ctypes.c_void_p * max(1, n))(*queries)
    res = (P_LIST * max(1, n))()
    lib.ssa_align_batch(algorithm, qarr, n, hitcount, bit_width, align_type, res)
    out = []
    for i in range(n):
        out.append(_read_list(res[i]))
        lib.free_alignment(res[i])
    return out


def align_pairs(algorithm: int, queries: list, db_ids: list[int], bit_width: int, align_type: int) -> list[list[Hit]]:
    """Long-pair batch: query handle i against database sequence db_ids[i] alone.

    Each list equals sw_align / nw_align(queries[i], 1, ...) against a database
    holding only that sequence (one hit, or none for an empty sequence), with the
    hit's ID db_ids[i].  Raises ValueError for settings the call refuses.
    """
    lib = load()
    n = len(queries)
    if len(db_ids) != n:
        raise ValueError("one database ID per query")
    qarr = (ctypes.c_void_p * max(1, n))(*queries)
    ids = (ctypes.c_size_t * max(1, n))(*db_ids)
    res = (P_LIST * max(1, n))()
    if lib.ssa_align_pairs(algorithm, qarr, ids, n, bit_width, align_type, res) != 0:
        raise ValueError("ssa_align_pairs refused the settings or IDs")
    out = []
    for i in range(n):
        out.append(_read_list(res[i]))
        lib.free_alignment(res[i])
    return out


def set_db_memory(nbytes: int) -> None:
    """Device memory for the packed database (0 = automatic); a larger database is streamed."""
    load().ssa_b200_set_db_memory(nbytes)


def db_streamed() -> bool:
    return bool(load().ssa_b200_db_streamed())


def set_traceback_memory(nbytes: int) -> None:
    """Direction-matrix memory of one traceback wave (0 = automatic)."""
    load().ssa_b200_set_traceback_memory(nbytes)


def stats() -> Stats:
    s = Stats()
    load().ssa_get_stats(ctypes.byref(s))
    return s


SIMD_PROBE_OPS = ["__viaddmax_s16x2", "__vmaxs2", "__vimax3_s16x2", "__vaddss2", "__vsubss2", "__vaddss4",
                  "__vmaxs4", "__vsubus4", "__vaddus4", "__vmaxu4", "__vadd4", "__vsub4", "max.f16x2", "iadd"]


def simd_rates() -> dict[str, float]:
    """Warp intrinsics per clock per SM of each probed packed-integer intrinsic."""
    lib = load()
    out = {}
    for op, name in enumerate(SIMD_PROBE_OPS):
        v = ctypes.c_double(0)
        if lib.ssa_b200_simd_rate(op, ctypes.byref(v)) != 0:
            raise RuntimeError(f"probe of {name} failed")
        out[name] = v.value
    return out


def shard_scores(algorithm: int, queries: list, bit_width: int, id_lo: int, id_hi: int):
    """ssa_b200_shard_scores(): (scores int64, entry-width blocks int32,
    16-bit blocks int32), each n_queries x (id_hi - id_lo); blocks are -1 where
    the lane reported."""
    import numpy as np
    lib = load()
    n = len(queries)
    w = max(0, id_hi - id_lo)
    sc = np.zeros((n, w), dtype=np.int64)
    be = np.full((n, w), -1, dtype=np.int32)
    b16 = np.full((n, w), -1, dtype=np.int32)
    qarr = (ctypes.c_void_p * max(1, n))(*queries)
    if lib.ssa_b200_shard_scores(algorithm, qarr, n, bit_width, id_lo, id_hi, sc.ctypes.data, be.ctypes.data,
                                 b16.ctypes.data) != 0:
        raise ValueError("ssa_b200_shard_scores refused the settings or range")
    return sc, be, b16


def replay_gathered(algorithm: int, queries: list, hitcount: int, bit_width: int, align_type: int, scores,
                    blocks_entry, blocks_16) -> list[list[Hit]]:
    """ssa_b200_replay_gathered(): hit lists from per-record results of the
    whole database (n_queries x records arrays, as shard_scores returns them
    per range, concatenated in record order)."""
    import numpy as np
    lib = load()
    n = len(queries)
    sc = np.ascontiguousarray(scores, dtype=np.int64)
    be = np.ascontiguousarray(blocks_entry, dtype=np.int32)
    b16 = np.ascontiguousarray(blocks_16, dtype=np.int32)
    qarr = (ctypes.c_void_p * max(1, n))(*queries)
    res = (P_LIST * max(1, n))()
    if lib.ssa_b200_replay_gathered(algorithm, qarr, n, hitcount, bit_width, align_type, sc.ctypes.data,
                                    be.ctypes.data, b16.ctypes.data, res) != 0:
        raise ValueError("ssa_b200_replay_gathered refused the settings")
    out = []
    for i in range(n):
        out.append(_read_list(res[i]))
        lib.free_alignment(res[i])
    return out


def tuning_report() -> dict:
    """Origin of the entry-pass shape table and the shapes of the last search call."""
    import json
    lib = load()
    n = lib.ssa_b200_tuning_report(None, 0)
    buf = ctypes.create_string_buffer(n)
    lib.ssa_b200_tuning_report(buf, n)
    return json.loads(buf.value.decode())


def query_overflows() -> list[tuple[int, int]]:
    """(8->16, 16->64) overflow counters of each query of the last search call."""
    lib = load()
    n = lib.ssa_b200_query_overflows(None, None, 0)
    a = (ctypes.c_uint64 * max(1, n))()
    b = (ctypes.c_uint64 * max(1, n))()
    lib.ssa_b200_query_overflows(a, b, n)
    return [(int(a[i]), int(b[i])) for i in range(n)]


def int_peak() -> tuple[float, float]:
    """(operations per second, warp instructions per clock per SM) of the
    fused packed 16x2 add-max on the current device: the integer ALU pipe's
    ceiling, counting an add and a max per 16-bit half."""
    a, b = ctypes.c_double(0), ctypes.c_double(0)
    if load().ssa_b200_int_peak(ctypes.byref(a), ctypes.byref(b)) != 0:
        raise RuntimeError("integer peak probe failed")
    return a.value, b.value


def score64_noalloc(algorithm: int, d_query: int, query_len: int, d_codes: int, d_offsets: int,
                    d_lengths: int, count: int, max_seq_len: int, d_scores: int, stream: int = 0) -> int:
    """ssa_b200_score64_noalloc() on raw device addresses; returns its status
    code (NOALLOC_OK on success)."""
    return int(load().ssa_b200_score64_noalloc(algorithm, d_query, query_len, d_codes, d_offsets, d_lengths,
                                               count, max_seq_len, d_scores, stream or None))


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("waves", ctypes.c_uint64),
                ("cells", ctypes.c_uint64), ("busy_seconds", ctypes.c_double), ("device_seconds", ctypes.c_double),
                ("slots", ctypes.c_uint32), ("segments", ctypes.c_uint32), ("queued", ctypes.c_uint64),
                ("slot_waves", ctypes.c_uint64), ("max_pending", ctypes.c_uint32), ("max_occupied", ctypes.c_uint32)]


SERVE_MAX_QUERY = 8192


class Server:
    """The request loop of include/libssa_b200.h (ssa_server_*): queries are
    admitted into resident slots and folded into the running database scan;
    each result equals the query's sw_align/nw_align result alone."""

    def __init__(self, algorithm: int, hitcount: int, bit_width: int, align_type: int, slots: int = 64,
                 segments: int = 8, memory_budget: int = 0):
        self._lib = load()
        self._h = self._lib.ssa_server_start(algorithm, hitcount, bit_width, align_type, slots, segments,
                                             memory_budget)

    def submit(self, q) -> int:
        t = int(self._lib.ssa_server_submit(self._h, q))
        if t < 0:
            raise ValueError("request refused")
        return t

    def wait(self, ticket: int) -> tuple[list[Hit], float]:
        lat = ctypes.c_double(0)
        lp = self._lib.ssa_server_wait(self._h, ticket, ctypes.byref(lat))
        if not lp:
            raise KeyError(ticket)
        hits = _read_list(lp)
        self._lib.free_alignment(lp)
        return hits, lat.value

    def stats(self) -> ServerStats:
        st = ServerStats()
        self._lib.ssa_server_get_stats(self._h, ctypes.byref(st))
        return st

    def stop(self) -> None:
        if self._h:
            self._lib.ssa_server_stop(self._h)
            self._h = None


def translation_table(code: int) -> list[int]:
    """Amino-acid code of every nucleotide triple (a, b, c), codes 0-15, index
    a*256 + b*16 + c, under NCBI genetic code `code`."""
    out = (ctypes.c_uint8 * 4096)()
    if load().ssa_b200_translation_table(code, out) != 0:
        raise ValueError(f"no genetic code {code}")
    return list(out)


def query_length(q) -> int:
    return int(load().ssa_query_length(q))


def load_db_memory(seqs: list[bytes] | None = None, flat: np.ndarray | None = None,
                   offsets: np.ndarray | None = None) -> None:
    """Installs a database in the plugin from memory (ASCII residues)."""
    load()
    if seqs is not None:
        offsets = np.zeros(len(seqs) + 1, dtype=np.uint64)
        offsets[1:] = np.cumsum([len(s) for s in seqs])
        flat_bytes = b"".join(seqs)
    else:
        flat_bytes = np.ascontiguousarray(flat, dtype=np.uint8).tobytes()
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    rc = _plugin.ssa_db_b200_load_memory(len(offsets) - 1, flat_bytes,
                                         offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
    if rc != 0:
        raise MemoryError("database plugin could not store the sequences")
    # the library re-packs on the next search
    load().ssa_db_refresh()


def db_count() -> int:
    load()
    return int(_plugin.ssa_db_get_sequence_count())
