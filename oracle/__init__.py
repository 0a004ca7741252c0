"""The test-only oracle of the libssa B200 build.

TEST INFRASTRUCTURE ONLY.  Two programs live here and only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may use them:

* ``liboracle.so`` -- ``ssa_oracle.c``, a plain-C restatement of the reference
  search path (lane scheduler, saturating lanes, overflow cascade, min-heap,
  traceback).  ``Oracle`` below binds it with ctypes.
* ``ref_run`` -- the reference libssa itself, compiled from its own sources by
  ``oracle/Makefile`` into ``oracle/_ref/``.  ``run_reference`` drives it.

Neither is ever called by the product (``libssa_b200``).
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "liboracle.so")
REF_RUN = os.path.join(REF_DIR, "ref_run")

AA_SYMBOLS = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ"
NT_SYMBOLS = "-ACMGRSVTWYHKDBN"


def build(reference_root: str | None = None) -> None:
    """Builds liboracle.so, and ref_run when the reference sources are given
    (``reference_root``, else the ``SSA_REFERENCE_ROOT`` environment variable)
    and present."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    reference_root = reference_root or os.environ.get("SSA_REFERENCE_ROOT")
    if reference_root and os.path.isdir(os.path.join(reference_root, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={reference_root}"], check=True)


def reference_available() -> bool:
    return os.path.exists(REF_RUN)


class _Config(ctypes.Structure):
    _fields_ = [
        ("algo", ctypes.c_int),
        ("bit_width", ctypes.c_int),
        ("align_type", ctypes.c_int),
        ("lanes8", ctypes.c_int),
        ("lanes16", ctypes.c_int),
        ("gap_open", ctypes.c_int),
        ("gap_extend", ctypes.c_int),
        ("hitcount", ctypes.c_uint64),
        ("chunk_size", ctypes.c_uint64),
        ("matrix", ctypes.c_int64 * 1024),
    ]


class _Hit(ctypes.Structure):
    _fields_ = [
        ("score", ctypes.c_int64),
        ("id", ctypes.c_uint64),
        ("q_start", ctypes.c_uint64),
        ("q_end", ctypes.c_uint64),
        ("d_start", ctypes.c_uint64),
        ("d_end", ctypes.c_uint64),
        ("cigar", ctypes.c_char_p),
    ]


class _Stats(ctypes.Structure):
    _fields_ = [("overflow8", ctypes.c_uint64), ("overflow16", ctypes.c_uint64)]


class _Lane(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int64), ("overflow", ctypes.c_int), ("blocks", ctypes.c_int64)]


@dataclass
class SearchConfig:
    """Mirror of the global settings a libssa search reads."""

    algo: str = "sw"                 # "sw" or "nw"
    bit_width: int = 8
    align_type: int = 1
    hitcount: int = 10
    chunk_size: int = 1000
    gap_open: int = -11
    gap_extend: int = -1
    lanes8: int = 32                 # AVX2 schedule
    lanes16: int = 16
    matrix: np.ndarray = field(default_factory=lambda: np.full(1024, -1, dtype=np.int64))


@dataclass
class Hit:
    score: int
    id: int
    q_start: int = 0
    q_end: int = 0
    d_start: int = 0
    d_end: int = 0
    cigar: str | None = None

    def key(self):
        return (self.id, self.score, self.cigar, self.q_start, self.q_end, self.d_start, self.d_end)


def map_codes(text: str, nucleotide: bool, drop_unknown: bool) -> np.ndarray:
    """ASCII -> residue codes with the reference's NCBI maps."""
    lib = _lib()
    raw = text.encode("latin-1")
    out = np.zeros(max(1, len(raw)), dtype=np.uint8)
    n = lib.oracle_map(raw, len(raw), int(nucleotide), int(drop_unknown),
                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return out[:n].copy()


def parse_matrix(text: str) -> np.ndarray:
    lib = _lib()
    out = np.zeros(1024, dtype=np.int64)
    rc = lib.oracle_parse_matrix(text.encode("latin-1"), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    if rc != 0:
        raise ValueError("matrix text does not parse")
    return out


def constant_matrix(match: int, mismatch: int) -> np.ndarray:
    lib = _lib()
    out = np.zeros(1024, dtype=np.int64)
    lib.oracle_constant_matrix(match, mismatch, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return out


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        lib.oracle_search.restype = ctypes.c_int
        lib.oracle_search.argtypes = [
            ctypes.POINTER(_Config), ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, ctypes.c_uint64,
            ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(_Hit),
            ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(_Stats)]
        lib.oracle_free_hits.argtypes = [ctypes.POINTER(_Hit), ctypes.c_uint64]
        lib.oracle_lane_result.restype = _Lane
        lib.oracle_lane_result.argtypes = [
            ctypes.POINTER(_Config), ctypes.c_int, ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64,
            ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64]
        lib.oracle_map.restype = ctypes.c_uint64
        lib.oracle_map.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_uint8)]
        lib.oracle_parse_matrix.restype = ctypes.c_int
        lib.oracle_parse_matrix.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        lib.oracle_constant_matrix.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
        for name in ("oracle_full_sw", "oracle_full_nw"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int64
            fn.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64,
                           ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64]
        _LIB = lib
    return _LIB


def _cfg(c: SearchConfig) -> _Config:
    x = _Config()
    x.algo = 0 if c.algo == "sw" else 1
    x.bit_width = c.bit_width
    x.align_type = c.align_type
    x.lanes8 = c.lanes8
    x.lanes16 = c.lanes16
    x.gap_open = c.gap_open
    x.gap_extend = c.gap_extend
    x.hitcount = c.hitcount
    x.chunk_size = c.chunk_size
    m = np.ascontiguousarray(c.matrix, dtype=np.int64)
    ctypes.memmove(x.matrix, m.ctypes.data, 1024 * 8)
    return x


def _u8(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def pack_db(seqs: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    offsets = np.zeros(len(seqs) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([len(s) for s in seqs])
    flat = np.concatenate(seqs).astype(np.uint8) if seqs and offsets[-1] else np.zeros(1, np.uint8)
    return np.ascontiguousarray(flat), offsets


def search(c: SearchConfig, query: np.ndarray, db_seqs: list[np.ndarray]) -> tuple[list[Hit], tuple[int, int]]:
    """Oracle search of mapped query codes against mapped database records."""
    lib = _lib()
    cfg = _cfg(c)
    q = np.ascontiguousarray(query, dtype=np.uint8)
    if q.size == 0:
        q = np.zeros(1, np.uint8)[:0]
    flat, offsets = pack_db(db_seqs)
    hits = (_Hit * max(1, c.hitcount))()
    n = ctypes.c_uint64(0)
    st = _Stats()
    qbuf = np.ascontiguousarray(np.append(q, 0).astype(np.uint8))
    lib.oracle_search(ctypes.byref(cfg), _u8(qbuf), len(q), len(db_seqs), _u8(flat),
                      offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), hits, ctypes.byref(n),
                      ctypes.byref(st))
    out = []
    for i in range(n.value):
        h = hits[i]
        out.append(Hit(int(h.score), int(h.id), int(h.q_start), int(h.q_end), int(h.d_start), int(h.d_end),
                       h.cigar.decode() if h.cigar is not None else None))
    lib.oracle_free_hits(hits, n.value)
    return out, (int(st.overflow8), int(st.overflow16))


def lane_result(c: SearchConfig, width: int, query: np.ndarray, dseq: np.ndarray) -> tuple[int, bool, int]:
    """(score, overflowed, blocks) of one sequence in one saturating lane."""
    lib = _lib()
    cfg = _cfg(c)
    q = np.ascontiguousarray(np.append(query, 0).astype(np.uint8))
    d = np.ascontiguousarray(np.append(dseq, 0).astype(np.uint8))
    r = lib.oracle_lane_result(ctypes.byref(cfg), width, _u8(q), len(query), _u8(d), len(dseq))
    return int(r.score), bool(r.overflow), int(r.blocks)


def full_score(c: SearchConfig, query: np.ndarray, dseq: np.ndarray) -> int:
    lib = _lib()
    cfg = _cfg(c)
    q = np.ascontiguousarray(np.append(query, 0).astype(np.uint8))
    d = np.ascontiguousarray(np.append(dseq, 0).astype(np.uint8))
    fn = lib.oracle_full_sw if c.algo == "sw" else lib.oracle_full_nw
    return int(fn(ctypes.byref(cfg), _u8(d), len(dseq), _u8(q), len(query)))


# --------------------------------------------------------------------------
# The reference binary
# --------------------------------------------------------------------------
def write_fasta(path: str, seqs: list[str]) -> None:
    with open(path, "w") as f:
        for i, s in enumerate(seqs):
            f.write(f">s{i}\n")
            for k in range(0, len(s), 60):
                f.write(s[k:k + 60] + "\n")


def write_sdb(path: str, seqs: list[bytes] | None = None, flat: np.ndarray | None = None,
              lengths: np.ndarray | None = None) -> None:
    """Binary database file read by the plugin (magic, count, lengths, residues)."""
    if seqs is not None:
        lengths = np.array([len(s) for s in seqs], dtype=np.uint64)
        flat = np.frombuffer(b"".join(seqs), dtype=np.uint8)
    with open(path, "wb") as f:
        f.write(b"SSADB001")
        f.write(np.uint64(len(lengths)).tobytes())
        f.write(np.ascontiguousarray(lengths, dtype=np.uint64).tobytes())
        f.write(np.ascontiguousarray(flat, dtype=np.uint8).tobytes())


def run_reference(db_path: str, queries: list[str], *, algo="sw", width=8, align=1, hits=10, symtype=1,
                  strands=1, gencode=(1, 1), matrix="builtin:blosum62", gap=(-11, -1), chunk=1000, threads=1,
                  simd=2, timing=False, repeat=1, workdir: str | None = None) -> list[dict]:
    """Runs the reference libssa on each query; returns one dict per query."""
    if not reference_available():
        raise RuntimeError("oracle/_ref/ref_run is not built")
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        qpath = os.path.join(td, "q.fas")
        write_fasta(qpath, queries)
        out = os.path.join(td, "out.json")
        cmd = [REF_RUN, "--algo", algo, "--width", str(width), "--align", str(align), "--hits", str(hits),
               "--symtype", str(symtype), "--strands", str(strands), "--gencode", f"{gencode[0]},{gencode[1]}",
               "--matrix", matrix, "--gap", f"{gap[0]},{gap[1]}", "--chunk", str(chunk), "--threads",
               str(threads), "--simd", str(simd), "--db", db_path, "--queries", qpath, "--out", out,
               "--repeat", str(repeat)]
        if timing:
            cmd.append("--time")
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        res = []
        with open(out) as f:
            for line in f:
                d = json.loads(line)
                if not d.get("warmup"):
                    res.append(d)
        return res


def reference_matrix(spec: str) -> np.ndarray:
    out = subprocess.run([REF_RUN, "--dump-matrix", spec], check=True, capture_output=True, text=True).stdout
    return np.array(json.loads(out), dtype=np.int64)
