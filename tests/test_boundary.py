"""The drop-in boundary: exported symbols, binary layout, a C client, the plugin.

CPU tests (no CUDA device needed): the libraries load and export every
function include/*.h declares; the structs and constants of include/libssa.h
have the reference's layout (tests/golden/abi_layout.json, taken from the
reference's own headers); a C program written against the reference API
compiles and links against the build; the database plugin reads FASTA, .sdb
and in-memory databases with the reference's ID and record rules; without a
device a search fails loudly instead of falling back to the CPU.  The GPU test
runs the C client and checks its output against the reference's known answers
(tests/test_libssa.c:30-93).
"""
import ctypes
import json
import os
import re
import subprocess
import sys

import pytest

from helpers import DATA

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
CLIENT = os.path.join(ROOT, "tests", "c_client")
GOLDEN = os.path.join(ROOT, "tests", "golden")

PROTO = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s+\**\s*([a-z_][a-z0-9_]*)\s*\(", re.M)


def declared(header: str) -> list[str]:
    text = open(os.path.join(INCLUDE, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return sorted(set(PROTO.findall(text)))


def exported(path: str) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", path], check=True, capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_headers_declare_the_reference_api():
    assert declared("libssa.h") == sorted([
        "set_output_mode", "set_simd_compute_mode", "set_chunk_size", "set_thread_count", "init_score_matrix",
        "init_constant_scores", "init_gap_penalties", "init_symbol_translation", "init_db", "init_sequence_fasta",
        "free_sequence", "sw_align", "nw_align", "free_alignment", "ssa_exit"])
    assert declared("libssa_extern_db.h") == sorted(
        ["ssa_db_init", "ssa_db_get_sequence_count", "ssa_db_get_sequence", "ssa_db_close"])


def test_libraries_load_and_export_every_declared_function(built_library):
    import libssa_b200 as L
    lib_syms = exported(L.LIB_PATH)
    plugin_syms = exported(L.PLUGIN_PATH)
    for name in declared("libssa.h") + declared("libssa_b200.h"):
        where = plugin_syms if name.startswith("ssa_db_b200_") else lib_syms
        assert name in where, name
    for name in declared("libssa_extern_db.h"):
        assert name in plugin_syms, name
    # and ctypes resolves them in the loaded process
    lib = L.load()
    for name in declared("libssa.h") + declared("libssa_b200.h"):
        if not name.startswith("ssa_db_b200_"):
            assert hasattr(lib, name), name
    assert set(L.EXPORTED) <= lib_syms


def test_abi_layout_matches_reference(tmp_path):
    exe = tmp_path / "abi_layout"
    subprocess.run(["gcc", "-I" + INCLUDE, "-o", str(exe), os.path.join(CLIENT, "abi_layout.c")], check=True)
    ours = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    with open(os.path.join(GOLDEN, "abi_layout.json")) as f:
        ref = json.load(f)
    assert ours == ref


def _build_client(built_library, out: str) -> str:
    import libssa_b200 as L
    exe = os.path.join(out, "search_example")
    subprocess.run(["gcc", "-O2", "-I" + INCLUDE, "-o", exe, os.path.join(CLIENT, "search_example.c"),
                    "-L" + L.LIB_DIR, "-lssa", "-lsdb_b200", "-Wl,-rpath," + L.LIB_DIR], check=True)
    return exe


def test_c_client_compiles_and_links(built_library, tmp_path):
    exe = _build_client(built_library, str(tmp_path))
    assert os.path.exists(exe)
    out = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    assert "libssa.so" in out and "libsdb_b200.so" in out


@pytest.mark.gpu
def test_c_client_reproduces_reference_kat(built_library, tmp_path):
    from kats import KATS
    exe = _build_client(built_library, str(tmp_path))
    res = subprocess.run([exe, os.path.join(DATA, "AF091148.fas"), os.path.join(DATA, "one_seq.fas")],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    got = {"sw": [], "nw": []}
    for line in res.stdout.splitlines():
        algo, id_, score, cigar = line.split()[:4]
        got[algo].append((int(score), int(id_), cigar))
    kat = KATS[0]
    for algo, _w, _a, _h, _s, expected in kat["calls"]:
        assert got[algo] == [tuple(h) for h in expected["hits"]], algo


# --------------------------------------------------------------------------
# the database plugin (host code only)
# --------------------------------------------------------------------------
class SeqInfo(ctypes.Structure):
    _fields_ = [("ID", ctypes.c_size_t), ("seqlen", ctypes.c_size_t), ("seq", ctypes.c_char_p)]


@pytest.fixture()
def plugin(built_library):
    import libssa_b200 as L
    p = ctypes.CDLL(L.PLUGIN_PATH)
    p.ssa_db_init.argtypes = [ctypes.c_char_p]
    p.ssa_db_init.restype = ctypes.c_int
    p.ssa_db_get_sequence_count.restype = ctypes.c_size_t
    p.ssa_db_get_sequence.argtypes = [ctypes.c_size_t]
    p.ssa_db_get_sequence.restype = ctypes.POINTER(SeqInfo)
    p.ssa_db_b200_load_memory.argtypes = [ctypes.c_size_t, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)]
    return p


def _records(p) -> list[tuple[int, bytes]]:
    out = []
    for i in range(p.ssa_db_get_sequence_count()):
        info = p.ssa_db_get_sequence(i)
        out.append((info.contents.ID, ctypes.string_at(info.contents.seq, info.contents.seqlen)))
    assert not p.ssa_db_get_sequence(p.ssa_db_get_sequence_count())     # NULL past the end
    return out


def test_plugin_fasta_ids_and_records(plugin, tmp_path):
    fa = tmp_path / "db.fasta"
    fa.write_bytes(b">a first\nACGT\r\nAC\n>b\n\n>c third\nMKV\nLL\n")
    assert plugin.ssa_db_init(str(fa).encode()) == 0
    # IDs are record indexes in file order (reference: tests/test_libssa_extern_db.c:31-41);
    # line breaks are not residues; an empty record is kept
    assert _records(plugin) == [(0, b"ACGTAC"), (1, b""), (2, b"MKVLL")]


def test_plugin_fasta_reference_fixture(plugin):
    from helpers import read_fasta
    path = os.path.join(DATA, "AF091148.fas")
    assert plugin.ssa_db_init(path.encode()) == 0
    recs = _records(plugin)
    assert [r[1] for r in recs] == read_fasta(path)
    assert [r[0] for r in recs] == list(range(len(recs)))


def test_plugin_sdb_and_memory(plugin, tmp_path):
    import numpy as np
    import oracle
    seqs = [b"ACDE", b"", b"WYV" * 5]
    path = str(tmp_path / "db.sdb")
    oracle.write_sdb(path, seqs=seqs)
    assert plugin.ssa_db_init(path.encode()) == 0
    assert [r[1] for r in _records(plugin)] == seqs
    offs = np.zeros(len(seqs) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    assert plugin.ssa_db_b200_load_memory(len(seqs), b"".join(seqs),
                                          offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))) == 0
    assert [r[1] for r in _records(plugin)] == seqs


def _cuda_device_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


def test_search_without_device_fails_loudly(built_library, tmp_path):
    if _cuda_device_present():
        pytest.skip("a CUDA device is present")
    prog = (
        "import libssa_b200 as L\n"
        "L.load(); L.set_output_mode(L.OUTPUT_ERROR)\n"
        "L.init_symbol_translation(L.AMINOACID, L.FORWARD_STRAND, 1, 1)\n"
        "L.init_score_matrix(L.MATRIX_BUILDIN, 'blosum62'); L.init_gap_penalties(-11, -1)\n"
        "L.load_db_memory([b'ACDEFGHIK', b'MKVLL'])\n"
        "q = L.init_sequence_fasta(L.READ_FROM_STRING, 'ACDEF')\n"
        "L.sw_align(q, 2, L.BIT_WIDTH_8, L.COMPUTE_SCORE)\n"
        "print('searched without a device')\n")
    env = dict(os.environ, PYTHONPATH=ROOT)
    res = subprocess.run([sys.executable, "-c", prog], capture_output=True, text=True, env=env, timeout=300)
    assert res.returncode != 0
    assert "searched without a device" not in res.stdout
    assert res.stderr.strip()
