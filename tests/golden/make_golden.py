"""Generates the golden fixtures under tests/golden/ from the reference itself.

    python tests/golden/make_golden.py --reference REFERENCE_ROOT

Needs the reference sources (to build oracle/_ref/ref_run and to copy the FASTA
fixtures of its own test suite).  Writes:

* ``data/*``        -- the reference test-suite files the known-answer tests
  read (copied unchanged from the reference's tests/testdata/);
* ``matrices.json`` -- the reference's 32x32 score tables of every built-in
  matrix, of constant scoring and of the file matrices in data/;
* ``genetic_codes.json`` -- the reference's amino acid for every nucleotide
  triple under each genetic code (ref_run --dump-translation);
* ``frame_cases.json`` -- searches of query strands and translated query
  frames with the reference's complete answer, strand and frame fields included;
* ``abi_layout.json`` -- sizes, field offsets and constants of the
  reference's libssa.h / libssa_extern_db.h as its compiler sees them
  (tests/c_client/abi_layout.c built against the reference's headers);
* ``wide_cases.json`` and ``data/wide_scores.txt`` -- score-only searches
  with a score-matrix file whose 64-bit values leave the int32 range;
* ``cases.json``    -- seeded synthetic search cases (inputs stored inline, or
  regenerated from libssa_b200.workloads with the stored seed and checked by
  hash) with the reference's complete answer: hit IDs, scores, CIGARs,
  coordinates and overflow counts, at the 1-thread AVX2 or SSE settings.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from libssa_b200 import workloads as W  # noqa: E402

DATA_FILES = ["AF091148.fas", "one_seq.fas", "NP_009305.1.fas", "test.fas", "short_db.fas", "tmp.fas",
              "short_AA.fas", "short_nuc_db.fas", "blosum90.txt", "nuc_scoring_matrix.txt", "test_16_seq.fas",
              "AF091148_selection.fas", "one_seq_db.fas", "test2.fas"]

BUILTINS = ["blosum45", "blosum50", "blosum62", "blosum80", "blosum90", "pam30", "pam70", "pam250"]


def digest(queries: list[bytes], flat: np.ndarray, offsets: np.ndarray) -> str:
    h = hashlib.sha256()
    for q in queries:
        h.update(q + b"\0")
    h.update(np.ascontiguousarray(offsets, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(flat, dtype=np.uint8).tobytes())
    return h.hexdigest()


def run_case(case: dict, queries: list[bytes], records: list[bytes], tmp: str) -> list[dict]:
    db = os.path.join(tmp, "db.sdb")
    oracle.write_sdb(db, seqs=records)
    return oracle.run_reference(db, [q.decode() for q in queries], algo=case["algo"], width=case["width"],
                                align=case["align"], hits=case["hits"], symtype=case["symtype"],
                                matrix=case["matrix"], gap=tuple(case["gap"]), chunk=case["chunk"],
                                simd=case["simd"])


def synthetic_cases() -> list[tuple[dict, list[bytes], list[bytes], bool]]:
    """(case, queries, records, store_inline)."""
    out = []
    # config-shaped cases
    w = W.sw_plain(seed=1, scale=1.0)
    out.append(({"name": "sw_plain_full", "workload": "sw_plain", "seed": 1, "scale": 1.0}, w, False))
    w = W.sw_plain(seed=11, scale=0.2)
    out.append(({"name": "sw_plain_small", "workload": "sw_plain", "seed": 11, "scale": 0.2}, w, False))
    w = W.nw_nucleotide(seed=12, scale=0.005, n_queries=4)
    out.append(({"name": "nw_nucleotide_small", "workload": "nw_nucleotide", "seed": 12, "scale": 0.005,
                 "n_queries": 4}, w, False))
    w = W.sw_batched(seed=13, scale=0.004, n_queries=1024, n_db=500_000)
    out.append(({"name": "sw_batched_small", "workload": "sw_batched", "seed": 13, "scale": 0.004}, w, False))
    cases = []
    for meta, w, inline in out:
        case = dict(meta)
        case.update({"algo": w.algo, "width": w.bit_width, "align": 1, "hits": w.hitcount, "symtype": w.symtype,
                     "matrix": w.matrix, "gap": list(w.gap), "chunk": 1000, "simd": 2})
        case["digest"] = digest(w.queries, w.db_flat, w.db_offsets)
        cases.append((case, w.queries, w.db_records(), inline))

    # tie- and overflow-heavy small cases across widths, schedules and chunking
    rng = np.random.default_rng(2024)
    k = 0
    for algo in ("sw", "nw"):
        for width in (8, 16, 64):
            for simd in (2, 1):
                if width == 8 and simd == 0:
                    continue
                nuc = bool(k % 2)
                alpha = W.NT4 if nuc else W.AA20
                qlen = int(rng.integers(20, 300))
                q = W.random_residues(rng, qlen, alpha)
                recs = []
                for i in range(int(rng.integers(60, 400))):
                    r = rng.random()
                    if r < 0.15:
                        recs.append(W.mutate(rng, q, alpha, 0.05, 0.02, (1, 4)))
                    elif r < 0.2:
                        recs.append(W.mutate(rng, np.tile(q, 3), alpha, 0.01, 0.0, (1, 1)))
                    elif r < 0.22:
                        recs.append(np.zeros(0, np.uint8))
                    else:
                        recs.append(W.random_residues(rng, int(rng.integers(1, 400)), alpha))
                if nuc:
                    matrix = "const:%d,%d" % (int(rng.integers(1, 6)), -int(rng.integers(1, 6)))
                else:
                    matrix = "builtin:" + ["blosum62", "blosum50", "pam250", "blosum90"][k % 4]
                case = {"name": f"mixed_{algo}_{width}_{simd}", "algo": algo, "width": width, "align": 1,
                        "hits": int(rng.integers(3, 15)), "symtype": 0 if nuc else 1, "matrix": matrix,
                        "gap": [-int(rng.integers(1, 13)), -int(rng.integers(1, 3))],
                        "chunk": int([1000, 50, 17, 1][k % 4]), "simd": simd}
                recs_b = [r.tobytes() for r in recs]
                case["digest"] = digest([q.tobytes()], np.frombuffer(b"".join(recs_b), np.uint8),
                                        np.concatenate([[0], np.cumsum([len(r) for r in recs_b])]).astype(np.uint64))
                cases.append((case, [q.tobytes()], recs_b, True))
                k += 1
    return cases


def frame_cases() -> list[tuple[dict, list[bytes], list[bytes]]]:
    """Searches with query strands or translated query frames: nucleotide
    queries on the forward, complementary and both strands, and translated
    queries (3 or 6 frames, several genetic codes) against protein sequences."""
    rng = np.random.default_rng(77)
    out = []
    k = 0
    for symtype, strands_list in ((0, (1, 2, 3)), (2, (1, 2, 3))):
        for strands in strands_list:
            for algo, width, simd in (("sw", 8, 2), ("nw", 16, 1), ("sw", 64, 2), ("sw", 16, 2)):
                qlen = int(rng.integers(30, 400))
                q = W.random_residues(rng, qlen, W.NT4)
                if symtype == 0:
                    alpha = W.NT4
                    src = q
                else:
                    alpha = W.AA20
                    # protein records, some of them translations-like copies
                    src = W.random_residues(rng, max(10, qlen // 3), W.AA20)
                recs = []
                for i in range(int(rng.integers(40, 250))):
                    r = rng.random()
                    if r < 0.12:
                        recs.append(W.mutate(rng, src, alpha, 0.05, 0.02, (1, 3)))
                    elif r < 0.15:
                        recs.append(W.mutate(rng, np.tile(src, 4), alpha, 0.01, 0.0, (1, 1)))
                    elif r < 0.17:
                        recs.append(np.zeros(0, np.uint8))
                    else:
                        recs.append(W.random_residues(rng, int(rng.integers(1, 500)), alpha))
                if symtype == 0:
                    matrix = "const:%d,%d" % (int(rng.integers(1, 6)), -int(rng.integers(1, 6)))
                    gencode = [1, 1]
                else:
                    matrix = "builtin:" + ["blosum62", "pam30"][k % 2]
                    gencode = [[1, 1], [2, 1], [11, 1], [5, 1]][k % 4]
                case = {"name": f"frames_{symtype}_{strands}_{algo}_{width}", "algo": algo, "width": width,
                        "align": 1, "hits": int(rng.integers(3, 14)), "symtype": symtype, "strands": strands,
                        "gencode": gencode, "matrix": matrix,
                        "gap": [-int(rng.integers(1, 13)), -int(rng.integers(1, 3))],
                        "chunk": int([1000, 40, 7][k % 3]), "simd": simd}
                out.append((case, [q.tobytes()], [r.tobytes() for r in recs]))
                k += 1
    # translated queries against copies of their own frames' translations, so
    # that 8-bit lanes overflow in several frames of the same chunk
    with open(os.path.join(HERE, "genetic_codes.json")) as f:
        table = json.load(f)["1"]
    nt_code = {c: i for i, c in enumerate("-ACMGRSVTWYHKDBN")}
    compl = {"A": "T", "C": "G", "G": "C", "T": "A"}
    aa = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ"
    for strands, algo, width in ((3, "sw", 8), (1, "sw", 8), (2, "nw", 8)):
        q = W.random_residues(rng, 240, W.NT4).tobytes().decode()
        frames = []
        for st in (0, 1):
            seq = q if st == 0 else "".join(compl[c] for c in reversed(q))
            for fr in range(3):
                codes = [nt_code[c] for c in seq[fr:]]
                frames.append("".join(aa[table[(codes[i] << 8) | (codes[i + 1] << 4) | codes[i + 2]]]
                                      for i in range(0, len(codes) - 2, 3)).replace("*", "W"))
        recs = []
        for i in range(160):
            r = rng.random()
            fr = frames[int(rng.integers(0, 6))]
            src = np.frombuffer(fr.encode(), np.uint8)
            if r < 0.2:
                recs.append(W.mutate(rng, np.tile(src, 3), W.AA20, 0.02, 0.0, (1, 1)))
            elif r < 0.3:
                recs.append(W.mutate(rng, src, W.AA20, 0.05, 0.02, (1, 3)))
            else:
                recs.append(W.random_residues(rng, int(rng.integers(5, 300)), W.AA20))
        case = {"name": f"frames_ovf_2_{strands}_{algo}_{width}", "algo": algo, "width": width, "align": 1,
                "hits": 12, "symtype": 2, "strands": strands, "gencode": [1, 1], "matrix": "builtin:blosum62",
                "gap": [-11, -1], "chunk": 25, "simd": 2}
        out.append((case, [q.encode()], [r.tobytes() for r in recs]))
    return out


def write_frame_cases() -> None:
    import tempfile
    res_all = []
    with tempfile.TemporaryDirectory() as tmp:
        for case, queries, records in frame_cases():
            db = os.path.join(tmp, "db.sdb")
            oracle.write_sdb(db, seqs=records)
            res = oracle.run_reference(db, [q.decode() for q in queries], algo=case["algo"], width=case["width"],
                                       align=case["align"], hits=case["hits"], symtype=case["symtype"],
                                       strands=case["strands"], gencode=tuple(case["gencode"]),
                                       matrix=case["matrix"], gap=tuple(case["gap"]), chunk=case["chunk"],
                                       simd=case["simd"])
            case = dict(case)
            case["queries"] = [q.decode() for q in queries]
            case["records"] = [r.decode() for r in records]
            case["expected"] = [{"ovf8": r["ovf8"], "ovf16": r["ovf16"],
                                 "hits": [[h["id"], h["score"], h["cigar"], h["q_start"], h["q_end"], h["d_start"],
                                           h["d_end"], h["strand"], h["frame"], h["qstrand"], h["qframe"]]
                                          for h in r["hits"]]} for r in res]
            res_all.append(case)
            print(case["name"], "records", len(records))
    with open(os.path.join(HERE, "frame_cases.json"), "w") as f:
        json.dump(res_all, f, indent=0)


def write_genetic_codes() -> None:
    """The reference's translation of every nucleotide triple, per genetic code."""
    import subprocess
    codes = {}
    for gc in [1, 2, 3, 4, 5, 6, 9, 10, 11, 12, 13, 14, 15, 16, 21, 22, 23]:
        out = subprocess.run([oracle.REF_RUN, "--dump-translation", str(gc)], check=True, capture_output=True,
                             text=True).stdout
        codes[str(gc)] = json.loads(out)
    with open(os.path.join(HERE, "genetic_codes.json"), "w") as f:
        json.dump(codes, f)


def write_abi_layout(reference: str) -> None:
    import subprocess
    import tempfile
    src = os.path.join(os.path.dirname(HERE), "c_client", "abi_layout.c")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "abi_layout")
        subprocess.run(["gcc", "-I" + os.path.join(reference, "src"), "-o", exe, src], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    layout = json.loads(out)
    with open(os.path.join(HERE, "abi_layout.json"), "w") as f:
        json.dump(layout, f, indent=1)


WIDE_MATRIX = "wide_scores.txt"
WIDE_SCALE = 100_000_007


def write_wide_matrix(data: str) -> None:
    """A score-matrix file in the reference's text format with BLOSUM62's
    entries times 100,000,007: 64-bit scores far outside the int32 range, and
    8/16-bit truncations that scramble the table (the reference's lanes use
    them as they come, src/matrices.c:351-380)."""
    with open(os.path.join(HERE, "matrices.json")) as f:
        b62 = json.load(f)["blosum62"]
    sym = "ARNDCQEGHILKMFPSTWYVBZX*"
    aa = "-ABCDEFGHIKLMNPQRSTVWXYZU*OJ"
    with open(os.path.join(data, WIDE_MATRIX), "w") as f:
        f.write("# BLOSUM62 x %d\n" % WIDE_SCALE)
        f.write("   " + "  ".join(sym) + "\n")
        for a in sym:
            row = [b62[(aa.index(a) << 5) + aa.index(b)] * WIDE_SCALE for b in sym]
            f.write(a + " " + " ".join(str(v) for v in row) + "\n")


def wide_cases() -> list[tuple[dict, list[bytes], list[bytes]]]:
    """Score-only searches whose 64-bit values leave the int32 range: the
    64-bit entry and the 8->16->64 / 16->64 cascades, SW and NW."""
    rng = np.random.default_rng(4242)
    out = []
    for algo, width, chunk in (("sw", 64, 1000), ("nw", 64, 37), ("sw", 8, 50), ("nw", 16, 1000), ("sw", 16, 13)):
        q = W.random_residues(rng, int(rng.integers(150, 420)), W.AA20)
        recs = []
        for i in range(int(rng.integers(90, 160))):
            r = rng.random()
            if r < 0.15:
                recs.append(W.mutate(rng, q, W.AA20, 0.05, 0.02, (1, 4)))
            elif r < 0.18:
                recs.append(np.zeros(0, np.uint8))
            else:
                recs.append(W.random_residues(rng, int(rng.integers(1, 700)), W.AA20))
        case = {"name": f"wide_{algo}_{width}", "algo": algo, "width": width, "align": 0, "hits": 12, "symtype": 1,
                "matrix": "file:" + WIDE_MATRIX, "gap": [-11, -1], "chunk": chunk, "simd": 2}
        out.append((case, [q.tobytes()], [r.tobytes() for r in recs]))
    return out


def write_wide_cases() -> None:
    import tempfile
    data = os.path.join(HERE, "data")
    write_wide_matrix(data)
    res_all = []
    with tempfile.TemporaryDirectory() as tmp:
        for case, queries, records in wide_cases():
            db = os.path.join(tmp, "db.sdb")
            oracle.write_sdb(db, seqs=records)
            res = oracle.run_reference(db, [q.decode() for q in queries], algo=case["algo"], width=case["width"],
                                       align=case["align"], hits=case["hits"], symtype=case["symtype"],
                                       matrix="file:" + os.path.join(data, WIDE_MATRIX), gap=tuple(case["gap"]),
                                       chunk=case["chunk"], simd=case["simd"])
            case = dict(case)
            case["queries"] = [q.decode() for q in queries]
            case["records"] = [r.decode() for r in records]
            case["expected"] = [{"ovf8": r["ovf8"], "ovf16": r["ovf16"],
                                 "hits": [[h["id"], h["score"], h["cigar"], h["q_start"], h["q_end"], h["d_start"],
                                           h["d_end"]] for h in r["hits"]]} for r in res]
            res_all.append(case)
            print(case["name"], "records", len(records), "top", case["expected"][0]["hits"][:2])
    with open(os.path.join(HERE, "wide_cases.json"), "w") as f:
        json.dump(res_all, f, indent=0)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("SSA_REFERENCE_ROOT"), required="SSA_REFERENCE_ROOT" not in os.environ,
                    help="root of the reference source tree (default: $SSA_REFERENCE_ROOT)")
    ap.add_argument("--abi-only", action="store_true", help="only regenerate abi_layout.json")
    ap.add_argument("--frames-only", action="store_true",
                    help="only regenerate frame_cases.json and genetic_codes.json")
    ap.add_argument("--wide-only", action="store_true",
                    help="only regenerate wide_cases.json (and its matrix file)")
    args = ap.parse_args()
    if args.wide_only:
        oracle.build(args.reference)
        write_wide_cases()
        return
    write_abi_layout(args.reference)
    if args.abi_only:
        return
    oracle.build(args.reference)
    write_genetic_codes()
    write_frame_cases()
    if args.frames_only:
        return
    data = os.path.join(HERE, "data")
    os.makedirs(data, exist_ok=True)
    for f in DATA_FILES:
        shutil.copyfile(os.path.join(args.reference, "tests", "testdata", f), os.path.join(data, f))

    mats = {name: oracle.reference_matrix("builtin:" + name).tolist() for name in BUILTINS}
    mats["const:5,-4"] = oracle.reference_matrix("const:5,-4").tolist()
    mats["const:127,-128"] = oracle.reference_matrix("const:127,-128").tolist()
    mats["file:blosum90.txt"] = oracle.reference_matrix("file:" + os.path.join(data, "blosum90.txt")).tolist()
    mats["file:nuc_scoring_matrix.txt"] = oracle.reference_matrix(
        "file:" + os.path.join(data, "nuc_scoring_matrix.txt")).tolist()
    with open(os.path.join(HERE, "matrices.json"), "w") as f:
        json.dump(mats, f)

    import tempfile
    out = []
    with tempfile.TemporaryDirectory() as tmp:
        for case, queries, records, inline in synthetic_cases():
            res = run_case(case, queries, records, tmp)
            case = dict(case)
            case["expected"] = [{"ovf8": r["ovf8"], "ovf16": r["ovf16"],
                                 "hits": [[h["id"], h["score"], h["cigar"], h["q_start"], h["q_end"], h["d_start"],
                                           h["d_end"]] for h in r["hits"]]} for r in res]
            if inline:
                case["queries"] = [q.decode() for q in queries]
                case["records"] = [r.decode() for r in records]
            out.append(case)
            print(case["name"], "queries", len(queries), "records", len(records))
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(out, f, indent=0)
    write_wide_cases()


if __name__ == "__main__":
    main()
