"""Known-answer tests of the reference's own test suite, restated as data.

Each entry names the reference test it comes from.  The reference drives many
of them through internal calls (s_search with adp_init(hit_count)); here they
go through the public API with the same settings: the chunk size equals the
hit count, gap penalties are set with init_gap_penalties, constant scoring
with init_constant_scores(match, mismatch) and the SIMD capability with
set_simd_compute_mode.  Expected values are copied from the cited lines.
"""

HPEVY = "HPEVYILIIPGFGIISHVVSTYSKKPVFGEISMVYAMASIGLLGFLVWSHHMYIVGLDADTRAYFTSATMIIAIPTGIKI"

NP_QUERY = (
    "MVQRWLYSTNAKDIAVLYFMLAIFSGMAGTAMSLIIRLELAAPGSQYLHGNSQLFNVLVVGHAVLMIFFLVMPALIGGFG"
    "NYLLPLMIGATDTAFPRINNIAFWVLPMGLVCLVTSTLVESGAGTGWTVYPPLSSIQAHSGPSVDLAIFALHLTSISSLL"
    "GAINFIVTTLNMRTNGMTMHKLPLFVWSIFITAFLLLLSLPVLSAGITMLLLDRNFNTSFFEVSGGGDPILYEHLFWFFG"
    "HPEVYILIIPGFGIISHVVSTYSKKPVFGEISMVYAMASIGLLGFLVWSHHMYIVGLDADTRAYFTSATMIIAIPTGIKI"
    "FSWLATIHGGSIRLATPMLYAIAFLFLFTMGGLTGVALANASLDVAFHDTYYVVGHFHYVLSMGAIFSLFAGYYYWSPQI"
    "LGLNYNEKLAQIQFWLIFIGANVIFFPMHFLGINGMPRRIPDYPDAFAGWNYVASIGSFIATLSLFLFIYILYDQLVNGL"
    "NNKVNNKSVIYNKAPDFVESNTIFNLNTVKSSSIEFLLTSPPAVHSFNTPAVQS")


def _pairs(flat):
    return [(flat[i], flat[i + 1]) for i in range(0, len(flat), 2)]


# Each KAT: db file, query (("file", name) or ("string", text)), settings and
# a list of calls (algo, width, align, hits, simd, expected) where expected
# is {"hits": [(score, id[, cigar])...], "ovf": (n8, n16) or None}.
KATS = [
    {
        "source": "tests/test_libssa.c:30-93 (test_simple_one_thread)",
        "db": "AF091148.fas", "query": ("file", "one_seq.fas"), "symtype": 0,
        "matrix": ("const", 5, -4), "gap": (-4, -2), "chunk": 1000,
        "calls": [
            ("sw", 64, 1, 5, 2, {"hits": [
                (91, 877, "2MD2MIM2I3MD3MD4M2D8M5I3M5IM3I7MI7M3I5MI3M"),
                (91, 847, "2MD2MIM2I3MD3MD4M2D8M5I3M5IM3I7MI7M3I4MI4M"),
                (91, 753, "2MD2MIM2I3MD3MD3M2D9M5I3M5IM3I7MI7M3I5MI3M"),
                (91, 565, "2MD2MIM2I3MD3MD4M2D8M5I3M5IM3I7MI7M3I5MI3M"),
                (91, 398, "2MD2MIM2I3MD3MD3M2D9M5I3M5IM3I7MI7M3I5MI3M")], "ovf": None}),
            ("nw", 64, 1, 5, 2, {"hits": [
                (33, 1050, "2MI2MI6M3I6MD3M19I4M3IMI3M5I3M5IM3I7MI7M4IMIMI4MI2M7I"),
                (28, 908, "2MI2MI6M3I6MD3M5IM2I2M3I2M5IMI9MD2M3I3M9I2M3I2M4I2M2IMI4MI2M7I"),
                (24, 938, "2MI2MI6M3I6MD3M5IM2I2M3I2M5IMI9MD2M3I3M9I2M3I2M4IM3IMIMIM2I5M10I"),
                (21, 378, "2MI2MI6M3I5M9I2M7IM6IMI3M3I6M5I3M5IM3I7MI7M4IMIMI4MI2M7I"),
                (12, 75, "2MI2MI6M3I5M9I2M7IM6IMI3M3I6M5I3M5IM3I7MI7M4IMIMI4MI2M7I")], "ovf": None}),
        ],
    },
    {
        "source": "tests/test_bigger_databases.c:70-92 (test_AF091148)",
        "db": "AF091148.fas", "query": ("file", "one_seq.fas"), "symtype": 0,
        "matrix": ("const", 2, -2), "gap": (-4, -2), "chunk": 1000,
        "calls": [
            (algo, w, 0, 10, 2, {"hits": _pairs(exp), "ovf": None})
            for algo, exp in (
                ("nw", [-88, 908, -92, 1050, -94, 938, -98, 378, -102, 75, -104, 23, -106, 1229, -110, 1148,
                        -110, 612, -112, 1016]),
                ("sw", [20, 1177, 18, 384, 18, 277, 18, 215, 18, 214, 18, 210, 18, 151, 18, 126, 18, 114, 18,
                        101]))
            for w in (64, 16, 8)
        ],
    },
    {
        "source": "tests/algo/test_searcher.c:144-227 (multiple sequences)",
        "db": "short_nuc_db.fas", "query": ("string", "ATGCAAATTT"), "symtype": 0,
        "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 8,
        "calls": [
            (algo, w, 0, 8, simd, {"hits": _pairs(exp), "ovf": None})
            for algo, exp in (("nw", [-1, 0, -3, 3, -4, 7, -4, 6, -4, 4, -5, 2, -6, 5, -6, 1]),
                              ("sw", [4, 3, 4, 1, 4, 0, 3, 7, 3, 5, 3, 4, 3, 2, 2, 6]))
            for w, simd in ((64, 2), (16, 1), (16, 2), (8, 1), (8, 2))
        ],
    },
    {
        "source": "tests/algo/test_searcher.c:376-404 (test_searcher_AA_nw_8 / _sw_8)",
        "db": "short_AA.fas", "query": ("string", HPEVY), "symtype": 1,
        "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 1,
        "calls": [("nw", 8, 0, 1, 1, {"hits": [(-87, 0)], "ovf": None}),
                  ("sw", 8, 0, 1, 1, {"hits": [(3, 0)], "ovf": None})],
    },
    {
        "source": "tests/algo/test_searcher.c:406-505 (BLOSUM62)",
        "db": "short_AA.fas", "query": ("string", HPEVY), "symtype": 1,
        "matrix": ("builtin", "blosum62"), "gap": (-1, -1), "chunk": 1,
        "calls": [
            ("sw", 64, 0, 1, 2, {"hits": [(103, 0)], "ovf": None}),
            ("nw", 64, 0, 1, 2, {"hits": [(82, 0)], "ovf": None}),
            ("sw", 16, 0, 1, 0, {"hits": [(103, 0)], "ovf": None}),
            ("nw", 16, 0, 1, 0, {"hits": [(82, 0)], "ovf": None}),
            ("sw", 8, 0, 1, 1, {"hits": [(103, 0)], "ovf": None}),
            ("sw", 8, 0, 1, 2, {"hits": [(103, 0)], "ovf": None}),
            ("nw", 8, 0, 1, 1, {"hits": [(82, 0)], "ovf": None}),
        ],
    },
    {
        "source": "tests/algo/test_searcher.c:507-546 (overflow to 64 bit)",
        "db": "NP_009305.1.fas", "query": ("file", "NP_009305.1.fas"), "symtype": 1,
        "matrix": ("const", 127, -1), "gap": (-1, -1), "chunk": 1,
        "calls": [("sw", 8, 0, 1, 2, {"hits": [(67818, 0)], "ovf": (1, 1)}),
                  ("nw", 8, 0, 1, 2, {"hits": [(67818, 0)], "ovf": (1, 1)})],
    },
    {
        "source": "tests/algo/8/test_8_simd_avx2_sw.c:67-92 (simple)",
        "db": "short_db.fas", "query": ("string", "AT"), "symtype": 0,
        "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 1,
        "calls": [("sw", 8, 0, 1, 2, {"hits": [(2, 0)], "ovf": None})],
    },
    {
        "source": "tests/algo/8/test_8_simd_avx2_sw.c:94-115 (simple 2)",
        "db": "tmp.fas", "query": ("string", "ATGCAAA"), "symtype": 0,
        "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 1,
        "calls": [("sw", 8, 0, 1, 2, {"hits": [(4, 0)], "ovf": None})],
    },
    {
        "source": "tests/algo/8/test_8_simd_avx2_sw.c:117-141 (overflow)",
        "db": "NP_009305.1.fas", "query": ("string", NP_QUERY), "symtype": 1,
        "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 1,
        "calls": [("sw", 8, 0, 1, 2, {"hits": [(534, 0)], "ovf": (1, 0)})],
    },
    {
        "source": "tests/algo/8/test_8_simd_avx2_sw.c:143-160 (more sequences)",
        "db": "test.fas", "query": ("string", "ATGCCCAAGCTGAATAGCGTAGAGGGGTTTTCATCATTTGAGGACGATGTATAA"),
        "symtype": 0, "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 5,
        "calls": [("sw", 8, 0, 5, 2, {"hits": [(8, 4), (8, None), (8, None), (8, None), (8, None)],
                                      "ovf": None})],
    },
    {
        "source": "tests/algo/8/test_8_simd_avx2_nw.c:60-69 (simple)",
        "db": "short_db.fas", "query": ("string", "AT"), "symtype": 0,
        "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 1,
        "calls": [("nw", 8, 0, 1, 2, {"hits": [(-2, None)], "ovf": None})],
    },
    {
        "source": "tests/algo/8/test_8_simd_avx2_nw.c:71-88 (more sequences)",
        "db": "test.fas", "query": ("string", "ATGCCCAAGCTGAATAGCGTAGAGGGGTTTTCATCATTTGAGGACGATGTATAA"),
        "symtype": 0, "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 5,
        "calls": [("nw", 8, 0, 5, 2, {"hits": [(-43, None), (-50, None), (-52, None), (-52, None),
                                               (-147, None)], "ovf": (4, 0)})],
    },
]


def matches(expected: dict, hits: list[tuple], ovf: tuple[int, int] | None) -> bool:
    """hits: [(score, id, cigar)] in result order."""
    exp = expected["hits"]
    if len(exp) != len(hits):
        return False
    for e, h in zip(exp, hits):
        if e[0] != h[0]:
            return False
        if len(e) > 1 and e[1] is not None and e[1] != h[1]:
            return False
        if len(e) > 2 and e[2] != h[2]:
            return False
    if expected["ovf"] is not None and ovf is not None and tuple(expected["ovf"]) != tuple(ovf):
        return False
    return True

KATS.append({
    # tests/algo/test_searcher.c:247-325 (test_searcher_translate_*): a nucleotide
    # query translated in 6 frames (genetic code 3) against one protein sequence,
    # constant scores 1/-1, gaps 1/1, chunk = hit count = 6; the heap, sorted,
    # holds one entry per frame
    "source": "tests/algo/test_searcher.c:247-325 (test_searcher_translate)",
    "db": "short_AA.fas", "query": ("string", "ATGCCCAAAATTGACTTGAATAGGGGCGTGAGGAGGGGTTTTCAATACTATTTTTTG"),
    "symtype": 2, "strands": 3, "gencode": (3, 3),
    "matrix": ("const", 1, -1), "gap": (-1, -1), "chunk": 6,
    "calls": [
        (algo, w, 0, 6, simd, {"hits": [(s, 0) for s in exp], "ovf": None})
        for w, simd in ((64, 2), (16, 0), (8, 1))
        for algo, exp in (("nw", [-109, -109, -110, -110, -110, -113]), ("sw", [2, 2, 2, 2, 2, 1]))
    ],
})
