"""Genetic codes of translated searches, against the reference.

The translation tables of the build (NCBI genetic codes, with the reference's
rules for ambiguous IUPAC codes: one amino acid if all concrete codons agree,
B for D/N, Z for E/Q, X otherwise) must equal the reference's, which
tests/golden/genetic_codes.json holds for every genetic code it accepts
(oracle/_ref/ref_run --dump-translation).  Host code only: no device needed.
"""
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "genetic_codes.json")) as f:
    CODES = json.load(f)


@pytest.mark.parametrize("code", sorted(CODES, key=int))
def test_translation_table_matches_reference(built_library, code):
    import libssa_b200 as L
    assert L.translation_table(int(code)) == CODES[code]


def test_undefined_genetic_codes_are_refused(built_library):
    import libssa_b200 as L
    for code in (0, 7, 8, 17, 18, 19, 20, 26):
        with pytest.raises(ValueError):
            L.translation_table(code)
