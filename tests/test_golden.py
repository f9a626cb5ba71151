"""The known-answer fixture the oracle and host-model tests load
(tests/golden/known_answers.json): every value carries the reference file
and line it comes from, and -- when ORIGAMI_REFERENCE_DIR names a checkout
of the reference -- regenerating it from those sources gives the committed
file unchanged."""
from __future__ import annotations

import json
import os
import re
import sys

import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def committed():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def test_every_known_answer_cites_its_source():
    d = committed()
    assert len(d) >= 16
    for key, entry in d.items():
        assert set(entry) == {"value", "source", "note"}, key
        assert re.fullmatch(r"[\w./-]+:\d+", entry["source"]), (key, entry["source"])
        assert isinstance(entry["value"], (int, float)), key


@pytest.mark.skipif(not os.environ.get("ORIGAMI_REFERENCE_DIR"), reason="no reference checkout named")
def test_fixture_regenerates_from_the_reference():
    sys.path.insert(0, GOLDEN)
    import make_known_answers
    assert make_known_answers.extract(os.environ["ORIGAMI_REFERENCE_DIR"]) == committed()
