"""The schedule table format of the autotuner (disort_b200/autotune.py), on CPU."""
import pytest

from disort_b200 import autotune


def test_table_round_trip_and_lookup(tmp_path):
    p = str(tmp_path / "t.txt")
    entries = [(16, 1, 24, 1, 128, 0), (16, 25, 60, 2, 0, 0), (64, 1, 1000000, 0, 0, 1)]
    autotune.write_table(p, entries, ["measured somewhere"])
    assert autotune.read_table(p) == entries
    assert autotune.lookup(entries, 16, 24) == entries[0]
    assert autotune.lookup(entries, 16, 25) == entries[1]
    assert autotune.lookup(entries, 64, 500) == entries[2]
    assert autotune.lookup(entries, 8, 10) == (8, 0, 0, 0, 0, 0)  # no entry: built-in choices


def test_table_rejects_malformed_lines(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("# comment\n16 1 24 1 128\n")
    with pytest.raises(ValueError, match="line 2"):
        autotune.read_table(str(p))


def test_candidates_cover_both_forms():
    stages = {c[0] for c in autotune.FLUX_CANDIDATES}
    assert stages == {1, 2} and {c[1] for c in autotune.FLUX_CANDIDATES if c[0] == 1} == {64, 128}
    assert set(autotune.GENERAL_CANDIDATES) == {1, 2}
