"""LAsort's CPU restatement (oracle/las_sort.py) against the reference LAsort's outputs
(tests/golden/lasort), bytes and pad words included, up to the order of tied keys."""
import os

import pytest

from marvel_b200 import dazzdb

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lasort")


@pytest.mark.parametrize("name", ["cat", "s200"])
def test_oracle_las_sort_matches_reference(name, tmp_path):
    import las_sort
    n = las_sort.las_sort(os.path.join(GOLD, name + ".las"), str(tmp_path / "o.las"))
    assert n > 100
    ok, msg = dazzdb.las_equal(str(tmp_path / "o.las"), os.path.join(GOLD, name + ".S.las"), key="lasort", pad=True)
    assert ok, msg
    # the input is not sorted: the check has teeth
    ok, _ = dazzdb.las_equal(os.path.join(GOLD, name + ".las"), os.path.join(GOLD, name + ".S.las"), key="lasort")
    assert not ok
