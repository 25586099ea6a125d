"""The tuning table (include/tfim.h tfim_tuning): defaults, set/get, file loading and range
checks.  No GPU needed: the table is host state of the library."""
import json
import os

import pytest

from tensorfim_b200 import engine
from tensorfim_b200._lib import TfimError

HERE = os.path.dirname(os.path.abspath(__file__))
SHIPPED = os.path.join(os.path.dirname(HERE), "tensorfim_b200", "tuning.json")


@pytest.fixture
def restore():
    saved = engine.tuning()
    yield saved
    engine.set_tuning(**saved)


def test_table_in_range(restore):
    t = restore
    assert 16 <= t["wave_rows"] <= (1 << 20)
    assert t["l3_slices_per_sm"] > 0 and t["b1_tiles_per_sm"] > 0
    assert t["b1_min_rows"] >= 1 and t["b1_min_cols"] >= 1
    assert t["rate_b1_bitops"] > 0 and t["rate_lop3_bitops"] > 0 and t["rate_pair_incr"] > 0
    src = engine.tuning_source()
    assert src == "built-in" or src.endswith("tuning.json") or src == "set by the caller"


def test_set_and_get(restore):
    engine.set_tuning(wave_rows=1234, l3_slices_per_sm=3.5, b1_min_rows=7)
    t = engine.tuning()
    assert (t["wave_rows"], t["l3_slices_per_sm"], t["b1_min_rows"]) == (1234, 3.5, 7)
    assert engine.tuning_source() == "set by the caller"


@pytest.mark.parametrize("bad", [dict(wave_rows=0), dict(wave_rows=1 << 21), dict(l3_slices_per_sm=0.0),
                                 dict(b1_tiles_per_sm=-1.0), dict(b1_min_cols=0), dict(proj_auto=2),
                                 dict(rate_pair_incr=0.0)])
def test_out_of_range_rejected(restore, bad):
    before = engine.tuning()
    with pytest.raises(TfimError):
        engine.set_tuning(**bad)
    assert engine.tuning() == before


def test_load_partial_file(restore, tmp_path):
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"wave_rows": 777, "b1_tiles_per_sm": 6.0, "sweep:wave_rows": [[1, 2]], "note": "x"}))
    before = engine.tuning()
    engine.load_tuning(str(p))
    t = engine.tuning()
    assert t["wave_rows"] == 777 and t["b1_tiles_per_sm"] == 6.0
    assert t["l3_slices_per_sm"] == before["l3_slices_per_sm"]
    assert engine.tuning_source() == str(p)


def test_bad_files_rejected(restore, tmp_path):
    before = engine.tuning()
    with pytest.raises(TfimError):
        engine.load_tuning(str(tmp_path / "missing.json"))
    p = tmp_path / "bad.json"
    p.write_text('{"wave_rows": "many"}')
    with pytest.raises(TfimError):
        engine.load_tuning(str(p))
    p.write_text('{"wave_rows": 3}')   # below the minimum of 16
    with pytest.raises(TfimError):
        engine.load_tuning(str(p))
    assert engine.tuning() == before


@pytest.mark.skipif(not os.path.exists(SHIPPED), reason="no tuning table committed")
def test_shipped_table_loads(restore):
    engine.load_tuning(SHIPPED)
    doc = json.load(open(SHIPPED))
    t = engine.tuning()
    for k in ("wave_rows", "b1_min_rows", "b1_min_cols", "proj_auto"):
        assert t[k] == doc[k]
    for k in ("l3_slices_per_sm", "b1_tiles_per_sm", "rate_b1_bitops", "rate_lop3_bitops", "rate_pair_incr"):
        assert t[k] == pytest.approx(doc[k], rel=1e-6)


def test_dense_slices_field(restore, tmp_path):
    """The dense families' word-slice target is a field of the table like the others: set,
    range-checked, loaded from a file, and shipped in the committed table."""
    assert restore["l3_dense_slices_per_sm"] > 0
    engine.set_tuning(l3_dense_slices_per_sm=48.0)
    assert engine.tuning()["l3_dense_slices_per_sm"] == 48.0
    for bad in (0.0, -1.0, 2048.0):
        with pytest.raises(TfimError):
            engine.set_tuning(l3_dense_slices_per_sm=bad)
    assert engine.tuning()["l3_dense_slices_per_sm"] == 48.0
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"l3_dense_slices_per_sm": 96.0}))
    engine.load_tuning(str(p))
    assert engine.tuning()["l3_dense_slices_per_sm"] == 96.0
    with open(SHIPPED) as f:
        shipped = json.load(f)
    assert shipped["l3_dense_slices_per_sm"] > 0 and shipped["gram_min_rows"] >= 1
