"""The command-line drop-in: same invocation, same results file, same header statistics."""
import os
import shutil

import pytest

import tensorfim_b200 as tf
from conftest import GOLDEN, golden_input, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cfg1_full", "cfg4_s001", "edge_item0", "edge_format", "edge_dups", "edge_none"])
@pytest.mark.parametrize("engine,lookahead,graphs", [("resident", 2, 1), ("resident", 1, 0), ("batched", 1, 0),
                                                     ("plain", 1, 0)])
def test_cli_results_file(tmp_path, name, engine, lookahead, graphs):
    fx = load_golden(name)
    src = golden_input(fx, tmp_path)
    path = str(tmp_path / os.path.basename(src))
    if src != path:
        shutil.copyfile(src, path)
    minsup = fx["spec"]["minsup"]
    r = tf.mine_file(path, minsup, engine=engine, lookahead=lookahead, graphs=graphs)
    assert r.returncode == 0, r.stderr
    res = tf.result_path(path, minsup)
    assert os.path.exists(res)
    assert tf.load_results(res) == fx["expected"]
    hdr = tf.load_header(res)
    for k in ["transNum", "dimension", "itemIDmin", "itemIDmax", "transLengthMin", "transLengthMax",
              "dimensionReduced", "transNumReduced", "transLengthReducedMin", "transLengthReducedMax", "MFIsNumber"]:
        assert hdr[k] == fx["header"][k], k
    for k in ["transLengthMean", "transLengthReducedMean"]:
        a, b = hdr[k], fx["header"][k]
        assert a == b or float(a) == pytest.approx(float(b), rel=1e-5), k
    assert "computation_time(s)" in hdr and "total_time(s)" in hdr
