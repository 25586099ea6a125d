"""Full-size benchmark databases against the reference's own output: configurations 5
(2,000,000 transactions x 60 groups, minsup 70%) and 4 (1,000,000 transactions x 40,000
items, minsup 0.05%), opened from their text files (device parse) and mined by the resident
engine with the learned proposal, must give exactly the MFIs and frequencies of
tests/golden/full (produced by the reference's multithreaded CPU engine, make_golden.py)."""
import pytest

import tensorfim_b200 as tf
from conftest import golden_input, load_golden_full

pytestmark = pytest.mark.gpu


@pytest.mark.slow
@pytest.mark.parametrize("name", ["cfg5_full", "cfg4_full"])
def test_full_size_matches_reference_fixture(tmp_path, name):
    fx = load_golden_full(name)
    path = golden_input(fx, tmp_path)
    with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
        assert db.info["trans_num"] == int(fx["header"]["transNum"])
        assert db.info["dimension_reduced"] == int(fx["header"]["dimensionReduced"])
        assert db.mine(engine="resident", lookahead="learned").as_dict() == fx["expected"]
