"""The resident engine's superset check (a family whose head and tail lie inside an MFI
already found is dropped, at creation and before it leaves the stack) changes speed only:
with it on and off the MFI set and every support equal the reference engine's on every
golden fixture, under the host and the graph-driven wave loops and the lookahead modes, and
on larger generated databases."""
import pytest

import tensorfim_b200 as tf
from tensorfim_b200 import synth
from conftest import golden_input, golden_names, load_golden

pytestmark = pytest.mark.gpu

MODES = [dict(lookahead=True), dict(lookahead="learned"), dict(lookahead=False), dict(lookahead="all", wave_cap=29),
         dict(lookahead=True, graphs=True), dict(lookahead="learned", counter="lop3", top="bitmap")]


@pytest.mark.parametrize("name", golden_names())
def test_superset_check_keeps_the_reference_output(tmp_path, name):
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
        for m in MODES:
            for sup in (True, False):
                res = db.mine(engine="resident", superset=sup, **m)
                assert res.as_dict() == fx["expected"], (m, sup)
                assert len(res) == len(fx["expected"])
                if not sup:
                    assert res.stats["pruned_superset"] == 0


@pytest.mark.parametrize("cfg,kw,minsup", [(1, dict(scale=1.0), 0.05), (5, dict(scale=0.02), 0.6),
                                           (4, dict(scale=0.1), 0.001), (2, dict(scale=0.2), 0.8)])
def test_superset_check_on_generated_databases(cfg, kw, minsup):
    db0 = synth.generate(cfg, **kw)
    with tf.Database.from_csr(db0.offsets, db0.items, minsup) as db:
        exp = db.mine(engine="batched").as_dict()
        for la in (True, "learned"):
            on = db.mine(engine="resident", lookahead=la, superset=True)
            off = db.mine(engine="resident", lookahead=la, superset=False)
            assert on.as_dict() == exp and off.as_dict() == exp
            # a dropped family is never counted: the search with the check counts no more
            assert on.stats["nodes"] <= off.stats["nodes"]
