"""The learned lookahead proposal: GPU kernels against the CPU restatement of the
network, training on the GPU, and the engine's output unchanged by it."""
import os

import numpy as np
import pytest

import tensorfim_b200 as tf
from tensorfim_b200 import learn, synth
from conftest import golden_input, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mlp_oracle():
    from oracle import mlp_oracle
    return mlp_oracle


def _data(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.normal(0, 1, size=(n, 32)).astype(np.float32)
    w = rng.normal(0, 1, size=32)
    y = (x @ w + 0.3 * rng.normal(size=n) > 0.5).astype(np.float32)
    return x, y


def test_forward_matches_cpu_restatement(mlp_oracle):
    prop = learn.Proposal(seed=3)
    x, _ = _data(777, 1)
    got = prop.predict(x)
    exp = mlp_oracle.predict(prop.params(), x)
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-5)   # FP32 accumulation order differs


@pytest.mark.parametrize("pos_weight", [1.0, 7.5])
def test_gradients_match_cpu_restatement(mlp_oracle, pos_weight):
    prop = learn.Proposal(seed=5)
    x, y = _data(300, 2)    # not a multiple of the 64-sample block
    g, loss = prop.grad(x, y, pos_weight)
    g_ref, loss_ref = mlp_oracle.grad(prop.params(), x, y, pos_weight)
    assert loss == pytest.approx(loss_ref, rel=1e-4)
    scale = np.abs(g_ref).max()
    np.testing.assert_allclose(g, g_ref, rtol=2e-3, atol=2e-5 * scale)


def test_training_on_gpu_learns(mlp_oracle):
    prop = learn.Proposal(seed=7)
    x, y = _data(4096, 3)
    before = mlp_oracle.grad(prop.params(), x, y)[1]
    prop.train(x, y, epochs=30, batch=256, lr=3e-3, pos_weight=1.0)
    after = mlp_oracle.grad(prop.params(), x, y)[1]
    acc = ((prop.predict(x) >= 0.5) == (y > 0.5)).mean()
    assert after < 0.5 * before and acc > 0.9


@pytest.mark.parametrize("name", ["cfg1_full", "cfg1_t03", "cfg5_s002", "edge_ties", "cfg4_s001"])
def test_learned_lookahead_keeps_output_identical(tmp_path, name):
    """Any network (here an untrained one, and the shipped one when present) leaves the
    MFI set unchanged: it only orders exact checks."""
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    props = [learn.Proposal(seed=11)]
    if os.path.exists(learn.WEIGHTS):
        props.append(learn.Proposal.load())
    with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
        for prop in props:
            for thr in (0.0, 0.5, 1.01):
                db.set_proposal(prop, thr)
                assert db.mine(lookahead="learned").as_dict() == fx["expected"]
                assert db.mine(engine="resident", lookahead="learned").as_dict() == fx["expected"]


@pytest.mark.parametrize("engine", ["batched", "resident"])
def test_lookahead_log_records_outcomes(tmp_path, engine):
    fx = load_golden("cfg1_full")
    path = golden_input(fx, tmp_path)
    with tf.Database.from_file(path, 0.10) as db:
        r = db.mine(engine=engine, lookahead="filtered", log_lookahead=True)
        x, y = db.lookahead_log()
        assert x.shape == (r.stats["lookaheads"], 32)
        assert int(y.sum()) == r.stats["lookahead_hits"]
        assert np.isfinite(x).all()


@pytest.mark.slow
@pytest.mark.skipif(not os.path.exists(learn.WEIGHTS), reason="trained weights not present")
def test_learned_proposal_gain_on_cfg5():
    """Evaluation database of the learned proposal (2,000,000 tx x 60 groups, minsup 70%):
    the trained network keeps the output identical to the plain engine and issues no more
    lookaheads that miss than the filtered policy."""
    db0 = synth.generate(5)
    with tf.Database.from_csr(db0.offsets, db0.items, 0.70) as db:
        plain = db.mine(engine="plain").as_dict()
        base = db.mine(lookahead="filtered")
        lrn = db.mine(lookahead="learned")
        assert lrn.as_dict() == plain and base.as_dict() == plain
        wasted_base = base.stats["lookaheads"] - base.stats["lookahead_hits"]
        wasted_lrn = lrn.stats["lookaheads"] - lrn.stats["lookahead_hits"]
        assert wasted_lrn <= wasted_base
        assert lrn.stats["supports"] <= base.stats["supports"]


@pytest.mark.slow
@pytest.mark.skipif(not os.path.exists(learn.WEIGHTS), reason="trained weights not present")
@pytest.mark.parametrize("cfg,kw,minsup", [(3, dict(replicas=1), 0.06), (4, dict(scale=0.25), 0.0005)])
def test_learned_proposal_strictly_beats_the_filter(cfg, kw, minsup):
    """Where lookaheads matter -- the replicated configuration's generator at 6% (40,760
    nodes) and the sparse configuration at a quarter of its rows -- the trained network
    issues strictly fewer lookaheads that miss than the tail-pair filter and the search
    counts strictly fewer supports, with the same MFIs as the plain engine."""
    db0 = synth.generate(cfg, **kw)
    with tf.Database.from_csr(db0.offsets, db0.items, minsup) as db:
        plain = db.mine(engine="plain").as_dict()
        base = db.mine(lookahead="filtered")
        lrn = db.mine(lookahead="learned")
        assert lrn.as_dict() == plain and base.as_dict() == plain
        wasted_base = base.stats["lookaheads"] - base.stats["lookahead_hits"]
        wasted_lrn = lrn.stats["lookaheads"] - lrn.stats["lookahead_hits"]
        assert wasted_lrn < wasted_base, (wasted_lrn, wasted_base)
        assert lrn.stats["supports"] < base.stats["supports"], (lrn.stats["supports"], base.stats["supports"])
