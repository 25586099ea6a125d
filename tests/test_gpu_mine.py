"""MFI search on the GPU: set-identical output with identical supports.

Every fixture of tests/golden (produced by the reference engine) is mined by the plain
engine and by the batched engine under each counter and with lookahead on and off.  At
full benchmark sizes, where the reference takes too long, the batched engine is checked
against the plain engine and by the reference's own MFI test (every reported set is
frequent and no single counted item extends it)."""
import numpy as np
import pytest

import tensorfim_b200 as tf
from tensorfim_b200 import synth
from conftest import golden_input, golden_names, load_golden

pytestmark = pytest.mark.gpu

VARIANTS = [
    dict(engine="batched", counter="auto", lookahead=True),
    dict(engine="batched", counter="lop3", lookahead=True),
    dict(engine="batched", counter="tensor", lookahead=True),
    dict(engine="batched", counter="auto", lookahead=False),
    dict(engine="batched", counter="tensor", lookahead=False, wave_cap=37),
    dict(engine="batched", counter="auto", lookahead=True, top="pairs"),
    dict(engine="batched", counter="lop3", lookahead=False, top="bitmap"),
    dict(engine="batched", counter="tensor", lookahead=True, top="bitmap"),
    dict(engine="resident", counter="auto", lookahead=True),
    dict(engine="resident", counter="lop3", lookahead=False, top="bitmap"),
    dict(engine="resident", counter="tensor", lookahead=True, top="bitmap"),
    dict(engine="resident", counter="auto", lookahead="all", wave_cap=37),
    dict(engine="resident", counter="auto", lookahead=True, top="pairs"),
    dict(engine="resident", counter="proj", lookahead="learned"),
    dict(engine="resident", counter="proj", lookahead="all", wave_cap=29),
    dict(engine="resident", counter="auto", lookahead=True, graphs=True),
    dict(engine="resident", counter="tensor", lookahead="all", wave_cap=37, graphs=True),
    dict(engine="resident", counter="lop3", lookahead="learned", top="bitmap", graphs=True),
    dict(engine="resident", counter="proj", lookahead="all", wave_cap=29, graphs=True),
    dict(engine="resident", counter="i8", lookahead="learned"),
    dict(engine="resident", counter="i8", lookahead="all", wave_cap=37, graphs=True),
    dict(engine="resident", counter="i8", lookahead=False, top="bitmap", small_pools=True),
]
PLAIN_OK = {"cfg1_full", "cfg2_full", "cfg3_base", "cfg3_base_t30", "cfg4_s001", "cfg5_s002", "edge_dups",
            "edge_format", "edge_identical", "edge_item0", "edge_none", "edge_single", "edge_ties"}


@pytest.mark.parametrize("name", golden_names())
def test_batched_matches_reference(tmp_path, name):
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
        h = fx["header"]
        assert db.info["trans_num"] == int(h["transNum"])
        assert db.info["trans_num_reduced"] == int(h["transNumReduced"])
        assert db.info["dimension_reduced"] == int(h["dimensionReduced"])
        assert db.info["dimension"] == int(h["dimension"])
        assert db.info["item_id_max_dense"] == int(h["itemIDmax"])
        for v in VARIANTS:
            res = db.mine(**v)
            got = res.as_dict()
            assert len(got) == len(res.mfis), "duplicate MFI reported"
            assert got == fx["expected"], (v, len(got), len(fx["expected"]))


@pytest.mark.parametrize("name", sorted(PLAIN_OK))
def test_plain_matches_reference(tmp_path, name):
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
        res = db.mine(engine="plain")
        assert res.as_dict() == fx["expected"]


def test_empty_database():
    off = np.zeros(1, np.int64)
    with tf.Database.from_csr(off, np.zeros(0, np.int32), 0.5) as db:
        assert db.info["trans_num"] == 0
        assert db.mine().mfis == []


def _certify(db, mfis, d2o):
    """The reference's MFI test on every reported set: support as reported and no counted
    item outside the set keeps it frequent (nfreq == |X|)."""
    o2d = {int(o): i for i, o in enumerate(d2o)}
    lists = [[o2d[x] for x in items] for items, _ in mfis]
    minc = db.info["min_count"]
    for s in range(0, len(lists), 512):
        part = lists[s:s + 512]
        counts, nfreq = db.count_wave(part, minc)
        for k, l in enumerate(part):
            items, sup = mfis[s + k]
            if len(l) > 1:
                assert counts[k, l[0]] == sup
            assert nfreq[k] == len(l)


@pytest.mark.slow
def test_cfg5_full_size_batched_equals_plain():
    db0 = synth.generate(5)
    with tf.Database.from_csr(db0.offsets, db0.items, 0.70) as db:
        a = db.mine(engine="batched")
        b = db.mine(engine="plain")
        assert a.as_dict() == b.as_dict()
        _certify(db, a.mfis, db.dense_to_orig())


@pytest.mark.slow
def test_cfg4_scaled_matches_oracle(oracle_mod, tmp_path):
    db0 = synth.generate(4, scale=0.05)
    p = str(tmp_path / "c4.txt")
    synth.write_fimi(p, db0)
    exp = oracle_mod.mine_file(p, 0.002)
    with tf.Database.from_csr(db0.offsets, db0.items, 0.002) as db:
        for counter in ("auto", "lop3", "tensor"):
            assert db.mine(counter=counter).as_dict() == exp
        assert db.mine(engine="resident", graphs=True).as_dict() == exp


@pytest.mark.slow
def test_cfg4_full_size_certified():
    db0 = synth.generate(4)
    with tf.Database.from_csr(db0.offsets, db0.items, 0.0005) as db:
        res = db.mine(engine="batched")
        assert len(res.mfis) > 1000
        _certify(db, res.mfis, db.dense_to_orig())
        assert db.mine(engine="resident").as_dict() == res.as_dict()
        assert db.mine(engine="resident", lookahead="learned").as_dict() == res.as_dict()
        g = db.mine(engine="resident", lookahead="learned", graphs=True)
        assert g.as_dict() == res.as_dict()
        assert g.stats["waves"] > 1


@pytest.mark.parametrize("graphs", [False, True])
@pytest.mark.parametrize("name", ["cfg1_full", "cfg4_s001", "cfg5_s002", "edge_ties"])
def test_resident_pool_growth(tmp_path, name, graphs):
    """Start every pool of the resident engine at its minimum, so that the pack declines
    waves that do not fit and the host grows the pools mid-search; results unchanged."""
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
        for la in ("filtered", "all"):
            res = db.mine(engine="resident", lookahead=la, graphs=graphs, small_pools=True, log_lookahead=True)
            assert res.as_dict() == fx["expected"], (la, graphs)


@pytest.mark.slow
def test_cfg3_replicated_matches_base_scaled():
    """Exact replication scales every support by the factor: the replicated DB's MFIs are
    the base DB's with supports x factor (data/make_replica.py:1-13)."""
    base = synth.generate(3, replicas=1, scale=0.1)
    rep = synth.replicate(base, 64)
    with tf.Database.from_csr(base.offsets, base.items, 0.3) as db:
        a = db.mine().as_dict()
    with tf.Database.from_csr(rep.offsets, rep.items, 0.3) as db:
        b = db.mine().as_dict()
    assert b == {k: v * 64 for k, v in a.items()}
    assert len(a) > 10


@pytest.mark.slow
def test_dense_full_size_matches_reference_fixture(tmp_path):
    """The benchmark's dense database at full size -- 49,000 base rows x 256 exact replicas =
    12,544,000 transactions, minsup 6% -- mined from its text file (device parse) by the
    resident engine with the learned proposal, host and graph wave loops: the reference's
    MFIs of the base rows (tests/golden/cfg3_base_t06, produced by the reference engine)
    with every support x 256."""
    fx = load_golden("cfg3_base_t06")
    want = {k: v * 256 for k, v in fx["expected"].items()}
    p = str(tmp_path / "dense.txt")
    synth.write_fimi_replicated(p, synth.cfg3_base(), 256)
    with tf.Database.from_file(p, synth.CFG3_DEVIATION_MINSUP) as db:
        assert db.info["trans_num"] == 12_544_000
        for graphs in (False, True):
            assert db.mine(engine="resident", lookahead="learned", graphs=graphs).as_dict() == want, graphs


@pytest.mark.parametrize("name", ["cfg1_full", "cfg4_s001", "cfg5_s002", "edge_ties", "cfg3_base"])
def test_any_tuning_keeps_output(tmp_path, name):
    """The tuning table changes launch shapes and counter choices, never the MFI set."""
    from tensorfim_b200 import engine
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    saved = engine.tuning()
    try:
        with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
            for t in (dict(wave_rows=16, l3_slices_per_sm=64.0, b1_tiles_per_sm=32.0, b1_min_rows=2, b1_min_cols=2),
                      dict(wave_rows=65536, l3_slices_per_sm=1.0, b1_tiles_per_sm=1.0, b1_min_rows=512,
                           b1_min_cols=512, rate_pair_incr=1e6)):
                engine.set_tuning(**t)
                for eng in ("resident", "batched"):
                    assert db.mine(engine=eng).as_dict() == fx["expected"], (t, eng)
                assert db.mine(engine="resident", graphs=True).as_dict() == fx["expected"], t
    finally:
        engine.set_tuning(**saved)



def test_large_top_family_on_every_tensor_path(oracle_mod, tmp_path):
    """An empty-prefix family of 140 items counted as a bitmap Gram: the automatic choice
    (tcgen05 kind::i8 tiles from 128 items), b1 tiles and LOP3 tiles all give the oracle's
    MFI set (every pair frequent, no triple: 9,730 MFIs)."""
    rng = np.random.Generator(np.random.PCG64(21))
    x = rng.random((4000, 140)) < 0.6
    off = np.zeros(x.shape[0] + 1, np.int64)
    off[1:] = np.cumsum(x.sum(1))
    items = (np.nonzero(x)[1] + 1).astype(np.int32)
    p = str(tmp_path / "dense140.txt")
    synth.write_fimi(p, synth.Database(offsets=off, items=items, n_items=140))
    exp = oracle_mod.mine_file(p, 0.3)
    with tf.Database.from_csr(off, items, 0.3) as db:
        assert db.info["n_survivors"] == 140
        for counter in ("auto", "tensor", "lop3"):
            res = db.mine(engine="resident", counter=counter, top="bitmap", lookahead=False)
            assert res.as_dict() == exp, counter


def test_pools_handed_to_the_next_database(tmp_path):
    """A closed database leaves its grown pools for the next one opened on the device; the
    next database (another word count per row, another search) adopts them and mines the
    reference's MFIs, and so does one opened after the cache is released."""
    # batched-only databases close one after another (each leaves a larger mask pool than the
    # last), then resident ones adopt what is cached
    names = [("edge_ties", "batched"), ("cfg1_t03", "batched"), ("cfg4_s001", "batched"), ("cfg1_t03", "resident"),
             ("cfg4_s001", "resident"), ("cfg1_t03", "resident"), ("edge_ties", "resident")]
    for k, (name, engine) in enumerate(names):
        fx = load_golden(name)
        path = golden_input(fx, tmp_path)
        with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
            for graphs in ((False,) if engine == "batched" else (False, True)):
                assert db.mine(engine=engine, graphs=graphs).as_dict() == fx["expected"], (name, engine, graphs)
        if k == 5:
            tf.release_cached()
    tf.release_cached(0)


@pytest.mark.parametrize("graphs", [False, True])
def test_dense_families_take_the_gram_and_tensor_paths(tmp_path, graphs):
    """The dense fixture (the replicated configuration's generator at 6%) under the automatic
    choice counts its narrow dense families with the register-tiled Gram counter and its wide
    ones with the tcgen05 family counter; forcing the CUDA-core tiles uses neither.  Every
    variant gives the reference's MFIs."""
    from tensorfim_b200 import _lib
    gram, tc = _lib.PATHS.index("gram"), _lib.PATHS.index("tc")
    fx = load_golden("cfg3_base_t06")
    path = golden_input(fx, tmp_path)
    with tf.Database.from_file(path, fx["spec"]["minsup"]) as db:
        a = db.mine(engine="resident", counter="auto", graphs=graphs)
        assert a.as_dict() == fx["expected"]
        assert a.stats["path_supports"][gram] > 0 and a.stats["path_supports"][tc] > 0
        b = db.mine(engine="resident", counter="lop3", graphs=graphs)
        assert b.as_dict() == fx["expected"]
        assert b.stats["path_supports"][gram] == 0 and b.stats["path_supports"][tc] == 0


def _long_and_tied_db():
    """150 rows of items 1..70 (an MFI longer than the device sorts per warp; id 0, which the
    reference searches apart with lists of at most 64 items, is left out), and ten MFIs
    {300 + k, 500, 501} of support 10 that share their support and their two largest items
    (dense ids keep the original order), so their device sort keys are equal."""
    rows = [list(range(1, 71))] * 150
    for k in range(10):
        rows += [[300 + k, 500, 501]] * 10
    off = np.zeros(len(rows) + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in rows])
    return off, np.concatenate([np.asarray(x, np.int32) for x in rows])


def _output_order(db, mfis):
    """The documented output order of a set of (items, support): descending support, then
    the item lists, each in descending dense-id order, compared lexicographically, larger
    first."""
    d2o = db.dense_to_orig()
    o2d = {int(o): d for d, o in enumerate(d2o)}
    keyed = []
    for items, sup in mfis:
        dense = sorted((o2d[x] for x in items), reverse=True)
        keyed.append((-sup, [-x for x in dense], len(dense), items, sup))
    # larger list first: a list before its own extensions comes after them
    keyed.sort(key=lambda t: (t[0], t[1] + [1]))
    return [(tuple(int(d2o[-x]) for x in t[1]), t[4]) for t in keyed]


@pytest.mark.parametrize("name", ["cfg1_full", "cfg4_s001", "edge_ties", "cfg3_base", "cfg3_base_t06", "long_tied"])
def test_resident_output_order(tmp_path, name):
    """The resident engine sorts its MFIs on the device (support, then the two largest items)
    and finishes equal keys on the host; the batched engine sorts on the host.  Both give the
    documented order; the 70-item set (longer than the batched engine lists) is checked on
    the resident engine alone."""
    if name == "long_tied":
        off, items = _long_and_tied_db()
        db = tf.Database.from_csr(off, items, 0.04)   # 10 of 250 rows
    else:
        fx = load_golden(name)
        db = tf.Database.from_file(golden_input(fx, tmp_path), fx["spec"]["minsup"])
    with db:
        runs = [db.mine(engine="resident", lookahead="all" if name == "long_tied" else True, **v).mfis
                for v in (dict(), dict(graphs=True), dict(counter="lop3", top="bitmap"))]
        exp = _output_order(db, runs[0])
        for got in runs:
            assert got == exp
        if name != "long_tied":
            assert db.mine(engine="batched").mfis == exp
    if name == "long_tied":
        assert len(exp) == 11 and len(exp[0][0]) == 70 and exp[0][1] == 150
        keys = [(s, x[:2]) for x, s in exp]
        assert len(set(keys)) < len(keys)   # equal device keys were finished on the host
