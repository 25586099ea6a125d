"""The CPU oracle, pinned to the reference: its gold result files and its own engine."""
import os
import shutil

import numpy as np
import pytest

from conftest import REFERENCE, golden_input, golden_names, load_golden

GOLD = [("mushrooms.txt", 0.3), ("chess.txt", 0.8), ("connect.txt", 0.9), ("retail.txt", 0.01),
        ("T10I4D100K.txt", 0.005), ("connect.txt", 0.85)]


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "data", "gold_results")),
                    reason="reference gold files not mounted")
@pytest.mark.parametrize("dataset,minsup", GOLD)
def test_oracle_matches_reference_gold(oracle_mod, tmp_path, dataset, minsup):
    """Set-identical MFIs with identical frequencies to data/gold_results (the reference's
    own acceptance test, scripts/verify_all.py:39-45)."""
    src = os.path.join(REFERENCE, "data", "small", dataset)
    dst = tmp_path / dataset
    shutil.copyfile(src, dst)
    got = oracle_mod.mine_file(str(dst), minsup)
    gold = oracle_mod.load_results(os.path.join(REFERENCE, "data", "gold_results", "%s-%f=Results.txt" % (dataset, minsup)))
    assert got == gold


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_fixtures(oracle_mod, tmp_path, name):
    """Fixtures produced by the reference engine built from its sources (tests/golden)."""
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    db = oracle_mod.OracleDB(path, fx["spec"]["minsup"])
    got = db.mine()
    assert got == fx["expected"]
    info = db.info()
    assert info["trans_num"] == int(fx["header"]["transNum"])
    assert info["trans_num_reduced"] == int(fx["header"]["transNumReduced"])
    assert info["dimension_reduced"] == int(fx["header"]["dimensionReduced"])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "tfim_ref_mt")),
                    reason="reference binaries not built")
def test_reference_multithreaded_build_agrees(oracle_mod, tmp_path):
    """The reference's multithreaded CPU path (RUN_MODE 2, every node on the CPU) gives
    the same set as its serial path and the oracle."""
    fx = load_golden("cfg1_full")
    path = golden_input(fx, tmp_path)
    got, hdr = oracle_mod.run_reference(path, fx["spec"]["minsup"], binary=oracle_mod.REF_MT, threads=4)
    assert got == fx["expected"]


def _xorshift_bits(words, seed):
    """~12.5%-density random words from two xorshift streams (the reference microbench's
    KAT pattern, code/microbench/bmma_bench.cu:196-207), vectorised."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.integers(0, 2**32, size=words, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 2**32, size=words, dtype=np.uint64).astype(np.uint32)
    c = rng.integers(0, 2**32, size=words, dtype=np.uint64).astype(np.uint32)
    return a & b & c


def test_oracle_count_wave_kat(oracle_mod):
    rows = _xorshift_bits(40 * 97, 7).reshape(40, 97)
    lists = [[], [3], [1, 2], [5, 5, 7], list(range(10, 20))]
    counts, nfreq = oracle_mod.count_wave(rows, lists, 33, 300)
    for i, l in enumerate(lists):
        m = np.full(97, 0xFFFFFFFF, np.uint32)
        for x in l:
            m &= rows[x]
        exp = np.array([int(np.unpackbits((m & rows[e]).view(np.uint8)).sum()) for e in range(33)])
        assert (counts[i] == exp).all()
        assert nfreq[i] == (exp >= 300).sum()


def test_oracle_matches_reference_at_full_size_cfg5(oracle_mod, tmp_path):
    """The oracle against the reference's own output on configuration 5 at full size
    (2,000,000 transactions x 60 groups, minsup 70%): tests/golden/full/cfg5_full, produced by
    the reference's multithreaded CPU engine (make_golden.py)."""
    from conftest import load_golden_full
    fx = load_golden_full("cfg5_full")
    path = golden_input(fx, tmp_path)
    db = oracle_mod.OracleDB(path, fx["spec"]["minsup"])
    assert db.mine() == fx["expected"]
    assert db.info()["trans_num"] == int(fx["header"]["transNum"])
    db.close()
