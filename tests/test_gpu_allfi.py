"""All frequent itemsets, level by level on the counting contract (the reference's level-wise
prototype, code/batch_proto/batch_proto.cu:257-409): the prototype's own checks -- downward
closure and planted-pattern recall -- plus exact supports and completeness against a CPU
level-wise miner on the same bitmap."""
import itertools

import numpy as np
import pytest

import tensorfim_b200 as tf
from tensorfim_b200._lib import TfimError

pytestmark = pytest.mark.gpu


def _planted(n_tx=1 << 16, n_items=96, n_pat=10, seed=3):
    """Seeded planted database in the prototype's shape: patterns of 2..6 items firing i.i.d.
    per transaction with probability 0.2%..1.5%, plus light noise."""
    rng = np.random.Generator(np.random.PCG64(seed))
    words = n_tx // 32
    rows = np.zeros((n_items, words), np.uint32)
    pats = []
    for _ in range(n_pat):
        size = int(rng.integers(2, 7))
        items = sorted(int(x) for x in rng.choice(n_items, size=size, replace=False))
        freq = (0.2 + 1.3 * rng.random()) / 100.0 * 4   # scaled for the smaller database
        pats.append(items)
        t = np.nonzero(rng.random(n_tx) < freq)[0]
        for it in items:
            np.bitwise_or.at(rows[it], t // 32, np.left_shift(np.uint32(1), (t % 32).astype(np.uint32)))
    for it in range(n_items):
        t = rng.integers(0, n_tx, size=int(n_tx * 0.002))
        np.bitwise_or.at(rows[it], t // 32, np.left_shift(np.uint32(1), (t % 32).astype(np.uint32)))
    return rows, pats


def _bits(rows):
    return np.unpackbits(rows.view(np.uint8), bitorder="little").reshape(rows.shape[0], -1).astype(bool)


def _cpu_levelwise(bits, min_count, max_len):
    """Every frequent itemset (ascending ids) with its support, by exact boolean ANDs."""
    n_items = bits.shape[0]
    out = {}
    cur = []
    for i in range(n_items):
        s = int(bits[i].sum())
        if s >= min_count:
            out[(i,)] = s
            cur.append(((i,), bits[i]))
    for _ in range(2, max_len + 1):
        nxt = []
        for items, m in cur:
            for j in range(items[-1] + 1, n_items):
                mm = m & bits[j]
                s = int(mm.sum())
                if s >= min_count:
                    out[items + (j,)] = s
                    nxt.append((items + (j,), mm))
        cur = nxt
    return out


@pytest.mark.parametrize("counter", ["auto", "lop3", "tensor", "i8"])
def test_planted_database(counter):
    rows, pats = _planted()
    n_tx = rows.shape[1] * 32
    min_count = int(n_tx * 0.006)
    with tf.Database.from_bitmap(rows, n_tx, rows.shape[0]) as db:
        db.set_counter(counter)
        res = db.mine_all(min_count=min_count, max_len=8)
    got = {tuple(k): v for k, v in res.mfis}
    # exact supports and completeness against the CPU miner
    exp = _cpu_levelwise(_bits(rows), min_count, 8)
    assert got == exp
    # the prototype's checks: downward closure and planted recall
    for items in got:
        for sub in itertools.combinations(items, len(items) - 1):
            if sub:
                assert sub in got, (items, sub)
    for p in pats:
        sup = int(np.logical_and.reduce(_bits(rows)[p]).sum())
        assert (tuple(p) in got) == (sup >= min_count), (p, sup)
    assert res.stats["waves"] >= 1 and len(got) > len(pats)


def test_transaction_database_and_limits():
    """A database opened from transactions: original ids, the reference's min count, the
    result cap, and max_len."""
    rng = np.random.Generator(np.random.PCG64(9))
    x = rng.random((3000, 40)) < 0.35
    off = np.zeros(x.shape[0] + 1, np.int64)
    off[1:] = np.cumsum(x.sum(1))
    items = (np.nonzero(x)[1] * 3 + 7).astype(np.int32)   # original ids 7, 10, 13, ...
    with tf.Database.from_csr(off, items, 0.05) as db:
        mc = db.info["min_count"]
        res = db.mine_all(max_len=4)
        got = {tuple(k): v for k, v in res.mfis}
        exp = {tuple(i * 3 + 7 for i in k): v for k, v in _cpu_levelwise(x.T.copy(), mc, 4).items()}
        assert got == exp
        assert max(len(k) for k in got) <= 4
        with pytest.raises(TfimError):
            db.mine_all(max_len=4, max_itemsets=len(got) - 1)
        assert db.mine_all(max_len=1).mfis and all(len(k) == 1 for k, _ in db.mine_all(max_len=1).mfis)
