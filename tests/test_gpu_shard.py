"""Transaction-sharded databases on the GPU: shards of one database, each holding a slice of
the transactions, must report exactly what the unsharded database reports (header fields,
MFIs with supports, count waves, all frequent itemsets, the results file) and what the
reference engine reported for the golden fixtures.

The shards run as host threads of one process on one GPU (ThreadGroup): they meet on the
host at every all-reduce and one thread sums the partial buffers, so no kernel ever waits
for another.  The NCCL group (TorchGroup) is checked through its all-reduce on one rank."""
import numpy as np
import pytest

import tensorfim_b200 as tf
from tensorfim_b200 import _lib, synth
from tensorfim_b200.engine import read_fimi
from tensorfim_b200.shard import ThreadGroup, TorchGroup, shard_csr
from conftest import golden_input, load_golden

pytestmark = pytest.mark.gpu

NAMES = ["edge_dups", "edge_format", "edge_identical", "edge_item0", "edge_none", "edge_single", "edge_ties",
         "cfg1_full", "cfg2_full", "cfg3_base_t30", "cfg4_s001", "cfg5_s002"]
INFO_KEYS = ["trans_num", "trans_num_reduced", "dimension", "dimension_reduced", "item_id_min", "item_id_max",
             "item_id_max_dense", "n_dense", "n_survivors", "min_count", "frequency_threshold", "trans_len_min",
             "trans_len_max", "trans_len_mean", "trans_len_red_min", "trans_len_red_max"]


def _sharded(off, items, minsup, world, fn):
    """fn(db, member) on every shard of (off, items); results in rank order."""
    g = ThreadGroup(world)

    def body(m):
        o, it = shard_csr(off, items, m.rank, world)
        with tf.Database.from_csr_sharded(o, it, minsup, m) as db:
            return fn(db, m)
    return g.run(body)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", NAMES)
def test_sharded_mine_matches_reference(tmp_path, name, world):
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    minsup = fx["spec"]["minsup"]
    off, items = read_fimi(path)
    with tf.Database.from_file(path, minsup) as db:
        info = db.info
        assert db.mine(engine="batched").as_dict() == fx["expected"]
        whole = tmp_path / "whole.txt"
        db.write_results(path, str(whole))

    def run(db, m):
        out = {"info": db.info, "mine": {}}
        for engine, counter, la in [("batched", "auto", True), ("batched", "lop3", False), ("batched", "tensor", "all"),
                                    ("plain", "auto", False)]:
            out["mine"][(engine, counter, la)] = db.mine(engine=engine, counter=counter, lookahead=la).as_dict()
        if m.rank == 0:
            db.write_results(path, str(tmp_path / "shard.txt"))
        return out
    res = _sharded(off, items, minsup, world, run)
    for r in res:
        for k in INFO_KEYS:
            a, b = r["info"][k], info[k]
            assert a == b or (a != a and b != b), (k, a, b)
        for v, got in r["mine"].items():
            assert got == fx["expected"], (v, len(got), len(fx["expected"]))
    assert (tmp_path / "shard.txt").read_text() == whole.read_text()


@pytest.mark.parametrize("counter", ["auto", "lop3", "tensor", "i8"])
def test_sharded_count_wave_and_all_itemsets(counter):
    db0 = synth.generate(4, scale=0.02)
    minsup = 0.004
    with tf.Database.from_csr(db0.offsets, db0.items, minsup) as db:
        d = db.info["n_survivors"]
        rng = np.random.default_rng(5)
        lists = [sorted(rng.choice(d, size=int(rng.integers(0, 4)), replace=False).tolist()) for _ in range(200)]
        mc = db.info["min_count"]
        exp_counts, exp_nfreq = db.count_wave(lists, mc, counter=counter)
        db.set_counter(counter)
        exp_all = db.mine_all(max_len=4).as_dict()

    def run(sdb, m):
        c, n = sdb.count_wave(lists, mc, counter=counter)
        sdb.set_counter(counter)
        return c, n, sdb.mine_all(max_len=4).as_dict()
    for c, n, fis in _sharded(db0.offsets, db0.items, minsup, 3, run):
        np.testing.assert_array_equal(c, exp_counts)
        np.testing.assert_array_equal(n, exp_nfreq)
        assert fis == exp_all


def test_sharded_bitmap_matches_whole():
    rng = np.random.default_rng(11)
    n_bits, n_rows = 50_000, 40
    dense = rng.random((n_rows, n_bits)) < 0.3
    lists = [sorted(rng.choice(n_rows, size=2, replace=False).tolist()) for _ in range(64)]

    def pack(bits):   # bit t of word t // 32 = transaction t
        w = (bits.shape[1] + 31) // 32
        padded = np.zeros((bits.shape[0], w * 32), bool)
        padded[:, :bits.shape[1]] = bits
        return np.ascontiguousarray(np.packbits(padded, axis=1, bitorder="little").view("<u4"))
    with tf.Database.from_bitmap(pack(dense), n_bits, n_rows) as db:
        exp, _ = db.count_wave(lists, 1)
    cuts = [0, 12_345, 31_000, n_bits]   # word-unaligned shard boundaries
    g = ThreadGroup(3)

    def body(m):
        part = dense[:, cuts[m.rank]:cuts[m.rank + 1]]
        with tf.Database.from_bitmap_sharded(pack(part), part.shape[1], n_rows, m) as sdb:
            assert sdb.info["trans_num_reduced"] == n_bits
            return sdb.count_wave(lists, 1)[0]
    for got in g.run(body):
        np.testing.assert_array_equal(got, exp)


def test_empty_shards_and_refusals(tmp_path):
    fx = load_golden("edge_ties")
    path = golden_input(fx, tmp_path)
    off, items = read_fimi(path)
    # more shards than rows: some shards hold nothing
    few = off[:4]
    g = ThreadGroup(6)
    with tf.Database.from_csr(few, items[:few[-1]], 0.5) as db:
        exp = db.mine(engine="batched").as_dict()
        exp_info = db.info

    def body(m):
        o, it = shard_csr(few, items[:few[-1]], m.rank, 6)
        with tf.Database.from_csr_sharded(o, it, 0.5, m) as sdb:
            return sdb.info, sdb.mine().as_dict()
    for info, got in g.run(body):
        assert got == exp
        assert info["trans_num"] == exp_info["trans_num"] == 3
    # the resident engine is refused on every shard (before any collective)

    def resident(db, m):
        with pytest.raises(tf.TfimError) as e:
            db.mine(engine="resident")
        return e.value.code
    assert _sharded(off, items, 0.2, 2, resident) == [_lib.TFIM_E_STATE] * 2
    # shards that disagree on the threshold are all refused
    g = ThreadGroup(2)

    def disagree(m):
        o, it = shard_csr(off, items, m.rank, 2)
        with pytest.raises(tf.TfimError, match="differs across the group"):
            tf.Database.from_csr_sharded(o, it, [0.2, 0.3][m.rank], m)
    g.run(disagree)


def test_torch_group_allreduce_on_the_library_stream():
    import datetime
    import socket

    import torch
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda:0"))
    try:
        grp = TorchGroup(device=0)
        assert (grp.rank, grp.world) == (0, 1)
        stream = torch.cuda.Stream()
        for dtype, tdt in [(_lib.DT_I32, torch.int32), (_lib.DT_I64, torch.int64)]:
            for op in (_lib.RED_SUM, _lib.RED_MIN, _lib.RED_MAX):
                t = torch.arange(-5, 1000, device="cuda:0", dtype=tdt)
                ref = t.clone()
                torch.cuda.synchronize()
                grp.allreduce(t.data_ptr(), t.numel(), dtype, op, stream.cuda_stream)
                stream.synchronize()
                assert torch.equal(t, ref)
        # the callback the library calls: status 0, and 1 with the error kept for a bad dtype
        st = grp.struct()
        t = torch.ones(8, device="cuda:0", dtype=torch.int32)
        assert st.allreduce(t.data_ptr(), 8, _lib.DT_I32, _lib.RED_SUM, None, None) == 0
        assert st.allreduce(t.data_ptr(), 8, 7, _lib.RED_SUM, None, None) == 1
        assert grp.last_error
    finally:
        dist.destroy_process_group()
