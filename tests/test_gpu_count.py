"""Counting contract on the GPU: exact integer supports, every counter, against the oracle.

Inputs follow the reference microbench's KAT advice (code/microbench/RESULTS.md:39-47):
sparse random bits (~12.5% density; all-ones data hides layout bugs), b and d not
multiples of 64, N not a multiple of 2048, item lists of length 0..31."""
import numpy as np
import pytest

import tensorfim_b200 as tf

pytestmark = pytest.mark.gpu


def _bits(rows, n_bits, seed, density_and=3):
    rng = np.random.Generator(np.random.PCG64(seed))
    w = (n_bits + 31) // 32
    x = np.full((rows, w), 0xFFFFFFFF, np.uint32)
    for _ in range(density_and):
        x &= rng.integers(0, 2**32, size=(rows, w), dtype=np.uint64).astype(np.uint32)
    if n_bits % 32:
        x[:, -1] &= np.uint32((1 << (n_bits % 32)) - 1)
    return x


def _lists(b, n_rows, seed, max_len=31):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(b):
        k = int(rng.integers(0, max_len + 1)) if i else 0
        out.append([int(v) for v in rng.integers(0, n_rows, size=k)])
    return out


SHAPES = [
    # n_rows, n_counted, n_bits, b, (density: ANDs of random words)
    (40, 33, 5_000, 5, 2),
    (150, 130, 100_003, 67, 3),
    (70, 17, 70_001, 1, 1),
    (90, 64, 262_144, 64, 3),
    (300, 257, 20_000, 200, 2),
    (24, 20, 1_500_001, 70, 3),
]


@pytest.mark.parametrize("counter", ["lop3", "tensor", "auto", "i8"])
@pytest.mark.parametrize("shape", SHAPES)
def test_count_wave_matches_oracle(oracle_mod, shape, counter):
    n_rows, d, n_bits, b, dens = shape
    rows = _bits(n_rows, n_bits, seed=n_rows * 7 + b, density_and=dens)
    lists = _lists(b, n_rows, seed=b + 11, max_len=min(31, n_rows))
    min_count = int(n_bits * 0.125 ** dens * 0.9)
    ref_c, ref_n = oracle_mod.count_wave(rows, lists, d, min_count)
    with tf.Database.from_bitmap(rows, n_bits, d) as db:
        got_c, got_n = db.count_wave(lists, min_count, counter=counter)
    assert got_c.shape == ref_c.shape
    assert (got_c == ref_c).all(), np.argwhere(got_c != ref_c)[:5]
    assert (got_n == ref_n).all()


def test_count_wave_threshold_ties(oracle_mod):
    rows = _bits(30, 4096, seed=3, density_and=1)
    lists = [[0], [1, 2], []]
    ref_c, _ = oracle_mod.count_wave(rows, lists, 30, 0)
    thr = int(ref_c[1, 5])   # a count exactly at the threshold is frequent
    ref_c, ref_n = oracle_mod.count_wave(rows, lists, 30, thr)
    with tf.Database.from_bitmap(rows, 4096, 30) as db:
        for counter in ("lop3", "tensor", "i8"):
            c, n = db.count_wave(lists, thr, counter=counter)
            assert (c == ref_c).all() and (n == ref_n).all()


def test_count_wave_rejects_long_lists():
    rows = _bits(8, 1000, seed=1)
    with tf.Database.from_bitmap(rows, 1000, 8) as db:
        with pytest.raises(tf.TfimError) as e:
            db.count_wave([[0] * 65], 1)
        assert e.value.code == 4
        with pytest.raises(tf.TfimError):
            db.count_wave([[9]], 1)


def test_count_wave_device_pointers(oracle_mod):
    import torch
    rows = _bits(100, 300_000, seed=5)
    lists = _lists(48, 100, seed=9)
    d = 90
    ref_c, ref_n = oracle_mod.count_wave(rows, lists, d, 4000)
    offs = np.zeros(len(lists) + 1, np.int64)
    offs[1:] = np.cumsum([len(x) for x in lists])
    flat = np.array([x for l in lists for x in l], np.int32)
    dev = torch.device("cuda:0")
    t_items = torch.from_numpy(flat).to(dev)
    t_offs = torch.from_numpy(offs).to(dev)
    t_counts = torch.zeros((len(lists), d), dtype=torch.int32, device=dev)
    t_nfreq = torch.zeros(len(lists), dtype=torch.int32, device=dev)
    with tf.Database.from_bitmap(rows, 300_000, d) as db:
        s = torch.cuda.current_stream().cuda_stream
        db.count_wave_device(t_items.data_ptr(), t_offs.data_ptr(), len(lists), 31, 4000, t_counts.data_ptr(),
                             t_nfreq.data_ptr(), s)
        torch.cuda.synchronize()
    assert (t_counts.cpu().numpy() == ref_c).all()
    assert (t_nfreq.cpu().numpy() == ref_n).all()
