"""Transaction-file parse on the GPU (tfim_parse_text / tfim_open_text / tfim_open_file)
against the oracle's restatement of the reference scanner (code/engine/src/kernel_bitmap.cu:
205-233): the CSR must be identical byte for byte on the golden input files, on generated
databases, on random byte strings over the characters the scanner distinguishes, and on
inputs shaped against the device layout (4 KiB tiles, a 64-byte halo, 8 MiB upload chunks)."""
import os

import numpy as np
import pytest

import tensorfim_b200 as tf
from tensorfim_b200 import synth
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TEXT_FILES = sorted(f for f in os.listdir(GOLDEN) if f.endswith(".txt"))


def oracle_csr(oracle_mod, tmp_path, data: bytes):
    p = tmp_path / "t.txt"
    p.write_bytes(data)
    return oracle_mod.parse_file(str(p))


def assert_same(got, want):
    assert got[0].shape == want[0].shape and (got[0] == want[0]).all()
    assert got[1].shape == want[1].shape and (got[1] == want[1]).all()


@pytest.mark.parametrize("name", TEXT_FILES)
def test_golden_files(oracle_mod, name):
    path = os.path.join(GOLDEN, name)
    with open(path, "rb") as f:
        data = f.read()
    assert_same(tf.parse_text(data), oracle_mod.parse_file(path))


@pytest.mark.parametrize("cfg,kw", [(1, {}), (4, dict(scale=0.02)), (5, dict(scale=0.01))])
def test_generated_databases(oracle_mod, tmp_path, cfg, kw):
    p = str(tmp_path / "db.txt")
    synth.write_fimi(p, synth.generate(cfg, **kw))
    with open(p, "rb") as f:
        data = f.read()
    assert_same(tf.parse_text(data), oracle_mod.parse_file(p))


def random_text(rng, n: int) -> bytes:
    """Random bytes over digits, '-', separators, CR and LF, with runs of up to 18 digits."""
    out = bytearray()
    seps = b" \t\r\n-,x\n\n"
    while len(out) < n:
        if rng.random() < 0.55:
            out += bytes(rng.integers(48, 58, size=int(rng.integers(1, 19))).tolist())
        else:
            out += bytes([seps[int(rng.integers(0, len(seps)))]])
    return bytes(out[:n])


@pytest.mark.parametrize("seed,n", [(0, 1), (1, 17), (2, 4095), (3, 4096), (4, 4097), (5, 70_000), (6, 1_000_003)])
def test_random_bytes(oracle_mod, tmp_path, seed, n):
    data = random_text(np.random.Generator(np.random.PCG64(seed)), n)
    assert_same(tf.parse_text(data), oracle_csr(oracle_mod, tmp_path, data))


def test_empty_and_newline_only(oracle_mod, tmp_path):
    for data in [b"", b"\n", b"\n\n\n", b"-", b"-5", b"7", b"1 2\n-3", b"1 2\n3", b"\r\n\r\n"]:
        assert_same(tf.parse_text(data), oracle_csr(oracle_mod, tmp_path, data))


def test_tile_and_halo_boundaries(oracle_mod, tmp_path):
    """Ids and '-' signs straddling the 4 KiB tiles, and digit runs longer than the 64-byte
    halo (values taken modulo 2^32, as the reference's int conversion of its accumulator)."""
    parts = []
    for k in range(1, 6):
        pad = b" " * (4096 * k - 3 - sum(len(p) for p in parts))
        parts += [pad, b"12345 -678 9\n"]
    data = b"".join(parts)
    assert_same(tf.parse_text(data), oracle_csr(oracle_mod, tmp_path, data))
    long_run = b"9" * 150
    for lead in [0, 4000, 4095, 4096 - 64, 4096 - 65]:
        data = b" " * lead + long_run + b" 4\n" + b"-" + long_run + b" 5"
        off, items = tf.parse_text(data)
        want = np.array([int(long_run) % (1 << 32), 4, 5], np.uint32).view(np.int32)
        assert off.tolist() == [0, 2, 3] and items.tolist() == want.tolist()


def test_upload_paths(oracle_mod, tmp_path):
    """Above the 8 MiB upload chunk: pageable bytes (staged by worker threads), a pinned
    buffer (one copy), and a file read straight into the staging; all give the same CSR
    and the same database as the oracle's parse."""
    import torch
    data = random_text(np.random.Generator(np.random.PCG64(9)), 20_000_017)
    want = oracle_csr(oracle_mod, tmp_path, data)
    assert_same(tf.parse_text(data), want)
    pinned = torch.empty(len(data), dtype=torch.uint8).pin_memory()
    pinned.numpy()[:] = np.frombuffer(data, np.uint8)
    assert_same(tf.parse_text(pinned.numpy()), want)
    # a database file of about 22 MB (the random text above has ids beyond int32)
    p = str(tmp_path / "db.txt")
    synth.write_fimi(p, synth.generate(4, scale=0.4))
    assert os.path.getsize(p) > 16 << 20
    off, items = oracle_mod.parse_file(p)
    with tf.Database.from_file(p, 0.001) as a, tf.Database.from_csr(off, items, 0.001) as b:
        assert a.info == b.info
        assert (a.dense_to_orig() == b.dense_to_orig()).all()


@pytest.mark.parametrize("name", ["edge_format.txt", "edge_item0.txt", "edge_dups.txt"])
def test_open_text_matches_open_db(oracle_mod, name):
    path = os.path.join(GOLDEN, name)
    off, items = oracle_mod.parse_file(path)
    with open(path, "rb") as f:
        data = f.read()
    for minsup in (0.05, 0.3):
        with tf.Database.from_text(data, minsup) as a, tf.Database.from_csr(off, items, minsup) as b:
            assert a.info == b.info
            assert a.mine().as_dict() == b.mine().as_dict()


def test_errors():
    with pytest.raises(tf.TfimError) as e:
        tf.Database.from_file("/nonexistent/transactions.txt", 0.1)
    assert e.value.code == 7
    with pytest.raises(tf.TfimError) as e:   # an id above INT32_MAX reads as negative
        tf.Database.from_text(b"1 2\n3000000000 1\n", 0.1)
    assert e.value.code == 1
