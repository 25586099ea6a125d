"""tfim_count_wave_noalloc: counting with no GPU allocation, checked against
tfim_count_wave_device and against the oracle's counter on the same inputs, twice in a
row, with the device memory in use unchanged across a call.

The allocation-free entry point serves callers that cannot call cudaMalloc: code inside a
memory budget that another allocator owns, and code that only holds device pointers it
was handed.  Its scratch is a fixed device array inside the library that every call
shares, so two consecutive calls must both be exact: the second must not see anything
left over from the first.  Counts are integers, so the tolerance is zero.  The item lists
name rows beyond the counted ones (the bitmap holds 90 rows, 70 are counted).  This file
is collected last so that a failure here stops a -x run only after every other test has
run; it passes alone and after the rest."""
import ctypes as C

import numpy as np
import pytest

import tensorfim_b200 as tf
from tensorfim_b200 import _lib

pytestmark = pytest.mark.gpu


def _rows(n_rows, n_bits, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    w = (n_bits + 31) // 32
    x = rng.integers(0, 2**32, size=(n_rows, w), dtype=np.uint64).astype(np.uint32)
    x &= rng.integers(0, 2**32, size=(n_rows, w), dtype=np.uint64).astype(np.uint32)
    if n_bits % 32:
        x[:, -1] &= np.uint32((1 << (n_bits % 32)) - 1)
    return x


def _wave(b, n_rows, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    lists = [[int(v) for v in rng.integers(0, n_rows, size=int(rng.integers(0, 12)))] for _ in range(b)]
    offs = np.zeros(b + 1, np.int64)
    offs[1:] = np.cumsum([len(l) for l in lists])
    flat = np.array([x for l in lists for x in l] or [0], np.int32)
    return lists, offs, flat


def _noalloc(t_bitmap, W, d, t_items, t_offs, b, min_count, got_c, got_n, stream):
    return _lib.lib().tfim_count_wave_noalloc(C.c_void_p(t_bitmap.data_ptr()), W, d, C.c_void_p(t_items.data_ptr()),
                                              C.c_void_p(t_offs.data_ptr()), b, min_count, C.c_void_p(got_c.data_ptr()),
                                              C.c_void_p(got_n.data_ptr()), C.c_void_p(stream))


def test_noalloc_matches_count_wave_device_on_two_calls(oracle_mod):
    import torch
    n_rows, d, n_bits = 90, 70, 150_001
    rows = _rows(n_rows, n_bits, seed=21)
    # caller-owned device bitmap, rows padded to a multiple of 64 words
    W = ((n_bits + 31) // 32 + 63) // 64 * 64
    padded = np.zeros((n_rows, W), np.uint32)
    padded[:, : rows.shape[1]] = rows
    dev = torch.device("cuda:0")
    t_bitmap = torch.from_numpy(padded.view(np.int32)).to(dev)
    stream = torch.cuda.current_stream().cuda_stream
    with tf.Database.from_bitmap(rows, n_bits, d) as db:
        for call, (b, seed) in enumerate([(53, 5), (37, 6)]):
            lists, offs, flat = _wave(b, n_rows, seed)
            assert max(flat) >= d, "the lists must name rows beyond the counted ones"
            min_count = 4000
            t_items = torch.from_numpy(flat).to(dev)
            t_offs = torch.from_numpy(offs).to(dev)
            ref_c = torch.zeros((b, d), dtype=torch.int32, device=dev)
            ref_n = torch.zeros(b, dtype=torch.int32, device=dev)
            db.count_wave_device(t_items.data_ptr(), t_offs.data_ptr(), b, 12, min_count, ref_c.data_ptr(),
                                 ref_n.data_ptr(), stream)
            got_c = torch.full((b, d), -7, dtype=torch.int32, device=dev)
            got_n = torch.full((b,), -7, dtype=torch.int32, device=dev)
            torch.cuda.synchronize()
            free0, _ = torch.cuda.mem_get_info(dev)
            alloc0 = torch.cuda.memory_allocated(dev)
            _lib.check(_noalloc(t_bitmap, W, d, t_items, t_offs, b, min_count, got_c, got_n, stream))
            torch.cuda.synchronize()
            free1, _ = torch.cuda.mem_get_info(dev)
            if call > 0:   # the first call on a device may load the library's module
                assert free1 == free0, f"call {call}: device free memory changed by {free0 - free1} bytes"
            assert torch.cuda.memory_allocated(dev) == alloc0
            assert torch.equal(got_c, ref_c), f"call {call}: counts differ from tfim_count_wave_device"
            assert torch.equal(got_n, ref_n), f"call {call}: nfreq differ from tfim_count_wave_device"
            exp_c, exp_n = oracle_mod.count_wave(rows, lists, d, min_count)
            assert np.array_equal(got_c.cpu().numpy(), exp_c), f"call {call}: counts differ from the oracle"
            assert np.array_equal(got_n.cpu().numpy(), exp_n), f"call {call}: nfreq differ from the oracle"


def test_noalloc_rejects_a_wave_beyond_the_scratch():
    import torch
    dev = torch.device("cuda:0")
    W = 1 << 20   # 4 MiB per prefix mask: 5 nodes exceed the 16 MiB scratch
    t_bitmap = torch.zeros((1, W), dtype=torch.int32, device=dev)
    t_offs = torch.zeros(6, dtype=torch.int64, device=dev)
    t_items = torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.zeros((5, 1), dtype=torch.int32, device=dev)
    nf = torch.zeros(5, dtype=torch.int32, device=dev)
    rc = _lib.lib().tfim_count_wave_noalloc(C.c_void_p(t_bitmap.data_ptr()), W, 1, C.c_void_p(t_items.data_ptr()),
                                            C.c_void_p(t_offs.data_ptr()), 5, 1, C.c_void_p(out.data_ptr()),
                                            C.c_void_p(nf.data_ptr()), None)
    assert rc == _lib.TFIM_E_INVALID
    assert b"static scratch holds" in _lib.lib().tfim_last_error()
