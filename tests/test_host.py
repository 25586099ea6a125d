"""Host-side logic that needs no GPU: parser, generators, results files, the C ABI's
exports and argument checks, and the command-line front end's failure paths."""
import os
import re
import subprocess

import numpy as np
import pytest

import tensorfim_b200 as tf
from tensorfim_b200 import _lib, synth
from conftest import GOLDEN, ROOT, golden_input, load_golden


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "tfim.h")).read()
    return sorted(set(re.findall(r"TFIM_API\s+[\w\s\*]+?\b(tfim_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import ctypes
    declared = _declared_symbols()
    assert len(declared) >= 17
    assert sorted(declared) == sorted(_lib.EXPORTS)
    L = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared:
        assert hasattr(L, name), name
    assert b"sm_100a" in _lib.lib().tfim_version()


def test_invalid_threshold_is_rejected_before_any_device_work():
    off = np.array([0, 2], np.int64)
    items = np.array([1, 2], np.int32)
    for thr in (0.0, -0.1, 1.5, float("nan")):
        with pytest.raises(tf.TfimError) as e:
            tf.Database.from_csr(off, items, thr)
        assert e.value.code == _lib.TFIM_E_INVALID


def _has_gpu():
    try:
        r = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=20)
        return r.returncode == 0 and "GPU" in r.stdout
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour on a machine without a GPU")
def test_no_gpu_fails_loudly():
    off = np.array([0, 2], np.int64)
    items = np.array([1, 2], np.int32)
    with pytest.raises(tf.TfimError) as e:
        tf.Database.from_csr(off, items, 0.5)
    assert e.value.code == _lib.TFIM_E_CUDA


def test_cli_usage_and_missing_file(tmp_path):
    assert os.path.exists(_lib.CLI_PATH)
    r = subprocess.run([_lib.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 1
    r = subprocess.run([_lib.CLI_PATH, str(tmp_path / "nope.txt"), "0.5"], capture_output=True, text=True)
    assert r.returncode == 1 and "open failed!" in r.stdout


@pytest.mark.parametrize("extra,msg", [(["--engine", "fast"], "unknown engine"), (["--counter", "fp8"], "unknown counter"),
                                       (["--frobnicate", "1"], "unknown option")])
def test_cli_rejects_unknown_flags_before_reading(tmp_path, extra, msg):
    r = subprocess.run([_lib.CLI_PATH, str(tmp_path / "nope.txt"), "0.5", *extra], capture_output=True, text=True)
    assert r.returncode == 1 and msg in r.stderr and "open failed!" not in r.stdout


def test_sharded_open_checks_the_group_before_any_device_work():
    import ctypes as C
    off = np.array([0, 2], np.int64)
    items = np.array([1, 2], np.int32)
    h = C.c_void_p()
    for rank, world, fn in [(0, 0, None), (2, 2, None), (-1, 2, None), (1, 2, None)]:
        g = _lib.Group(rank, world, _lib.ALLREDUCE_FN() if fn is None else fn, None)
        rc = _lib.lib().tfim_open_db_sharded(off.ctypes.data, items.ctypes.data, 1, 0.5, 0, C.byref(g), C.byref(h))
        assert rc == _lib.TFIM_E_INVALID, (rank, world)
        assert "tfim_group" in _lib.lib().tfim_last_error().decode()
        rc = _lib.lib().tfim_open_bitmap_sharded(np.zeros(4, np.uint32).ctypes.data, 1, 64, 1, 0, C.byref(g), C.byref(h))
        assert rc == _lib.TFIM_E_INVALID
    assert _lib.lib().tfim_open_db_sharded(off.ctypes.data, items.ctypes.data, 1, 0.5, 0, None, C.byref(h)) \
        == _lib.TFIM_E_INVALID
    assert _lib.lib().tfim_mine_all(None, 1, 4, 10, None) == _lib.TFIM_E_INVALID
    assert _lib.lib().tfim_num_all(None) == -1


@pytest.mark.parametrize("name", ["edge_format", "edge_dups", "edge_item0", "edge_single", "cfg1_full"])
def test_read_fimi_matches_oracle_parse(oracle_mod, tmp_path, name):
    """The Python parser (Database.from_file) follows the reference byte scanner: same row
    count (empty lines included), same reduced rows."""
    fx = load_golden(name)
    path = golden_input(fx, tmp_path)
    off, items = tf.read_fimi(path)
    assert off.shape[0] - 1 == int(fx["header"]["transNum"])
    assert int(items.max(initial=0)) <= 10**9
    lens = np.diff(off)
    assert lens.min(initial=0) >= 0
    if fx["header"]["transLengthMax"] is not None and off.shape[0] > 1:
        assert lens.max() == int(fx["header"]["transLengthMax"])


def test_read_fimi_edge_bytes(tmp_path):
    p = tmp_path / "x.txt"
    p.write_bytes(b"1 2\r\n\n-3 4 -5\n7x8\t9\n10")
    off, items = tf.read_fimi(str(p))
    assert list(np.diff(off)) == [2, 0, 1, 3, 1]
    assert list(items) == [1, 2, 4, 7, 8, 9, 10]
    p.write_bytes(b"1 2\n\n")
    off, items = tf.read_fimi(str(p))
    assert list(np.diff(off)) == [2, 0]


def test_synth_shapes_and_determinism():
    a = synth.generate(1)
    b = synth.generate(1)
    assert a.n_rows == 10_000 and (a.items == b.items).all()
    assert (np.diff(a.offsets) == 23).all() and a.n_items == 115
    c = synth.generate(2, scale=0.1)
    assert c.n_items == 129 and (np.diff(c.offsets) == 43).all()
    d = synth.generate(3, replicas=2, scale=0.01)
    assert d.n_rows == 2 * 490 and abs(d.n_items - 2100) <= 40
    assert (d.items[: d.offsets[490]] == d.items[d.offsets[490]:]).all()
    e = synth.generate(4, scale=0.002)
    assert e.n_rows == 2000 and e.items.min() >= 1 and e.items.max() <= 40_000
    rows_sorted = all((np.diff(e.items[e.offsets[r]:e.offsets[r + 1]]) > 0).all() for r in range(e.n_rows))
    assert rows_sorted
    f = synth.generate(5, scale=0.001)
    assert (np.diff(f.offsets) == 60).all() and 400 <= f.n_items <= 600


def test_write_fimi_round_trip(tmp_path):
    db = synth.generate(4, scale=0.001)
    p = str(tmp_path / "r.txt")
    synth.write_fimi(p, db)
    off, items = tf.read_fimi(p)
    assert (off == db.offsets).all() and (items == db.items).all()


def test_results_parser_and_compare(tmp_path):
    p = tmp_path / "r.txt"
    p.write_text("MFIsNumber: 2\n1th: 2 { 9 3 }   support: 0.5  frequency: 50\n2th: 1 { 4 }   support: 0.4  frequency: 40\n")
    r = tf.load_results(str(p))
    assert r == {frozenset({3, 9}): 50, frozenset({4}): 40}
    assert tf.load_header(str(p))["MFIsNumber"] == "2"
    c = tf.compare(r, {frozenset({3, 9}): 51})
    assert not c["identical"] and c["freq_mismatch"] == [((3, 9), 50, 51)]


def test_levelwise_generator_plants_patterns():
    from tensorfim_b200.levelwise import generate, support
    n = 20_000
    rows, pats = generate(n, 64, 6, seed=1)
    assert rows.shape == (64, (n + 31) // 32) and rows.dtype == np.uint32
    assert len(pats) == 6 and all(2 <= len(p) <= 6 and p == sorted(set(p)) for p in pats)
    bits = np.unpackbits(rows.view(np.uint8), axis=1, bitorder="little")[:, :n].astype(bool)
    for p in pats:
        s = support(rows, p)
        assert s == int(np.logical_and.reduce(bits[p], axis=0).sum())
        assert s >= int(0.001 * n)   # every pattern fires on at least 0.2% of rows in expectation


def test_bench_reference_support_counts_match_the_oracle_search(oracle_mod):
    """bench.py's reference-equivalent support counts are the reference search's node count x
    survivors; the oracle runs that search (the replicated workload at its base size, where
    the search is the same and only supports scale)."""
    import bench
    for name, db in (("cfg1", synth.generate(1)), ("cfg3dev", synth.cfg3_base())):
        w = bench.WORKLOADS[name]
        o = oracle_mod.OracleDB(None, w["minsup"], csr=(db.offsets, db.items))
        o.mine(0)
        assert o.nodes * o.info()["n_survivors"] == w["ref_supports"], name
        o.close()


def test_replicated_text_is_the_base_text_repeated(tmp_path):
    base = synth.generate(3, replicas=1, scale=0.01)
    p1, p2 = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
    synth.write_fimi_replicated(p1, base, 3)
    synth.write_fimi(p2, synth.replicate(base, 3))
    assert open(p1, "rb").read() == open(p2, "rb").read()


def test_path_rooflines_arithmetic():
    from tensorfim_b200 import measure
    st = {"path_ms": [2.0, 0, 1.0, 0, 0, 0], "path_launches": [2, 0, 1, 0, 0, 0],
          "path_bytes": [4e9, 0, 1e9, 0, 0, 0], "path_bitops": [8e12, 0, 5e10, 0, 0, 0]}
    p = measure.path_rooflines([st, st], hbm_gbs=6000.0, i8_macs=1e15)
    assert set(p) == {"lop3", "tc"}
    assert p["lop3"]["achieved_gbs"] == 2000.0 and p["lop3"]["launches"] == 4
    assert abs(p["tc"]["tensor_frac"] - 0.05) < 1e-12
    assert abs(p["lop3"]["share_of_counting"] - 2 / 3) < 1e-12
    r = measure.headline_roofline(p, 6000.0, 1e15, "measured", "measured")
    assert r["kernel"] == "k_count_lop3" and r["bound"] == "hbm" and abs(r["frac"] - 1 / 3) < 1e-12
    assert r["traffic"] is None
    # a measured DRAM-per-algorithmic-byte ratio scales with each run's algorithmic bytes
    p = measure.path_rooflines([st, st], hbm_gbs=6000.0, i8_macs=1e15, traffic={"lop3": 0.25})
    assert p["lop3"]["traffic_per_launch"] == 0.25 * 8e9 / 4 and "traffic_per_launch" not in p["tc"]
    r = measure.headline_roofline(p, 6000.0, 1e15, "measured", "measured")
    assert r["traffic"] == 0.5e9


def test_family_counter_shared_memory_windows():
    """The tcgen05 family counter's shared-memory layout (csrc/count_fam.cu), restated: for
    every tile the pack can emit (nF <= 128 columns, rows a run [s0, s0 + nr) of them), every
    expanded row, every A window (128 rows from a K block's start) and every B window stays
    inside the allocation, K blocks are 1024-byte aligned and a warp's units fit its lanes."""
    stage_bytes, stages, guard, kbytes, align = 2 * 144 * 128, 5, 128 * 128, 128, 1024
    smem = stages * stage_bytes + guard + align
    assert smem <= 227 * 1024 - 256
    worst = 0
    for nF in range(1, 129):
        for s0 in range(0, nF):
            for nr in range(1, nF - s0 + 1):
                b8 = s0 & ~7
                N = (s0 + nr - b8 + 15) & ~15
                assert 16 <= N <= 144 and N % 16 == 0
                rows_alloc = max((nF + 7) & ~7, b8 + N)
                assert rows_alloc % 8 == 0 and rows_alloc <= 136
                if nF <= 32 and rows_alloc * kbytes * 8 <= stage_bytes:
                    KB = 8
                elif nF <= 64 and rows_alloc * kbytes * 4 <= stage_bytes:
                    KB = 4
                else:
                    KB = 2
                kb_bytes = rows_alloc * kbytes
                assert kb_bytes % 1024 == 0 and KB * kb_bytes <= stage_bytes
                nrw = (nF + 7) // 8
                assert nrw * KB <= 32
                last = (stages - 1) * stage_bytes + (KB - 1) * kb_bytes
                a_end = last + 128 * kbytes
                b_end = last + (b8 + N) * kbytes
                worst = max(worst, a_end, b_end)
    # the aligned base lies at most align - 1 bytes into the allocation
    assert worst + align - 1 <= smem


def test_oracle_parse_matches_read_fimi_on_random_bytes(oracle_mod, tmp_path):
    """The oracle's parse (the restated reference scanner, the checker of the GPU parse)
    and the numpy reader agree on the golden input files and on random byte strings over
    digits, '-', separators, CR and LF."""
    names = sorted(f for f in os.listdir(os.path.join(ROOT, "tests", "golden")) if f.endswith(".txt"))
    paths = [os.path.join(ROOT, "tests", "golden", f) for f in names]
    rng = np.random.Generator(np.random.PCG64(11))
    for k in range(20):
        out = bytearray()
        n = int(rng.integers(0, 3000))
        while len(out) < n:
            if rng.random() < 0.55:
                out += bytes(rng.integers(48, 58, size=int(rng.integers(1, 19))).tolist())
            else:
                out += b" \t\r\n-,x\n"[int(rng.integers(0, 8)):][:1]
        p = tmp_path / f"r{k}.txt"
        p.write_bytes(bytes(out[:n]))
        paths.append(str(p))
    for path in paths:
        a_off, a_items = oracle_mod.parse_file(path)
        b_off, b_items = tf.read_fimi(path)
        assert a_off.tolist() == b_off.tolist(), path
        assert a_items.tolist() == b_items.tolist(), path


def test_dense_lop3_pair_blocks_cover_each_pair_once():
    """The dense-family tile of csrc/count_lop3.cu (lop3_dense_impl), restated: for every tile
    shape the pack emits (1-8 rows x 1-64 columns) and the row block chosen by its row count,
    the pair blocks of a 256-thread block cover every (row, column) pair of the tile exactly
    once, every thread index maps to at most one block, at least 8 threads share a block, and
    every shared-memory sum index stays inside the 8 x 64 accumulator."""
    threads = 256
    br_of = {1: 1, 2: 2, 3: 3, 4: 4, 5: 3, 6: 3, 7: 4, 8: 4}
    bc_of = {1: 16, 2: 8, 3: 5, 4: 4}
    for nr in range(1, 9):
        BR = br_of[nr]
        BC = bc_of[BR]
        for nc in range(1, 65):
            rb, cb = -(-nr // BR), -(-nc // BC)
            nb = rb * cb
            assert nb <= 32
            G = threads // nb
            assert G >= 8
            seen = {}
            for tid in range(threads):
                b = tid // G
                if b >= nb:
                    continue
                br, bc = (b // cb) * BR, (b % cb) * BC
                for x in range(BR):
                    for y in range(BC):
                        r, c = br + x, bc + y
                        # loads are clamped to the last row / column; only in-tile pairs are summed
                        assert min(r, nr - 1) < nr and min(c, nc - 1) < nc
                        if r < nr and c < nc:
                            assert r * 64 + c < 8 * 64
                            seen.setdefault((r, c), set()).add(b)
            assert len(seen) == nr * nc, (nr, nc)
            assert all(len(v) == 1 for v in seen.values()), (nr, nc)


def test_pack_tile_groups_map_back_to_their_jobs():
    """The resident pack's CUDA-core tile order (csrc/resident.cu res_pack), restated: dense,
    heavy and light jobs get exclusive prefix sums of their tile counts within their own group
    (jobs of other groups add zero), tiles are numbered [dense | heavy | light], and the binary
    search for the last job whose prefix is <= the tile's index within its group
    (find_job_by_tile) returns the job that owns the tile, with every tile of every job found
    exactly once."""
    rng = np.random.Generator(np.random.PCG64(3))
    for _ in range(200):
        nj = int(rng.integers(1, 40))
        grp = rng.integers(0, 3, size=nj)            # 0 dense, 1 heavy, 2 light
        ntiles = rng.integers(0, 6, size=nj)
        pref = np.zeros((3, nj), np.int64)
        tot = [0, 0, 0]
        for j in range(nj):
            for g in range(3):
                pref[g, j] = tot[g]
            tot[grp[j]] += int(ntiles[j])

        def find(g, t):
            lo, hi = 0, nj - 1
            while lo < hi:
                mid = (lo + hi + 1) >> 1
                if pref[g, mid] <= t:
                    lo = mid
                else:
                    hi = mid - 1
            return lo

        owned = {}
        starts = [0, tot[0], tot[0] + tot[1]]
        for t in range(sum(tot)):
            g = 0 if t < starts[1] else 1 if t < starts[2] else 2
            j = find(g, t - starts[g])
            local = t - starts[g] - pref[g, j]
            assert grp[j] == g and 0 <= local < ntiles[j]
            owned.setdefault(j, []).append(local)
        for j in range(nj):
            assert sorted(owned.get(j, [])) == list(range(int(ntiles[j])))


def test_header_is_plain_c_and_links(tmp_path):
    """include/tfim.h compiles as C99 and a C program links against libtfim.so and calls the
    entry points that need no GPU (version, tuning table, argument checks), as a cgo / FFI
    binding of the reference's side would."""
    import shutil
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    src = tmp_path / "abi.c"
    src.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "tfim.h"
int main(void) {
    tfim_tuning t;
    tfim_tuning_get(&t);
    if (t.wave_rows < 16 || t.l3_dense_slices_per_sm <= 0.f) return 2;
    tfim_ctx* ctx = 0;
    const int64_t off[2] = {0, 2};
    const int32_t items[2] = {1, 2};
    if (tfim_open_db(off, items, 1, 1.5, 0, &ctx) != TFIM_E_INVALID || ctx) return 3;
    int64_t rows = 0, n = 0;
    if (tfim_parse_text(0, -1, 0, 0, 0, 0, 0, &rows, &n) != TFIM_E_INVALID) return 4;
    printf("%s\n", tfim_version());
    return 0;
}
''')
    exe = tmp_path / "abi"
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L", lib_dir, "-ltfim", "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "sm_100a" in r.stdout, (r.returncode, r.stdout, r.stderr)
