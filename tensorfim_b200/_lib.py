"""ctypes binding of libtfim.so (include/tfim.h).

The library is loaded from tensorfim_b200/_lib/; there is no fallback implementation:
if it is missing or a call fails, a TfimError is raised.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libtfim.so")
CLI_PATH = os.path.join(HERE, "_lib", "tfim")

TFIM_OK = 0
TFIM_E_INVALID = 1
TFIM_E_CUDA = 2
TFIM_E_NOMEM = 3
TFIM_E_DEPTH = 4
TFIM_E_TIMEOUT = 5
TFIM_E_STATE = 6
TFIM_E_IO = 7
TFIM_E_COMM = 8

ENGINE_PLAIN = 0
ENGINE_BATCHED = 1
ENGINE_RESIDENT = 2
COUNTER_AUTO = 0
COUNTER_LOP3 = 1
COUNTER_TENSOR = 2
COUNTER_PROJ = 3
COUNTER_I8 = 4
DT_I32 = 0
DT_I64 = 1
RED_SUM = 0
RED_MIN = 1
RED_MAX = 2

# every entry point declared in include/tfim.h
EXPORTS = [
    "tfim_version", "tfim_last_error", "tfim_open_db", "tfim_open_bitmap", "tfim_db_info_get",
    "tfim_dense_to_orig", "tfim_dense_freq", "tfim_count_wave", "tfim_set_counter",
    "tfim_count_wave_device", "tfim_mine_opts_default", "tfim_mine", "tfim_num_mfis",
    "tfim_mfi_item_total", "tfim_get_mfis", "tfim_write_results", "tfim_close",
    "tfim_count_wave_noalloc", "tfim_open_db_sharded", "tfim_open_bitmap_sharded",
    "tfim_mlp_create", "tfim_mlp_num_params", "tfim_mlp_set_params", "tfim_mlp_get_params", "tfim_mlp_predict",
    "tfim_mlp_grad", "tfim_mlp_train", "tfim_mlp_free", "tfim_set_proposal", "tfim_lookahead_log",
    "tfim_tuning_get", "tfim_tuning_set", "tfim_tuning_load", "tfim_tuning_source",
    "tfim_mine_all", "tfim_num_all", "tfim_all_item_total", "tfim_get_all", "tfim_release_cached",
    "tfim_open_text", "tfim_open_file", "tfim_parse_text",
]


class TfimError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"tfim error {code}: {msg}")
        self.code = code


class DbInfo(C.Structure):
    _fields_ = [
        ("trans_num", C.c_int64), ("dimension", C.c_int64), ("item_id_min", C.c_int64),
        ("item_id_max", C.c_int64), ("item_id_max_dense", C.c_int64),
        ("trans_len_min", C.c_int64), ("trans_len_max", C.c_int64), ("trans_len_mean", C.c_double),
        ("trans_num_reduced", C.c_int64), ("trans_len_red_min", C.c_int64), ("trans_len_red_max", C.c_int64),
        ("trans_len_red_mean", C.c_double), ("dimension_reduced", C.c_int64),
        ("support_threshold", C.c_double), ("frequency_threshold", C.c_double),
        ("min_count", C.c_int32), ("n_survivors", C.c_int32), ("n_dense", C.c_int32), ("words_per_row", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class MineOpts(C.Structure):
    _fields_ = [("engine", C.c_int32), ("counter", C.c_int32), ("wave_cap", C.c_int32),
                ("lookahead", C.c_int32), ("use_graphs", C.c_int32), ("top_counter", C.c_int32),
                ("log_lookahead", C.c_int32), ("proj_auto", C.c_int32), ("small_pools", C.c_int32),
                ("superset", C.c_int32), ("reserved", C.c_int32 * 6)]


class Tuning(C.Structure):
    _fields_ = [("wave_rows", C.c_int32), ("l3_slices_per_sm", C.c_float), ("b1_tiles_per_sm", C.c_float),
                ("b1_min_rows", C.c_int32), ("b1_min_cols", C.c_int32), ("proj_auto", C.c_int32),
                ("rate_b1_bitops", C.c_double), ("rate_lop3_bitops", C.c_double), ("rate_pair_incr", C.c_double),
                ("i8_min_rows", C.c_int32), ("i8_min_cols", C.c_int32), ("rate_i8_bitops", C.c_double),
                ("tc_min_work", C.c_int32), ("tc_min_density", C.c_float), ("tc_tiles_per_sm", C.c_float),
                ("gram_min_rows", C.c_int32), ("l3_dense_slices_per_sm", C.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# int allreduce(void* buf, int64_t count, int32_t dtype, int32_t op, void* stream, void* user)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p)


class Group(C.Structure):
    _fields_ = [("rank", C.c_int32), ("world", C.c_int32), ("allreduce", ALLREDUCE_FN), ("user", C.c_void_p)]


class MineStats(C.Structure):
    _fields_ = [("mine_seconds", C.c_double), ("device_ms", C.c_double), ("kernel_ms", C.c_double),
                ("nodes", C.c_int64), ("supports", C.c_int64), ("bit_ops", C.c_int64), ("bytes_alg", C.c_int64),
                ("waves", C.c_int64), ("launches", C.c_int64), ("count_launches", C.c_int64),
                ("lookaheads", C.c_int64), ("lookahead_hits", C.c_int64), ("pruned_pep", C.c_int64),
                ("n_mfi", C.c_int64), ("host_ms", C.c_double), ("sync_ms", C.c_double),
                ("lookaheads_skipped", C.c_int64), ("top_ms", C.c_double), ("pruned_superset", C.c_int64),
                ("path_ms", C.c_double * 6), ("path_bytes", C.c_int64 * 6), ("path_bitops", C.c_int64 * 6),
                ("path_supports", C.c_int64 * 6), ("path_launches", C.c_int64 * 6),
                ("pack_ms", C.c_double), ("expand_ms", C.c_double), ("mask_ms", C.c_double), ("zero_ms", C.c_double),
                ("setup_ms", C.c_double), ("readback_ms", C.c_double)]

    def as_dict(self) -> dict:
        out = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            out[k] = list(v) if k.startswith("path_") else v
        return out


# counting paths of MineStats.path_* (include/tfim.h TFIM_PATH_*)
PATHS = ["lop3", "b1", "tc", "pairs", "proj", "gram"]


_lib = None


def lib() -> C.CDLL:
    """Load libtfim.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise TfimError(-1, f"{LIB_PATH} is missing: build it with `python -m tensorfim_b200.build`")
    L = C.CDLL(LIB_PATH)
    p = C.c_void_p
    i32, i64 = C.c_int32, C.c_int64
    P = C.POINTER
    L.tfim_version.restype = C.c_char_p
    L.tfim_last_error.restype = C.c_char_p
    L.tfim_open_db.argtypes = [p, p, i64, C.c_double, i32, P(p)]
    L.tfim_open_bitmap.argtypes = [p, i32, i64, i32, i32, P(p)]
    L.tfim_open_text.argtypes = [p, i64, C.c_double, i32, P(p)]
    L.tfim_open_file.argtypes = [C.c_char_p, C.c_double, i32, P(p)]
    L.tfim_parse_text.argtypes = [p, i64, i32, p, i64, p, i64, P(i64), P(i64)]
    L.tfim_db_info_get.argtypes = [p, P(DbInfo)]
    L.tfim_dense_to_orig.argtypes = [p, p]
    L.tfim_dense_freq.argtypes = [p, p]
    L.tfim_count_wave.argtypes = [p, p, p, i32, i32, p, p]
    L.tfim_set_counter.argtypes = [p, i32]
    L.tfim_count_wave_device.argtypes = [p, p, p, i32, i32, i32, p, p, p]
    L.tfim_count_wave_noalloc.argtypes = [p, i64, i32, p, p, i32, i32, p, p, p]
    L.tfim_mine_opts_default.argtypes = [P(MineOpts)]
    L.tfim_mine_opts_default.restype = None
    L.tfim_mine.argtypes = [p, P(MineOpts), P(MineStats)]
    L.tfim_release_cached.argtypes = [i32]
    L.tfim_num_mfis.argtypes = [p]
    L.tfim_num_mfis.restype = i64
    L.tfim_mfi_item_total.argtypes = [p]
    L.tfim_mfi_item_total.restype = i64
    L.tfim_get_mfis.argtypes = [p, p, p, p]
    L.tfim_write_results.argtypes = [p, C.c_char_p, C.c_char_p, C.c_double, C.c_double]
    L.tfim_close.argtypes = [p]
    L.tfim_close.restype = None
    L.tfim_mlp_create.argtypes = [i32, C.c_uint64, P(p)]
    L.tfim_mlp_set_params.argtypes = [p, p]
    L.tfim_mlp_get_params.argtypes = [p, p]
    L.tfim_mlp_predict.argtypes = [p, p, i64, p]
    L.tfim_mlp_grad.argtypes = [p, p, p, i64, C.c_float, p, p]
    L.tfim_mlp_train.argtypes = [p, p, p, i64, i32, i32, C.c_float, C.c_float, C.c_float, p]
    L.tfim_mlp_free.argtypes = [p]
    L.tfim_mlp_free.restype = None
    L.tfim_set_proposal.argtypes = [p, p, C.c_float]
    L.tfim_lookahead_log.argtypes = [p, p, p, i64]
    L.tfim_lookahead_log.restype = i64
    L.tfim_tuning_get.argtypes = [P(Tuning)]
    L.tfim_tuning_get.restype = None
    L.tfim_tuning_set.argtypes = [P(Tuning)]
    L.tfim_tuning_load.argtypes = [C.c_char_p]
    L.tfim_tuning_source.restype = C.c_char_p
    L.tfim_mine_all.argtypes = [p, i32, i32, i64, P(MineStats)]
    L.tfim_num_all.argtypes = [p]
    L.tfim_num_all.restype = i64
    L.tfim_all_item_total.argtypes = [p]
    L.tfim_all_item_total.restype = i64
    L.tfim_get_all.argtypes = [p, p, p, p]
    L.tfim_open_db_sharded.argtypes = [p, p, i64, C.c_double, i32, P(Group), P(p)]
    L.tfim_open_bitmap_sharded.argtypes = [p, i32, i64, i32, i32, P(Group), P(p)]
    for name in EXPORTS:
        getattr(L, name)   # raises AttributeError if an export is missing
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != TFIM_OK:
        raise TfimError(rc, lib().tfim_last_error().decode(errors="replace"))
