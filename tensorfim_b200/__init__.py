"""TensorFIM-B200: exact maximal-frequent-itemset mining on B200 (sm_100a).

A drop-in for the hap04210384/TensorFIM engines: same command line, same results file,
same counting contract; hand-written CUDA kernels behind a C ABI (include/tfim.h).
"""
from ._lib import TfimError, lib
from .engine import Database, MineResult, mine_file, parse_text, read_fimi, release_cached, result_path
from .results import compare, load_header, load_results

__all__ = ["Database", "MineResult", "TfimError", "lib", "mine_file", "parse_text", "read_fimi", "release_cached", "result_path",
           "compare", "load_header", "load_results"]
