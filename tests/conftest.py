import gzip
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
# the reference project checkout, present only where it is mounted
REFERENCE = os.environ.get("TFIM_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def golden_names():
    return sorted(f[:-8] for f in os.listdir(GOLDEN) if f.endswith(".json.gz"))


def load_golden(name):
    with gzip.open(os.path.join(GOLDEN, name + ".json.gz"), "rt") as f:
        fx = json.load(f)
    fx["expected"] = {frozenset(s): f for s, f in fx["mfis"]}
    return fx


def load_golden_full(name):
    """A full-size fixture of tests/golden/full (the reference's output on a full-size
    benchmark database)."""
    with gzip.open(os.path.join(GOLDEN, "full", name + ".json.gz"), "rt") as f:
        fx = json.load(f)
    fx["expected"] = {frozenset(s): f for s, f in fx["mfis"]}
    return fx


def golden_input(fx, tmpdir):
    """Path of the fixture's transaction file (synthetic ones are regenerated from their seed)."""
    spec = fx["spec"]
    if spec["kind"] == "file":
        return os.path.join(GOLDEN, spec["file"])
    from tensorfim_b200 import synth
    db = synth.generate(spec["config"], **spec["kwargs"])
    path = os.path.join(str(tmpdir), "cfg%d.txt" % spec["config"])
    synth.write_fimi(path, db)
    return path


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    if not os.path.exists(oracle.LIB):
        oracle.build()
    return oracle
