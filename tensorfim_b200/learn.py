"""Learned lookahead proposal: data collection, GPU training, weights on disk.

The exact engine logs, for every head-union-tail lookahead it issues, the node's 32
features and the outcome (1 = head + tail was frequent).  A 32 -> 64 -> 64 -> 1 MLP
(BF16 weights, FP32 accumulation) is trained on those logs by the library's own CUDA
kernels (tfim_mlp_train: forward, backward and Adam on the GPU).  With
``Database.mine(lookahead="learned")`` the engine then issues a lookahead first only for
nodes the network scores >= threshold; all other nodes are expanded directly.  Supports
are always counted exactly, so the MFI output is the same with or without the network.

Training data: the generators of benchmark configurations 1-3 at seeds 100-119 (their
own minimum supports), mined with the lookahead on every node that passes the exact
tail-pair filter.

    python -m tensorfim_b200.learn            # collect, train, write proposal_weights.bin
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib, synth
from ._lib import check, lib
from .engine import Database

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "proposal_weights.bin")
MAGIC = b"TFIMMLP1"
N_FEATURES = 32


class Proposal:
    """A tfim_mlp on one GPU."""

    def __init__(self, device: int = 0, seed: int = 0):
        self._h = C.c_void_p()
        check(lib().tfim_mlp_create(device, seed, C.byref(self._h)))
        self.n_params = lib().tfim_mlp_num_params()
        self.threshold = 0.5

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        check(lib().tfim_mlp_get_params(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.shape == (self.n_params,)
        check(lib().tfim_mlp_set_params(self._h, p.ctypes.data_as(C.c_void_p)))

    def predict(self, feats: np.ndarray) -> np.ndarray:
        feats = np.ascontiguousarray(feats, dtype=np.float32).reshape(-1, N_FEATURES)
        out = np.zeros(feats.shape[0], np.float32)
        if feats.shape[0]:
            check(lib().tfim_mlp_predict(self._h, feats.ctypes.data_as(C.c_void_p), feats.shape[0],
                                         out.ctypes.data_as(C.c_void_p)))
        return out

    def grad(self, feats: np.ndarray, labels: np.ndarray, pos_weight: float = 1.0) -> tuple[np.ndarray, float]:
        feats = np.ascontiguousarray(feats, dtype=np.float32).reshape(-1, N_FEATURES)
        labels = np.ascontiguousarray(labels, dtype=np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float()
        check(lib().tfim_mlp_grad(self._h, feats.ctypes.data_as(C.c_void_p), labels.ctypes.data_as(C.c_void_p),
                                  feats.shape[0], pos_weight, g.ctypes.data_as(C.c_void_p), C.byref(loss)))
        return g, float(loss.value)

    def train(self, feats: np.ndarray, labels: np.ndarray, epochs: int = 40, batch: int = 256, lr: float = 3e-3,
              pos_weight: float | None = None, weight_decay: float = 1e-4, seed: int = 0) -> float:
        feats = np.ascontiguousarray(feats, dtype=np.float32).reshape(-1, N_FEATURES)
        labels = np.ascontiguousarray(labels, dtype=np.float32)
        if pos_weight is None:
            pos = float(labels.sum())
            pos_weight = float(np.clip((labels.size - pos) / max(pos, 1.0), 1.0, 50.0))
        order = np.random.Generator(np.random.PCG64(seed)).permutation(feats.shape[0])
        fx, ly = feats[order], labels[order]
        loss = C.c_float()
        check(lib().tfim_mlp_train(self._h, fx.ctypes.data_as(C.c_void_p), ly.ctypes.data_as(C.c_void_p), fx.shape[0],
                                   epochs, batch, lr, pos_weight, weight_decay, C.byref(loss)))
        return float(loss.value)

    def save(self, path: str = WEIGHTS) -> None:
        """Raw little-endian file: magic "TFIMMLP1", int32 n_params, float32 threshold,
        float32 params[n_params] (read by the `tfim` command line too)."""
        p = self.params()
        with open(path, "wb") as f:
            f.write(MAGIC)
            f.write(np.int32(p.shape[0]).tobytes())
            f.write(np.float32(self.threshold).tobytes())
            f.write(p.astype("<f4").tobytes())

    @classmethod
    def load(cls, path: str = WEIGHTS, device: int = 0) -> "Proposal":
        blob = open(path, "rb").read()
        if blob[:8] != MAGIC:
            raise ValueError(f"{path}: not a proposal weights file")
        n = int(np.frombuffer(blob[8:12], "<i4")[0])
        thr = float(np.frombuffer(blob[12:16], "<f4")[0])
        params = np.frombuffer(blob[16:16 + 4 * n], "<f4").copy()
        prop = cls(device)
        prop.set_params(params)
        prop.threshold = thr
        return prop

    def close(self) -> None:
        if self._h:
            lib().tfim_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


TRAIN_CONFIGS = (1, 2, 3)
TRAIN_SEEDS = range(100, 120)
MINSUP = {1: 0.10, 2: 0.90, 3: 0.85}


def collect(configs=TRAIN_CONFIGS, seeds=TRAIN_SEEDS, device: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Mine each training database with logging on; return the features and outcomes of
    every lookahead the exact engine issued."""
    xs, ys = [], []
    for cfg in configs:
        for seed in seeds:
            db0 = synth.training_db(cfg, seed)
            with Database.from_csr(db0.offsets, db0.items, MINSUP[cfg], device) as db:
                db.mine(lookahead="filtered", log_lookahead=True)
                x, y = db.lookahead_log()
            xs.append(x)
            ys.append(y)
    return np.concatenate(xs) if xs else np.zeros((0, N_FEATURES), np.float32), np.concatenate(ys) if ys else np.zeros(0, np.float32)


def choose_threshold(probs: np.ndarray, labels: np.ndarray, miss_cost: float = 3.0, waste_cost: float = 1.0) -> float:
    """Score threshold minimising  miss_cost * (hits scored below it) + waste_cost *
    (misses scored above it) on the logged outcomes.  A lookahead that is skipped but would
    have hit costs the counts of the subtree it would have closed; one that is issued and
    misses costs one count and one wave of latency."""
    if labels.size == 0 or labels.sum() == 0:
        return 0.5
    best_t, best_c = 0.5, float("inf")
    for t in np.linspace(0.01, 0.99, 99):
        keep = probs >= t
        cost = miss_cost * float(((~keep) & (labels > 0.5)).sum()) + waste_cost * float((keep & (labels < 0.5)).sum())
        if cost < best_c:
            best_t, best_c = float(t), cost
    return best_t


def main() -> None:
    x, y = collect()
    print(f"collected {len(y)} lookahead outcomes, {int(y.sum())} hits")
    prop = Proposal(seed=1)
    loss = prop.train(x, y)
    p = prop.predict(x)
    prop.threshold = choose_threshold(p, y)
    kept = p >= prop.threshold
    print(f"final loss {loss:.4f}; threshold {prop.threshold:.3f}; keeps {int(kept.sum())}/{len(y)} lookaheads, "
          f"{int((kept & (y > 0.5)).sum())}/{int(y.sum())} hits")
    prop.save()
    print(f"wrote {WEIGHTS}")


if __name__ == "__main__":
    main()
