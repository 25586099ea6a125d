"""Measurement helpers of the benchmark: roofline figures per counting path, peaks, and SM
clock sampling during a timed region.

Units (one support = popc(prefix mask & item row) over the N transactions):
  * bit-ops = supports x N, the reference microbenchmark's unit (bmma_bench.cu:400);
  * algorithmic bytes of a count job = (N/8)(rows + columns + base rows) + 4 rows columns:
    every operand row read once as a dense row, every count written once.
Each path is reported against the roof that bounds it: the CUDA-core AND+popc tiles and
the pair counter against HBM bandwidth (and the popc pipe, for the former), the tensor-core
paths against the tensor pipe (the measured int8 GEMM rate: one bit-op is one multiply-
accumulate of two 0/1 operands).
"""
from __future__ import annotations

import json
import os
import statistics
import subprocess
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATHS = ["lop3", "b1", "tc", "pairs", "proj", "gram"]
KERNELS = {"lop3": "k_count_lop3", "b1": "k_count_b1", "tc": "k_count_fam", "pairs": "k_pair_count",
           "proj": "k_count_proj", "gram": "k_count_gram"}
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def peaks() -> tuple[dict, str]:
    """The driver-measured peaks of this pool's B200s, else the recipe's fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return dict(PEAKS_FALLBACK), "fallback"


def popc_ceiling(sm_count: int = 148, sm_mhz: float = 1965.0) -> float:
    """Bit-ops/s of the CUDA-core AND+popc tiles at one 32-bit POPC per lane of 16 per SM and
    clock: each POPC counts 32 bit-ops."""
    return sm_count * 16 * 32 * sm_mhz * 1e6


def path_rooflines(stats: list[dict], hbm_gbs: float, i8_macs: float | None, sm_mhz: float = 1965.0,
                   sm_count: int = 148, traffic: dict | None = None) -> dict:
    """Per counting path over the given mines (tfim_mine_stats as dicts): launches, device
    time, algorithmic bytes and bit-ops per launch, achieved rates and their fractions.
    `traffic[path]` is DRAM bytes per algorithmic byte from an ncu capture (or absent)."""
    out = {}
    for q, name in enumerate(PATHS):
        ms = sum(s["path_ms"][q] for s in stats)
        if ms <= 0:
            continue
        launches = max(1, sum(s["path_launches"][q] for s in stats))
        by = sum(s["path_bytes"][q] for s in stats)
        bo = sum(s["path_bitops"][q] for s in stats)
        sec = ms / 1000.0
        gbs = by / sec / 1e9
        e = {"kernel": KERNELS[name], "launches": launches, "ms_per_launch": ms / launches,
             "bytes_alg_per_launch": by / launches, "bitops_per_launch": bo / launches,
             "achieved_gbs": gbs, "hbm_frac": gbs / hbm_gbs, "bitops_per_s": bo / sec if bo else 0.0,
             "share_of_counting": None}
        if name in ("lop3", "gram"):
            e["popc_frac"] = (bo / sec) / popc_ceiling(sm_count, sm_mhz)
        if name in ("b1", "tc") and i8_macs:
            e["tensor_frac"] = (bo / sec) / i8_macs
        if traffic and name in traffic and traffic[name]:
            e["traffic_per_launch"] = traffic[name] * by / launches
        out[name] = e
    tot = sum(v["ms_per_launch"] * v["launches"] for v in out.values())
    for v in out.values():
        v["share_of_counting"] = v["ms_per_launch"] * v["launches"] / tot if tot else None
    return out


def headline_roofline(paths: dict, hbm_gbs: float, i8_macs: float | None, peak_src: str, i8_src: str) -> dict | None:
    """The roofline object of the dominant counting path (the most device time)."""
    if not paths:
        return None
    name, e = max(paths.items(), key=lambda kv: kv[1]["ms_per_launch"] * kv[1]["launches"])
    if name in ("b1", "tc") and i8_macs:
        ach = 2.0 * e["bitops_per_s"] / 1e12
        peak = 2.0 * i8_macs / 1e12
        r = {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
             "peak_source": i8_src}
    else:
        r = {"bound": "hbm", "achieved": e["achieved_gbs"], "peak": hbm_gbs, "unit": "GB/s",
             "frac": e["achieved_gbs"] / hbm_gbs, "peak_source": peak_src}
    r.update({"kernel": e["kernel"], "path": name, "traffic": e.get("traffic_per_launch"),
              "bytes_alg_per_launch": e["bytes_alg_per_launch"], "bitops_per_launch": e["bitops_per_launch"],
              "ms_per_launch": e["ms_per_launch"]})
    return r


class Clocks:
    """SM clocks and throttle reasons sampled every `period_s` while a region runs: NVML
    from a thread, or `nvidia-smi -lms` when NVML is unavailable."""
    # clocks event reason bits (nvml.h)
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, index: int, period_s: float = 0.02):
        self.index, self.period = index, period_s
        self.samples, self.maxes, self.reasons = [], [], set()
        self._stop = threading.Event()
        self._proc = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self._nv = None
            self._f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            try:
                q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                     "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
                self._proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                               "--format=csv,noheader,nounits", "-lms", "100"],
                                              stdout=self._f, stderr=subprocess.DEVNULL)
            except Exception:
                self._proc = None

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                self.maxes.append(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
                try:
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                except AttributeError:
                    bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                for b, name in self.REASONS.items():
                    if bits & b:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def stop(self) -> dict:
        if self._nv is not None:
            self._stop.set()
            self._t.join(timeout=5)
            src = "nvml"
        else:
            src = "nvidia-smi"
            if self._proc is None:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
            time.sleep(0.2)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            self._f.seek(0)
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for ln in self._f.read().splitlines():
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) < 6:
                    continue
                try:
                    self.samples.append(float(parts[0]))
                    self.maxes.append(float(parts[1]))
                except ValueError:
                    continue
                for k, name in enumerate(names):
                    if parts[2 + k].lower() == "active":
                        self.reasons.add(name)
            self._f.close()
            os.unlink(self._f.name)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": max(self.maxes) if self.maxes else None, "reasons": sorted(self.reasons),
                "samples": len(self.samples), "source": src}


def i8_gemm_peak(device, n: int = 8192, reps: int = 10) -> float | None:
    """Measured dense int8 GEMM rate (multiply-accumulates per second) of torch._int_mm
    (cuBLASLt) on `device`: the tensor-pipe roof of the kind::i8 counter, whose bit-ops are
    0/1 multiply-accumulates.  None when the call is unavailable."""
    import torch
    try:
        a = torch.randint(-8, 8, (n, n), dtype=torch.int8, device=device)
        b = torch.randint(-8, 8, (n, n), dtype=torch.int8, device=device)
        for _ in range(3):
            torch._int_mm(a, b)
        torch.cuda.synchronize(device)
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1) / 1000.0
            best = t if best is None else min(best, t)
        del a, b
        return float(n) ** 3 / best
    except Exception:
        return None
