"""Per-size-class autotuner for the batched decryption path.

The kernel launchers choose their shapes from cost models (Pippenger window
width and segment count, lanes per GT exponentiation in the transforms,
joint or lane-split G1/G2 transform stages).  A cost model is only as good as
its constants, and the best choice moves with the batch size and with how
many batches share a launch.  For each size class the autotuner times a few
candidate knob settings on a trial group of that class (coordinate descent
from the cost models' own choice: GT lanes, then the transform mode, then
the window width), keeps the fastest, and caches it in a JSON file keyed by
GPU name, scheme, class size and committee size, so later runs reuse it.

Results never depend on the knobs (every launch configuration computes the
same canonical values); the tests check the decryptions under tuned knobs.
"""
from __future__ import annotations

import json
import os
import threading
from typing import Dict, List, Optional

from . import _lib
from . import weighted_btx as wb

DEFAULT_PATH = os.path.join(os.path.expanduser("~"), ".cache", "wbte", "autotune.json")
KNOBS = ("gt_lanes", "ntt_joint", "msm_window")
DEFAULTS = {"gt_lanes": 0, "ntt_joint": -1, "msm_window": 0, "msm_segments": 0}


def default_window(n: int) -> int:
    """The Pippenger window width the MSM cost model picks for n terms."""
    lg = max(0, n.bit_length() - 1)
    c = lg - 1 if n < (1 << 14) else lg - 2
    return max(4, min(13, c))


def candidates(knob: str, B: int) -> List[int]:
    if knob == "gt_lanes":
        return [1, 2, 4]
    if knob == "ntt_joint":
        return [0, 1]
    if knob == "msm_window":
        c = default_window(B)
        return [w for w in (c - 1, c + 1) if 4 <= w <= 13]
    return []


class Autotuner:
    """Picks and caches the knobs of each size class (thread-safe)."""

    def __init__(self, path: Optional[str] = DEFAULT_PATH, trial_batches: int = 8, enabled: bool = True):
        self.path = path
        self.trial_batches = max(1, int(trial_batches))
        self.enabled = enabled
        self._lock = threading.Lock()
        self._table: Dict[str, dict] = {}
        self.trials: Dict[str, list] = {}
        if path and os.path.exists(path):
            try:
                with open(path) as f:
                    self._table = json.load(f)
            except (OSError, ValueError):
                self._table = {}

    def _key(self, scheme: str, B: int, T: int) -> str:
        torch = wb._t()
        name = torch.cuda.get_device_name(torch.cuda.current_device()).replace(" ", "_")
        return f"{name}|{scheme}|B={B}|T={T}"

    def _save(self):
        if not self.path:
            return
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            tmp = self.path + f".{os.getpid()}.tmp"
            with open(tmp, "w") as f:
                json.dump(self._table, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except OSError:
            pass

    def lookup(self, scheme: str, B: int, T: int) -> Optional[dict]:
        with self._lock:
            return self._table.get(self._key(scheme, B, T))

    def knobs_for(self, B: int, size_class, decryptor) -> dict:
        """The knobs of weighted_pfe class B, tuned on first use: the trial
        group is `trial_batches` batches of the class's dummy ciphertexts
        decrypted by the class's committee on the calling thread's stream."""
        T = len(size_class.party_keys)
        key = self._key("wpfe", B, T)
        with self._lock:
            hit = self._table.get(key)
        if hit is not None or not self.enabled:
            return dict(hit or {})
        from . import wpfe_batched as wpb

        pool = size_class.dummies
        trial = [[pool[(t * B + i) % len(pool)] for i in range(B)] for t in range(self.trial_batches)]
        rng_seed = 12345

        def run(knobs: dict) -> float:
            torch = wb._t()
            ctx = wb._ctx()
            wpb._apply_knobs(ctx, knobs)
            try:
                stream = torch.cuda.current_stream()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                out = wpb.decrypt_group(size_class.material.encryption_key, size_class.material.decryption_key,
                                        trial, size_class.party_keys, _rng(rng_seed), decryptor.cache,
                                        device_output=True)
                b.record(stream)
                b.synchronize()
                for o in out:
                    if isinstance(o, BaseException):
                        raise o
                return a.elapsed_time(b)
            finally:
                wpb._apply_knobs(ctx, {})

        run(dict(DEFAULTS))  # warm-up: committee preparation, twiddles, tables
        best = dict(DEFAULTS)
        best_ms = run(best)
        log = [(dict(best), best_ms)]
        for knob in KNOBS:
            for v in candidates(knob, B):
                trial_knobs = dict(best)
                trial_knobs[knob] = v
                ms = run(trial_knobs)
                log.append((dict(trial_knobs), ms))
                if ms < best_ms * 0.97:
                    best, best_ms = trial_knobs, ms
        best = dict(best)
        best["trial_ms"] = round(best_ms, 3)
        best["trial_batches"] = self.trial_batches
        with self._lock:
            self._table[key] = best
            self.trials[key] = log
            self._save()
        return dict(best)


def _rng(seed: int):
    from .rng import ChaCha20Rng

    return ChaCha20Rng.seed_from_u64(seed)


def knob_values(knobs: dict) -> dict:
    """The library knobs of a tuned entry (drops bookkeeping fields)."""
    return {k: int(knobs.get(k, DEFAULTS[k])) for k in DEFAULTS}


__all__ = ["Autotuner", "DEFAULT_PATH", "knob_values", "default_window", "candidates", "_lib"]
