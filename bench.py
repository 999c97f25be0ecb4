#!/usr/bin/env python
"""Benchmark: batched threshold decryption over BLS12-381 on B200.

Headline (the `value` of the JSON line): weighted_btx batch decryption, B =
512 ciphertexts per batch, n = 128 parties with Zipf(1) weights summing to W =
4096, authorized weight > W/3, heaviest-first minimal committee.  One batch
is the reference's decryption sequence: ciphertext validation, partial
decryption by every committee member, share acceptance, committee
preparation, cross-term precomputation and opening
(weighted_btx/examples/paper_reproduction.rs:240-340, plus validation).
Every form is bit-exact against the plaintexts (asserted after timing).

  plain         one batch per step on one stream, committee prepared every
                batch: the reference's `decrypt()` sequence, one batch at a time
  plain_cached  one batch per step, the committee preparation cached (the
                reference documents it as reusable for the same batch size and
                party set, weighted_btx/src/decryption.rs:424-426): the "plain
                one-batch-per-launch" GPU path with the same cache policy as
                the batched form, the like-for-like denominator of the
                batched/plain ratio
  value         the batched form: each step runs C groups concurrently on C
                CUDA streams (default 3), a group being G batches (default 128)
                whose every GPU phase is one launch over all of them; committee
                cached (the timed region starts with an empty cache, so its
                first group prepares)
  e2e           the served form through the public API (serving.DecryptionServer)
                with host ciphertext objects and host results: throughput with
                all requests submitted at once, and p50/p99 request latency
                under Poisson arrivals at half that rate (continuous batching)

Further sections (flat keys, so every figure survives in the parsed line):
  roofline / rooflines   the batched form's kernels on their own Fp-product
                counts (weighted_bte_b200/workcount.py) against the measured
                integer-pipe peak; `traffic` from the committed ncu capture
  wpfe_batched  the batched weighted_pfe form: 256 batches with sizes
                log-uniform in [8, 2048] (seed 3) padded to power-of-two
                classes, n = 64 Zipf(1) W = 2048, per-class autotuned knobs
  wpfe_served   the served weighted_pfe form: n = 1000 Pareto(1.2) W = 16384,
                every class 16..4096 resident, requests log-uniform in
                [16, 4096] (seed 4): burst capacity, the plain per-request
                path, p50/p99 under Poisson arrivals at 30/60/90 % of capacity
  sweep         the kernel sweep: G1/G2 MSM 2^10..2^20, G1/G2/GT transforms
                2^8..2^16, multi-pairings of k in {1, 16, 256, 4096} + one
                final exponentiation (seed 2), each with its own roofline
  cpu_baseline  the CPU restatement (oracle/) on the host cores at the same
                B = 512 with the committee preparation cached

Device times use CUDA events; L2 is flushed (256 MB write) before every step.
Multi-GPU: replicas only -- every rank decrypts its own batches with its own
copy of the public key; no collective on the data path (scaling "weak").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}]
                  [--concurrency C] [--group G] [--no-e2e] [--no-cpu-baseline]
                  [--no-wpfe] [--no-served] [--no-sweep]
"""
from __future__ import annotations

import argparse
import json
import os
import random
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# The batched form runs one CUDA stream per concurrent batch; CUDA maps streams
# onto this many hardware work queues (default 8), so more streams than queues
# serialise.  Read once, when the CUDA context is created.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

# Fp multiplication in the 12-limb CIOS kernel: 12 rows x (24 products for
# a*b_i + 24 for m*p + 1) 32-bit IMAD instructions (lo and hi halves).
IMAD_PER_FP_MUL = 12 * 49
METRIC = "ciphertexts decrypted/s (weighted_btx batch decryption, B=512)"
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "roofline_traffic.json")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--batch-size", type=int, default=512)
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed samples of the CPU arm (plus one warm-up)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-wpfe", action="store_true", help="skip the batched weighted_pfe section")
    ap.add_argument("--no-sweep", action="store_true", help="skip the kernel sweep")
    ap.add_argument("--no-plain", action="store_true", help="skip the one-batch-per-step arms (profiling runs)")
    ap.add_argument("--no-graph", action="store_true", help="skip the graph-replayed batched arm")
    ap.add_argument("--wpfe-passes", type=int, default=2, help="timed passes over the 256 weighted_pfe batches")
    ap.add_argument("--no-served", action="store_true", help="skip the served weighted_pfe section")
    ap.add_argument("--served-requests", type=int, default=48, help="requests per pass of the served section")
    ap.add_argument("--served-seconds", type=float, default=6.0, help="seconds of Poisson arrivals per rate")
    ap.add_argument("--concurrency", type=int, default=3, help="concurrent groups (streams) of the batched form")
    ap.add_argument("--group", type=int, default=128, help="batches per group (one launch sequence) in the batched form")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: str):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for name, flag in zip(names, parts[5:9]):
                    if flag.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def event_ms(torch, fn, stream=None):
    """Device milliseconds of fn() on the current stream (CUDA events)."""
    stream = stream or torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    out = fn()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b), out


def load_traffic() -> dict:
    try:
        with open(TRAFFIC_FILE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# --------------------------------------------------------------- CPU leg
class CpuArm:
    """The oracle's restatement of the weighted_btx decryption on the host
    cores, at the GPU arm's batch size with the committee preparation cached
    (prepared once, untimed, as the batched form does).  Timed per batch:
    validation, the committee's partial decryptions, the aggregate share
    check, precomputation and opening (weighted_btx/src/decryption.rs:85-709).

    The oracle's own keygen and committee preparation of this size (4.3 M
    fixed-base G2 products, then the preparation's G2 MSMs) take minutes on
    CPU, so the key material, the prepared committee and the ciphertexts are
    produced by the GPU library, whose outputs the parity tests hold
    byte-identical to the oracle's; only the decryption is timed."""

    def __init__(self, cfg, B: int, seed: int = 1):
        from oracle import oracle as O
        from weighted_bte_b200 import weighted_btx as wb
        from weighted_bte_b200.rng import ChaCha20Rng
        from weighted_bte_b200.workloads import minimal_authorized_parties

        O.lib()
        self.threads = O.num_threads()
        self.B = B
        rng = ChaCha20Rng.seed_from_u64(seed)
        mat = wb.keygen_with_rng(wb.KeygenConfig(B, cfg.weights, cfg.threshold), rng)
        dk = mat.decryption_key
        committee, _ = minimal_authorized_parties(cfg.weights, cfg.threshold)
        self.parties = sorted(committee)
        N = dk.party_count()
        vk = wb.to_host(dk.verification_keys, 192 * B * N)
        self.key = dict(N=N, vk=[vk[192 * i : 192 * (i + 1)] for i in range(B * N)], setup_id=dk.setup_id())
        self.qs = [mat.party_keys[j].secret_scalar() for j in self.parties]
        keys = [mat.party_keys[j] for j in self.parties]
        batch = wb.validate_batch(dk, wb.encrypt_many(mat.encryption_key, [wb.gt_generator()] * B, rng))
        acc = wb.accept_decryption_shares(dk, batch, wb.partial_decrypt_many(keys, batch), rng)
        pre = wb.prepare_decryption(dk, acc)
        m = wb.transform_size_for(B)
        kern = wb.to_host(pre.transformed_kernel, 192 * m)
        opening = wb.to_host(pre.opening_keys, 192 * B * len(self.parties))
        self.pre = dict(kernel=[kern[192 * i : 192 * (i + 1)] for i in range(m)],
                        opening=[opening[192 * i : 192 * (i + 1)] for i in range(B * len(self.parties))], m=m, B=B)
        self.mat, self.rng = mat, rng

    def sample(self, steps: int):
        from oracle import wbtx_oracle as W
        from weighted_bte_b200 import weighted_btx as wb

        times = []
        for _ in range(steps):
            msgs = wb.messages_from_bytes([self.rng.fill_bytes(32) for _ in range(self.B)])
            cts = wb.encrypt_many(self.mat.encryption_key, msgs, self.rng)
            octs = [dict(first=c.first, second=c.second, commitment=c.proof.commitment, response=c.proof.response)
                    for c in cts]
            challenges = [W.sample_nonzero(self.rng) for _ in self.parties]
            t0 = time.perf_counter()
            batch = W.validate(self.key["setup_id"], octs, self.threads)
            sig = [W.partial_decrypt(q, batch) for q in self.qs]
            ok = W.verify_shares(self.key, batch, self.parties, sig, challenges, self.threads)
            beta = W.precompute(self.pre, batch)
            out = W.open_batch(self.pre, sig, batch, octs, beta)
            times.append(time.perf_counter() - t0)
            assert ok and out == msgs, "CPU restatement failed its round trip"
        return times

    def describe(self) -> str:
        return (f"oracle decryption of one B={self.B} batch per step (validate + {len(self.parties)} partial "
                f"decryptions + aggregate share check + precompute + open; committee preparation cached, as in the "
                f"batched form; key material, prepared committee and ciphertexts made by the GPU library, "
                f"byte-identical to the oracle's), {self.threads} host threads")


def run_reference(args, cfg):
    """--impl reference: the CPU restatement of the reference path on all host
    threads (the Rust crates cannot be built here: no cargo/rustc)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    try:
        import torch

        if torch.cuda.is_available():
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    except ImportError:
        pass
    arm = CpuArm(cfg, args.batch_size)
    times = arm.sample(args.warmup + args.steps)
    timed = times[args.warmup:] or times
    value = args.batch_size / statistics.median(timed)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ciphertexts/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.median(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 limbs (Fp/Fr)",
        "data": "synthetic", "config": {"workload": cfg.name, "batch_size": args.batch_size,
                                        "form": "one batch per step, committee preparation cached"},
        "cpu_baseline": {"value": value, "unit": "ciphertexts/s", "cores": arm.threads, "kind": "port",
                         "sample": arm.describe()},
        "e2e": {"value": value, "unit": "ciphertexts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU arm
def make_batches(wb, mat, rng, B, count):
    """`count` fresh batches of B ciphertexts of random 32-byte plaintexts."""
    host, dev, plain = [], [], []
    for _ in range(count):
        msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
        cts = wb.encrypt_many(mat.encryption_key, msgs, rng)
        host.append(cts)
        dev.append(wb.CiphertextBatch.upload(cts))
        plain.append(msgs)
    return host, dev, plain


def run_batched(torch, fn, items, slots, steps, flush_buf):
    """Each step runs `slots` items concurrently, one per stream; between
    steps every stream waits for an L2 flush (a write of a buffer larger than
    L2) issued after all streams finished the previous step.  Returns the
    outputs and the device time from the first flush to the last step's
    completion (CUDA events)."""
    streams = [torch.cuda.Stream() for _ in range(slots)]
    main = torch.cuda.current_stream()
    gate = threading.Barrier(slots + 1)
    ends = [[None] * slots for _ in range(steps)]
    flush_ev = [None] * steps
    outs = [None] * len(items)
    errors = []
    device = torch.cuda.current_device()

    def worker(w):
        try:
            torch.cuda.set_device(device)
            s = streams[w]
            for k in range(steps):
                gate.wait()  # flush of step k enqueued
                s.wait_event(flush_ev[k])
                with torch.cuda.stream(s):
                    i = k * slots + w
                    outs[i] = fn(items[i])
                    e = torch.cuda.Event(enable_timing=True)
                    e.record(s)
                    ends[k][w] = e
                gate.wait()  # step k enqueued by every stream
        except BaseException as exc:  # noqa: BLE001
            errors.append(exc)
            gate.abort()

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(slots)]
    for t in threads:
        t.start()
    t0 = None
    try:
        for k in range(steps):
            if k:
                for e in ends[k - 1]:
                    main.wait_event(e)
            flush_buf.add_(1)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(main)
            if t0 is None:
                t0 = ev
            flush_ev[k] = ev
            gate.wait()
            gate.wait()
    except threading.BrokenBarrierError:
        pass
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    torch.cuda.synchronize()
    ms = max(t0.elapsed_time(e) for e in ends[-1])
    return outs, ms


def timed_steps(torch, fn, items, flush, stream):
    """One item per step on `stream`, L2 flushed before each; returns outputs
    and the summed device milliseconds of the steps (CUDA events)."""
    outs, total = [], 0.0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for it in items:
        flush.add_(1)
        ev0.record(stream)
        outs.append(fn(it))
        ev1.record(stream)
        torch.cuda.synchronize()
        total += ev0.elapsed_time(ev1)
    return outs, total


def roof(name, ms, products, peak, **extra):
    """A roofline entry: achieved G Fp products/s on the kernel's own count."""
    if not ms or ms <= 0:
        return {"kernel": name, "ms": ms, "achieved": None, "frac": None}
    achieved = products / (ms / 1000.0)
    out = {"kernel": name, "bound": "int", "unit": "G Fp products/s", "ms": round(ms, 3),
           "fp_products": int(products), "achieved": achieved / 1e9, "peak": peak / 1e9, "frac": achieved / peak}
    out.update(extra)
    return out


# ------------------------------------------------------- batched weighted_pfe
def wpfe_section(args, torch, wb, flush, world, max_over_ranks, barrier):
    """The batched weighted_pfe form over 256 uneven batches (seed 3)."""
    from weighted_bte_b200 import autotune
    from weighted_bte_b200 import weighted_pfe as wp
    from weighted_bte_b200 import wpfe_batched as wpb
    from weighted_bte_b200.rng import ChaCha20Rng
    from weighted_bte_b200.workloads import WPFE_BATCHED as cfg
    from weighted_bte_b200.workloads import minimal_authorized_parties

    t0 = time.perf_counter()
    committee, _ = minimal_authorized_parties(cfg.weights, cfg.threshold)
    sizes = cfg.sizes()
    classes = wpb.class_keys([wpb.size_class(s) for s in sizes], cfg.weights, cfg.threshold, committee, cfg.seed)
    keygen_s = time.perf_counter() - t0
    rng = ChaCha20Rng.seed_from_u64(cfg.seed)
    msgs, batches = [], []
    for s in sizes:
        m = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(s)])
        msgs.append(m)
        batches.append(wp.encrypt_many(classes[wpb.size_class(s)].material.encryption_key, m, rng))
    tuner = autotune.Autotuner()
    dec = wpb.UnevenBatchDecryptor(classes, streams=4, tuner=tuner)
    t1 = time.perf_counter()
    warm = dec.decrypt(batches, seed=1)  # tunes every class, fills the committee caches
    tune_s = time.perf_counter() - t1
    for b in range(len(sizes)):
        assert warm[b] == msgs[b], "batched weighted_pfe decryption mismatch"
    torch.cuda.synchronize()
    barrier()
    walls, gpu_ms = [], []
    for p in range(args.wpfe_passes):
        flush.add_(1)
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = dec.decrypt(batches, seed=2 + p)
        walls.append(time.perf_counter() - t)
        gpu_ms.append(sum(dec.class_ms.values()))
        for b in range(len(sizes)):
            assert out[b] == msgs[b], "batched weighted_pfe decryption mismatch"
    barrier()
    wall = max_over_ranks(statistics.median(walls))
    # per-kernel device time of one group of the largest class, alone on one stream
    from weighted_bte_b200 import _lib

    big = max(classes)
    idx = [b for b, s in enumerate(sizes) if wpb.size_class(s) == big]
    sc = classes[big]
    _lib.profile_enable(True)
    wpb.decrypt_group(sc.material.encryption_key, sc.material.decryption_key, [sc.pad(batches[b]) for b in idx],
                      sc.party_keys, ChaCha20Rng.seed_from_u64(7), dec.cache, device_output=True)
    torch.cuda.synchronize()
    prof = _lib.profile_read()
    _lib.profile_enable(False)
    class_kernels = {k: round(v[0], 2) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
    real = sum(sizes)
    slots = sum(wpb.size_class(s) for s in sizes)
    per_class = {}
    for B, sc in sorted(classes.items()):
        n_b = sum(1 for s in sizes if wpb.size_class(s) == B)
        knobs = tuner.lookup("wpfe", B, len(committee)) or {}
        per_class[str(B)] = {"batches": n_b, "ms": round(dec.class_ms.get(B, 0.0), 2),
                             "knobs": autotune.knob_values(knobs)}
    return {
        "value": world * real / wall, "unit": "ciphertexts/s",
        "slots_per_s": world * slots / wall, "ms_per_pass": 1000 * wall, "passes": args.wpfe_passes,
        "batches": len(sizes), "ciphertexts": real, "padded_slots": slots, "committee": committee,
        "workload": cfg.name, "timing": "wall clock of a pass over the 256 batches: host ciphertext lists in, "
        "host plaintext lists out, classes on 4 CUDA streams, committees cached",
        "class_ms_summed": round(statistics.median(gpu_ms), 2), "classes": per_class,
        "keygen_s": round(keygen_s, 1), "warm_and_tune_s": round(tune_s, 1),
        "largest_class_kernel_ms": {"class": big, "batches": len(idx), "kernels": class_kernels},
    }


# ------------------------------------------------------- served weighted_pfe
def wpfe_served_section(args, torch, wb, world, max_over_ranks, barrier, rank):
    """The served weighted_pfe form: requests with sizes log-uniform in
    [16, 4096] (seed 4) routed to resident power-of-two classes (n = 1000
    Pareto(1.2) weights scaled to W = 16384, t = W/3, the key material of
    every class in HBM), continuous batching of same-class requests,
    admission by HBM budget.  Reported: burst capacity, p50/p99 latency
    under Poisson arrivals at swept rates, and the plain per-request path
    (one request per launch sequence) on the same stream of requests."""
    from weighted_bte_b200 import serving
    from weighted_bte_b200 import weighted_pfe as wp
    from weighted_bte_b200 import wpfe_batched as wpb
    from weighted_bte_b200.rng import ChaCha20Rng
    from weighted_bte_b200.workloads import WPFE_SERVED as cfg
    from weighted_bte_b200.workloads import log_uniform_sizes, minimal_authorized_parties

    t0 = time.perf_counter()
    committee, _ = minimal_authorized_parties(cfg.weights, cfg.threshold)
    class_list = [1 << k for k in range((cfg.lo - 1).bit_length(), (cfg.hi - 1).bit_length() + 1)]
    classes = wpb.class_keys(class_list, cfg.weights, cfg.threshold, committee, cfg.seed)
    keygen_s = time.perf_counter() - t0
    resident = sum(sc.material.decryption_key.d1.numel() * 2 + sc.material.decryption_key.verification_keys.numel()
                   for sc in classes.values())
    rng = ChaCha20Rng.seed_from_u64(cfg.seed + 7919 * rank)
    sizes = log_uniform_sizes(args.served_requests, cfg.lo, cfg.hi, cfg.seed + rank)
    reqs, msgs = [], []
    for s in sizes:
        m = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(s)])
        msgs.append(m)
        reqs.append(wp.encrypt_many(classes[wpb.size_class(s)].material.encryption_key, m, rng))
    keys_of = {B: sc.party_keys for B, sc in classes.items()}
    backend = wpb.WpfeBackend(classes)
    out = {"workload": cfg.name, "committee_size": len(committee), "classes": class_list,
           "resident_key_bytes": int(resident), "keygen_s": round(keygen_s, 1), "requests_per_pass": len(sizes),
           "ciphertexts_per_pass": sum(sizes)}

    shared = serving.CommitteeCache(48 << 30)

    def burst(max_group):
        with serving.DecryptionServer(backend=backend, slots=3, max_group=max_group, cache=shared) as srv:
            # warm: every class's committee prepared before timing
            for B in class_list:
                s = next(x for x in sizes if wpb.size_class(x) == B) if any(wpb.size_class(x) == B for x in sizes) \
                    else None
                if s is not None:
                    i = sizes.index(s)
                    srv.submit(reqs[i], keys_of[B], seed=1).result()
            srv.latencies.clear()
            barrier()
            t = time.perf_counter()
            futs = [srv.submit(r, keys_of[wpb.size_class(len(r))], seed=k) for k, r in enumerate(reqs)]
            res = [f.result() for f in futs]
            dt = max_over_ranks(time.perf_counter() - t)
            st = srv.stats()
        for k, r in enumerate(res):
            assert r == msgs[k], "served weighted_pfe decryption mismatch"
        return dt, st

    dt, st = burst(16)
    cap_req = len(sizes) / dt
    out.update({"value": world * sum(sizes) / dt, "unit": "ciphertexts/s", "burst_p50_ms": st["p50_ms"],
                "burst_p99_ms": st["p99_ms"], "burst_requests_per_s": round(cap_req, 2)})
    dt1, st1 = burst(1)
    out.update({"plain_value": world * sum(sizes) / dt1, "plain_p50_ms": st1["p50_ms"], "plain_p99_ms": st1["p99_ms"],
                "served_over_plain": dt1 / dt,
                "plain_form": "the same requests through the same server with max_group = 1: one request per "
                              "launch sequence, committees cached"})
    # Poisson arrivals at fractions of the burst capacity
    arrivals = random.Random(4 + rank)
    for frac in (0.3, 0.6, 0.9):
        rate = frac * cap_req
        n = max(6, min(len(sizes), int(args.served_seconds * rate)))
        with serving.DecryptionServer(backend=backend, slots=3, max_group=16, cache=shared) as srv:
            for B in sorted({wpb.size_class(x) for x in sizes[:n]}):
                i = next(k for k, x in enumerate(sizes) if wpb.size_class(x) == B)
                srv.submit(reqs[i], keys_of[B], seed=1).result()
            srv.latencies.clear()
            t = time.perf_counter()
            t_next, futs = t, []
            for k in range(n):
                t_next += arrivals.expovariate(rate)
                delay = t_next - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futs.append(srv.submit(reqs[k], keys_of[wpb.size_class(len(reqs[k]))], seed=k))
            res = [f.result() for f in futs]
            el = time.perf_counter() - t
            st = srv.stats()
        for k, r in enumerate(res):
            assert r == msgs[k], "served weighted_pfe decryption mismatch"
        tag = f"at_{int(100 * frac)}pct"
        out[f"{tag}_offered_requests_per_s"] = round(rate, 2)
        out[f"{tag}_requests"] = n
        out[f"{tag}_ciphertexts_per_s"] = round(sum(sizes[:n]) / el)
        out[f"{tag}_p50_ms"] = st["p50_ms"]
        out[f"{tag}_p99_ms"] = st["p99_ms"]
    out["timing"] = ("wall clock, host ciphertext lists in and host plaintext lists out; latency per request from "
                     "submit to host result; Poisson arrivals at 30/60/90 % of the burst request rate")
    shared.clear()
    del classes, backend, shared
    torch.cuda.empty_cache()
    return out


# -------------------------------------------------------------- kernel sweep
def sweep_section(torch, wb, peak):
    """Config-3 kernel sweep (seed 2): each kernel on seeded inputs at the
    configuration's sizes, device time of one call after a warm-up call."""
    from weighted_bte_b200 import _lib, ops
    from weighted_bte_b200 import workcount as wc
    from weighted_bte_b200.rng import ChaCha20Rng, random_scalar

    rng = ChaCha20Rng.seed_from_u64(2)
    ctx = wb._ctx()
    out = {}
    dev = wb.empty_device

    def scal(n):
        return wb.to_device(ops.scalars_bytes([random_scalar(rng) for _ in range(n)]))

    # MSM: points = generator * u_i, uniform coefficients
    for g2 in (False, True):
        name = "g2_msm" if g2 else "g1_msm"
        size = 192 if g2 else 96
        big = 1 << 20
        pts = dev(size * big)
        ctx.call("wbte_g2_mul_generator" if g2 else "wbte_g1_mul_generator", pts, scal(big), big)
        sc = scal(big)
        res = dev(size)
        for lg in (10, 12, 14, 16, 18, 20):
            n = 1 << lg
            call = "wbte_g2_msm" if g2 else "wbte_g1_msm"
            ctx.call(call, res, pts, sc, n)
            ms, _ = event_ms(torch, lambda: ctx.call(call, res, pts, sc, n))
            prod = wc.msm_expected(n, 1, g2)
            out[f"{name}_2^{lg}"] = roof(call, ms, prod, peak, hbm_gbs=(size + 32) * n / (ms / 1000.0) / 1e9,
                                         work="expected Pippenger count of the plan")
        del pts, sc
    # group transforms of random elements, each path forced through the
    # context's knobs so that its exact count (workcount) applies; the entry
    # is the faster path, both are reported
    for lg in (8, 10, 12, 14, 16):
        n = 1 << lg
        for name, call, size, g2, knob, paths in (
                ("g1_ntt", "wbte_g1_ntt", 96, False, _lib.TUNE_NTT_JOINT, {"lanes": 0, "joint": 1}),
                ("g2_ntt", "wbte_g2_ntt", 192, True, _lib.TUNE_NTT_JOINT, {"lanes": 0, "joint": 1}),
                ("gt_ntt", "wbte_gt_ntt", 576, None, _lib.TUNE_GT_LANES, {"4_lanes": 4, "1_lane": 1})):
            buf = dev(size * n)
            if g2 is None:
                ctx.call("wbte_gt_pow", buf, wb.to_device(wb.gt_generator()), 1, scal(n), n)
            else:
                ctx.call("wbte_g2_mul_generator" if g2 else "wbte_g1_mul_generator", buf, scal(n), n)
            res = {}
            for pname, v in paths.items():
                ctx.set_tuning(knob, v)
                ctx.call(call, buf, n, 0)
                ms, _ = event_ms(torch, lambda: ctx.call(call, buf, n, 0))
                if g2 is None:
                    prod = wc.gt_ntt_single(n, v)
                else:
                    prod = wc.group_ntt_joint(n, g2) if v == 1 else wc.group_ntt_lanes(n, g2)
                res[pname] = roof(call, ms, prod, peak, path=pname, work="exact count of the forced path")
            ctx.set_tuning(_lib.TUNE_NTT_JOINT, -1)
            ctx.set_tuning(_lib.TUNE_GT_LANES, 0)
            best = min(res.values(), key=lambda r: r["ms"])
            entry = dict(best)
            entry["paths_ms"] = {k: r["ms"] for k, r in res.items()}
            out[f"{name}_2^{lg}"] = entry
            del buf
    # multi-pairing of k random pairs plus one final exponentiation
    for k in (1, 16, 256, 4096):
        p = dev(96 * k)
        q = dev(192 * k)
        ctx.call("wbte_g1_mul_generator", p, scal(k), k)
        ctx.call("wbte_g2_mul_generator", q, scal(k), k)
        f = dev(576)
        offs = [0, k]

        def pair():
            ctx.call("wbte_multi_miller_loop", f, p, q, _lib_i64(offs), 1)
            ctx.call("wbte_final_exp", f, f, 1, 0)

        pair()
        ms, _ = event_ms(torch, pair)
        prod = k * wc.MILLER_UNPREPARED + (k - 1) * wc.FP12_MUL + wc.FINAL_EXP
        out[f"multi_pairing_k{k}"] = roof("wbte_multi_miller_loop + wbte_final_exp", ms, prod, peak)
    return out


def _lib_i64(v):
    from weighted_bte_b200 import _lib

    return _lib.i64_array(v)


def main():
    args = parse_args()
    from weighted_bte_b200.workloads import WBTX_B512, minimal_authorized_parties

    cfg = WBTX_B512
    if args.impl == "reference":
        run_reference(args, cfg)
        return

    import numpy as np
    import torch

    from weighted_bte_b200 import replicas

    ranks = replicas.init("nccl")
    world, rank, local = ranks.world, ranks.rank, ranks.local_rank
    torch.cuda.set_device(local)
    from weighted_bte_b200 import _lib
    from weighted_bte_b200 import ops
    from weighted_bte_b200 import serving
    from weighted_bte_b200 import weighted_btx as wb
    from weighted_bte_b200 import workcount as wc
    from weighted_bte_b200.rng import ChaCha20Rng

    _lib.load()  # raises if the CUDA library is missing
    B, C, G = args.batch_size, args.concurrency, args.group
    weights, t = cfg.weights, cfg.threshold
    committee, _ = minimal_authorized_parties(weights, t)
    W_T = sum(weights[j] for j in committee)
    rng = ChaCha20Rng.seed_from_u64(ranks.seed(cfg.seed))

    t_setup = time.perf_counter()
    mat = wb.keygen_with_rng(wb.KeygenConfig(B, weights, t), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[j] for j in committee]
    host_p, dev_p, plain_p = make_batches(wb, mat, rng, B, args.warmup + args.steps)
    # distinct ciphertexts for two consecutive steps of the batched form; later
    # steps reuse them through fresh uploads (no encodings, digests or outputs
    # carry over, and L2 is flushed between steps)
    n_unique = 2 * C * G
    host_b, _, plain_b = make_batches(wb, mat, rng, B, n_unique)
    flush = torch.zeros(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup

    # loading key material from its wire format: a slice of the CRS as
    # compressed G2 points (96 B), decoded and checked on the device (canonical
    # x, square root on the curve, [r]P = O), host bytes in, HBM out
    n_crs = min(1 << 18, B * sum(weights))
    crs_blob = ops.g2_compress(dk.negative_material, n_crs)
    crs_out = torch.empty(192 * n_crs, dtype=torch.uint8, device="cuda")
    crs_load = {}
    for check in (True, False):
        _lib.default_context(local).call("wbte_g2_decompress", crs_out, None, crs_blob[: 96 * 1024], 1024, int(check))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.default_context(local).call("wbte_g2_decompress", crs_out, None, crs_blob, n_crs, int(check))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        crs_load["subgroup_checked_points_per_s" if check else "curve_checked_points_per_s"] = round(n_crs / dt)
    assert torch.equal(crs_out, dk.negative_material[: 192 * n_crs])
    del crs_out

    barrier, max_over_ranks = ranks.barrier, ranks.max
    stream = torch.cuda.current_stream()
    cache = serving.CommitteeCache(8 << 30)

    def step_plain(rb):
        return serving.decrypt_request(dk, rb, keys, ChaCha20Rng.seed_from_u64(99), None, device_output=True)

    def step_cached(rb):
        return serving.decrypt_request(dk, rb, keys, ChaCha20Rng.seed_from_u64(99), cache, device_output=True)

    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        gpu_id = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
    except (AttributeError, RuntimeError):
        gpu_id = str(local)
    sampler = ClockSampler(gpu_id)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    plain_value = cached_value = ms_plain = ms_cached = None
    launches_plain, prof = 0, {}
    if not args.no_plain:
        # ---- plain: one batch per step on one stream, committee prepared every batch
        for i in range(args.warmup):
            out = step_plain(dev_p[i])
        torch.cuda.synchronize()
        if args.warmup:  # correctness gate (untimed)
            assert wb.to_host(out, 576 * B) == b"".join(plain_p[args.warmup - 1])
        barrier()
        torch.cuda.synchronize()
        launches0 = _lib.load().wbte_ctx_launch_count(None)
        _lib.profile_enable(True)
        outs, ms_plain = timed_steps(torch, step_plain, dev_p[args.warmup:], flush, stream)
        barrier()
        prof = _lib.profile_read()
        _lib.profile_enable(False)
        launches_plain = _lib.load().wbte_ctx_launch_count(None) - launches0
        for i in range(args.steps):
            assert wb.to_host(outs[i], 576 * B) == b"".join(plain_p[args.warmup + i]), "decryption mismatch"
        ms_plain = max_over_ranks(ms_plain)
        plain_value = world * B * args.steps / (ms_plain / 1000.0)

        # ---- plain_cached: one batch per step, committee preparation cached
        for i in range(args.warmup):
            out = step_cached(dev_p[i])
        torch.cuda.synchronize()
        barrier()
        outs, ms_cached = timed_steps(torch, step_cached, dev_p[args.warmup:], flush, stream)
        barrier()
        for i in range(args.steps):
            assert wb.to_host(outs[i], 576 * B) == b"".join(plain_p[args.warmup + i]), "decryption mismatch"
        ms_cached = max_over_ranks(ms_cached)
        cached_value = world * B * args.steps / (ms_cached / 1000.0)

    # ---- batched: each step runs C groups concurrently (one CUDA stream each);
    # a group is G batches with every GPU phase launched once over all of them
    def step_group(idx):
        grp = [wb.CiphertextBatch.upload(host_b[i % n_unique]) for i in idx]
        return serving.decrypt_group(dk, grp, keys, ChaCha20Rng.seed_from_u64(99), cache, device_output=True)

    def groups(first_step, steps):
        return [list(range((first_step * C + g) * G, (first_step * C + g + 1) * G)) for g in range(steps * C)]

    run_batched(torch, step_group, groups(0, 1), C, 1, flush)  # warm-up (fills the committee cache)
    torch.cuda.synchronize()
    cache.clear()  # the timed region starts with an empty cache: its first group prepares
    launches0 = _lib.load().wbte_ctx_launch_count(None)
    barrier()
    timed_groups = groups(1, args.steps)
    outs_b, ms_b = run_batched(torch, step_group, timed_groups, C, args.steps, flush)
    barrier()
    launches_b = _lib.load().wbte_ctx_launch_count(None) - launches0
    clocks = sampler.stop()
    for idx, outs in zip(timed_groups, outs_b):
        for i, o in zip(idx, outs):
            assert wb.to_host(o, 576 * B) == b"".join(plain_b[i % n_unique]), "batched decryption mismatch"
    ms_b = max_over_ranks(ms_b)
    value = world * B * G * C * args.steps / (ms_b / 1000.0)

    # ---- the batched form with the decryption stage of every group replayed
    # as a captured CUDA graph (one capture per stream thread and shape)
    batched_graph = None
    try:
        if args.no_graph:
            raise RuntimeError("skipped (--no-graph)")
        graphs = serving.DecryptGraphs()

        def step_graph(idx):
            grp = [wb.CiphertextBatch.upload(host_b[i % n_unique]) for i in idx]
            return serving.decrypt_group(dk, grp, keys, ChaCha20Rng.seed_from_u64(99), cache, device_output=True,
                                         graphs=graphs)

        run_batched(torch, step_graph, groups(0, 1), C, 1, flush)  # warm-up: the captures
        torch.cuda.synchronize()
        replays0, launches0 = graphs.replays, _lib.load().wbte_ctx_launch_count(None)
        barrier()
        outs_g, ms_g = run_batched(torch, step_graph, timed_groups, C, args.steps, flush)
        barrier()
        direct = _lib.load().wbte_ctx_launch_count(None) - launches0
        replays = graphs.replays - replays0
        per = max(graphs.kernels.values()) if graphs.kernels else 0
        for idx, outs in zip(timed_groups, outs_g):
            for i, o in zip(idx, outs):
                assert wb.to_host(o, 576 * B) == b"".join(plain_b[i % n_unique]), "graph decryption mismatch"
        ms_g = max_over_ranks(ms_g)
        batched_graph = {"value": world * B * G * C * args.steps / (ms_g / 1000.0), "unit": "ciphertexts/s",
                         "ms_per_step": ms_g / args.steps, "graph_replays": replays, "kernels_per_replay": per,
                         "gpu_launches": int(direct + replays * per),
                         "form": "the batched form with each group's decryption stage (wbte_wbtx_decrypt_many) "
                                 "replayed as a captured CUDA graph"}
    except Exception as exc:  # reported beside the headline, never required
        batched_graph = {"value": None, "error": str(exc)[:200]}

    # ---- end to end: served requests with host ciphertexts and host results
    e2e = None
    if not args.no_e2e:
        with serving.DecryptionServer(dk, slots=C, max_group=G) as srv:
            for f in [srv.submit(host_b[i], keys, seed=99) for i in range(C * G)]:
                f.result()
            srv.latencies.clear()
            srv.cache.clear()  # as in the batched form, the timed region starts with an empty cache
            barrier()
            n_req = C * G * args.steps
            t0 = time.perf_counter()
            futs = [srv.submit(host_b[(C * G + i) % n_unique], keys, seed=99) for i in range(n_req)]
            res = [f.result() for f in futs]
            e2e_s = time.perf_counter() - t0
            st = srv.stats()
        barrier()
        e2e_s = max_over_ranks(e2e_s)
        for i, r in enumerate(res):
            assert r == plain_b[(C * G + i) % n_unique], "served decryption mismatch"
        h2d = B * (96 + 576 + 96 + 32)
        # request latency under load: Poisson arrivals at half the served rate
        # just measured, about 8 s of them, through a fresh server whose
        # committee is prepared before the first arrival
        req_rate = 0.5 * n_req / e2e_s
        n_load = max(2 * C, min(4 * n_req, int(8 * req_rate)))
        arrivals = random.Random(4 + rank)
        with serving.DecryptionServer(dk, slots=C, max_group=G) as srv:
            srv.submit(host_b[0], keys, seed=99).result()
            srv.latencies.clear()
            barrier()
            t0 = time.perf_counter()
            t_next, futs = t0, []
            for i in range(n_load):
                t_next += arrivals.expovariate(req_rate)
                delay = t_next - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futs.append(srv.submit(host_b[i % n_unique], keys, seed=99))
            res_l = [f.result() for f in futs]
            load_s = time.perf_counter() - t0
            st_l = srv.stats()
        for i, r in enumerate(res_l):
            assert r == plain_b[i % n_unique], "served decryption mismatch"
        e2e = {"value": world * B * n_req / e2e_s, "unit": "ciphertexts/s", "h2d_bytes_per_step": h2d * C * G,
               "d2h_bytes_per_step": B * 576 * C * G,
               "p50_ms": st_l["p50_ms"], "p99_ms": st_l["p99_ms"],
               "latency_basis": "p50/p99 request latency (submit to host result) under Poisson arrivals at half "
                                "the burst throughput",
               "offered_requests_per_s": round(req_rate, 1), "load_requests": n_load,
               "load_ciphertexts_per_s": round(B * n_load / load_s),
               "burst_p50_ms": st["p50_ms"], "burst_p99_ms": st["p99_ms"], "burst_requests": st["requests"],
               "slots": C, "max_group": G, "cache_hits": st["cache_hits"], "cache_misses": st["cache_misses"],
               "timing": "value: wall clock from the first submit to the last host result, all requests submitted "
                         "at once (burst)"}

    # ---- rooflines of the batched form's kernels, each on its own count of
    # Fp products, timed alone in one untimed profiled group (one stream)
    rate = np.zeros(1, dtype=np.float64)
    _lib.default_context(local).call("wbte_measure_imad_rate", rate)
    peak = float(rate[0]) / IMAD_PER_FP_MUL
    _lib.profile_enable(True)
    outs_p = step_group(groups(0, 1)[0])
    torch.cuda.synchronize()
    prof_g = _lib.profile_read()
    _lib.profile_enable(False)
    del outs_p
    m = wb.transform_size_for(B)
    T = len(committee)
    ms_of = {k: v[0] for k, v in prof_g.items()}
    top_g = max(prof_g.items(), key=lambda kv: kv[1][0])
    traffic = load_traffic()
    peak_basis = (f"measured {float(rate[0]) / 1e12:.2f} T IMAD/s (calibration kernel, mad.lo/mad.hi mix) / "
                  f"{IMAD_PER_FP_MUL} IMAD per Fp product")
    with open(os.path.join(ROOT, "weighted_bte_b200", "algorithmic_work.json")) as f:
        work = json.load(f)
    gt_own = wc.gt_prefix_ifft(m, B, G) if G % 32 == 0 and G >= 32 else None
    roofline = roof("gt_ifft (truncated cyclotomic inverse transform of a group: k_gt_radix4_pows_plan + "
                    "k_gt_radix4_outputs per radix-4 stage)", ms_of.get("gt_ifft"), gt_own or 0, peak,
                    peak_basis=peak_basis, batches_per_launch=G, dominant_in_group=top_g[0] == "gt_ifft",
                    work_basis="exact count of the Fp products the kernels run (warp-uniform NAF plans of the "
                               "twiddles, butterfly outputs); Fp additions not counted")
    tr = traffic.get("gt_ifft")
    if tr and ms_of.get("gt_ifft") and tr.get("group") == G and tr.get("batch_size") == B:
        # DRAM bytes of the phase's launches in one group, from the committed
        # one-metric ncu capture of this configuration; the stack traffic does
        # not grow in proportion to the group size, so no other size uses it
        roofline["traffic"] = tr["dram_bytes_per_group"]
        roofline["traffic_basis"] = tr["basis"]
    else:
        roofline["traffic"] = None
        roofline["traffic_basis"] = (f"no DRAM capture of this configuration (B = {B}, {G} batches per group) "
                                     "in profiles/roofline_traffic.json")
    if ms_of.get("gt_ifft") and m == work["cyclotomic_prefix_ifft"]["m"]:
        oracle_count = G * work["cyclotomic_prefix_ifft"]["fp_products"]
        roofline["oracle_count_frac"] = oracle_count / (ms_of["gt_ifft"] / 1000.0) / peak
        roofline["oracle_count_basis"] = ("the oracle's count of the reference algorithm (radix-2, plain tower "
                                          "arithmetic): a side figure, not the kernel's work")
    # run length of the share check's multi-Miller loops, from its profile tag
    miller_run = next((int(k[len("miller_c"):]) for k in ms_of if k.startswith("miller_c")), 1)
    rooflines = {
        "miller_lines": roof("k_miller_lines (precompute: prepared Miller loops of the transformed first "
                             "components)", ms_of.get("miller_lines"), wc.MILLER_WITH_LINES * m * G, peak),
        "miller_lines_multi": roof("k_miller_lines_multi (opening: one multi-Miller loop of T pairings per slot)",
                                   ms_of.get("miller_lines_multi"), wc.multi_miller_with_lines(T) * B * G, peak),
        "miller": roof(f"k_miller_chunks (share check: unprepared multi-Miller loops of B + 1 pairs per batch in "
                       f"runs of {miller_run} pairs per thread)", ms_of.get(f"miller_c{miller_run}"),
                       wc.multi_miller_unprepared(B + 1, miller_run) * G, peak),
        "final_exp_hard": roof("k_final_exp hard part (one per slot)", ms_of.get("final_exp_hard"),
                               wc.FINAL_EXP_HARD * B * G, peak),
        "ntt_g1": roof("k_ntt_stage_joint<Fp> (batched G1 transforms of the first components)",
                       ms_of.get("ntt_g1"), wc.g1_ntt_batched(m, G) if G % 32 == 0 else 0, peak),
        "msm_segments_g1": roof("k_segments<Fp> (partial decryptions: T x G G1 MSMs of B terms)",
                                ms_of.get("msm_segments_g1"), wc.msm_expected(B, T * G, False), peak,
                                work_basis="expected Pippenger count of the plan"),
    }
    group_kernels = {k: round(v[0], 2) for k, v in sorted(prof_g.items(), key=lambda kv: -kv[1][0])}

    # the plain path's dominant kernel: the preparation's G2 MSM segments
    top = max(prof.items(), key=lambda kv: kv[1][0]) if prof else ("none", (0.0, 0))
    msm_g2_ms = prof.get("msm_segments_g2", (0.0, 0))[0] / args.steps if prof else None
    msm_g2_work = sum(wc.msm_expected(weights[j], B, True) for j in committee) + wc.msm_expected(W_T, B - 1, True)
    roofline_plain = roof("k_segments<Fp2> (committee preparation: B x T party-block G2 MSMs and B - 1 kernel "
                          "G2 MSMs of W_T terms per batch)", msm_g2_ms, msm_g2_work, peak,
                          work_basis="expected Pippenger count of the plan", top_kernel_of_plain=top[0])

    # ---- batched weighted_pfe and the kernel sweep
    wpfe = None
    if not args.no_wpfe:
        wpfe = wpfe_section(args, torch, wb, flush, world, max_over_ranks, barrier)
        torch.cuda.empty_cache()
    served = None
    if not args.no_served:
        served = wpfe_served_section(args, torch, wb, world, max_over_ranks, barrier, rank)
    sweep = None
    if not args.no_sweep and rank == 0:
        sweep = sweep_section(torch, wb, peak)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            arm = CpuArm(cfg, B)
            times = arm.sample(1 + args.cpu_steps)[1:]
            cpu = {"value": B / statistics.median(times), "unit": "ciphertexts/s", "cores": arm.threads,
                   "kind": "port", "sample": arm.describe() + f"; median of {len(times)} timed batches after one "
                   f"warm-up", "seconds_per_batch": [round(x, 3) for x in times]}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "error": str(exc)[:200]}

    if rank == 0:
        phases = {k: round(v[0] / args.steps, 3) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
        line = {
            "metric": METRIC, "value": value, "unit": "ciphertexts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_b / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 limbs (Fp/Fr Montgomery)", "data": "synthetic",
            "config": {"workload": cfg.name, "batch_size": B, "parties": cfg.parties, "total_weight": cfg.total_weight,
                       "threshold": t, "committee": committee, "committee_weight": W_T,
                       "parallelism": f"replicas x{world}", "form": f"batched: {C} concurrent groups per step (one "
                       f"CUDA stream each), {G} batches per group with every GPU phase launched once per group; "
                       f"committee preparation cached (the timed region's first group prepares)",
                       "l2": "flushed before every step (256 MB write)"},
            "plain": {"value": plain_value, "unit": "ciphertexts/s",
                      "ms_per_batch": ms_plain / args.steps if ms_plain else None,
                      "form": "one batch per step on one stream, committee prepared every batch (reference decrypt())",
                      "gpu_launches": int(launches_plain)},
            "plain_cached": {"value": cached_value, "unit": "ciphertexts/s",
                             "ms_per_batch": ms_cached / args.steps if ms_cached else None,
                             "form": "one batch per step on one stream, committee preparation cached"},
            "batched_over_plain": value / plain_value if plain_value else None,
            "batched_over_plain_cached": value / cached_value if cached_value else None,
            "batched_graph": batched_graph,
            "e2e": e2e, "gpu_launches": int(launches_b), "roofline": roofline, "rooflines": rooflines,
            "roofline_plain": roofline_plain, "cpu_baseline": cpu, "clocks": clocks,
            "kernel_ms_per_batch_plain": phases, "kernel_ms_per_group": group_kernels,
            "wpfe_batched": wpfe, "wpfe_served": served, "sweep": sweep, "setup_s": round(setup_s, 2), "crs_load": crs_load,
        }
        print(json.dumps(line), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
