"""Batched and served weighted_btx decryption on one GPU.

`DecryptionServer` runs batch-decrypt requests of any size as they arrive.
Each request is one full decryption of an ordered ciphertext batch by a
committee -- validate, partial decryption by the committee members,
aggregate share acceptance, committee preparation, cross-term
precomputation and opening, the sequence of the reference's `decrypt`
(weighted_btx/src/decryption.rs:698-709) with the partial decryptions of
weighted_btx/src/decryption.rs:205-233 in front.

Continuous batching: `slots` worker threads each own a CUDA stream (CUDA maps
streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware queues, 8 unless the
environment sets more before the CUDA context exists; set it to at least
`slots`).  A
request is admitted as soon as a slot is free and its device-memory
estimate fits in what the HBM budget has left; admitted requests run
concurrently on their slots' streams, so the kernels of several batches
overlap on the device.  Requests are admitted in arrival order.

Committee cache: the reference documents the committee preparation as
independent of the ciphertexts and reusable for another batch of the same
size and accepted party set (weighted_btx/src/decryption.rs:424-426).  The
server keeps prepared committees in HBM, keyed by the reference's
decryption context id (setup id, batch size, accepted parties), evicting the
least recently used entry beyond `cache_bytes`.  A request whose committee
is being prepared by another slot waits for that preparation (a CUDA event
orders the streams) instead of repeating it.

Every request computes exactly what `weighted_btx.decrypt` computes for it
alone; the tests check that each result is byte-identical alone and in the
mix.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

from . import weighted_btx as wb
from .rng import ChaCha20Rng

GTB, G1B, G2B = wb.GTB, wb.G1B, wb.G2B


def request_bytes(batch_size: int, parties: int) -> int:
    """Device memory one request holds while it runs, without its committee
    preparation: the resident batch (first/second/commitment/response), the
    cross-term transform (G1 XYZZ work + GT values over the transform size),
    the per-slot pairing products of the opening and the outputs."""
    B, T = batch_size, parties
    m = wb.transform_size_for(B)
    batch = B * (G1B + GTB + G1B + 32 + 1)
    precompute = m * (G1B + 2 * G1B + GTB) + B * GTB
    opening = B * T * GTB + 2 * B * GTB
    return batch + precompute + opening + (1 << 20)


def preparation_bytes(batch_size: int, parties: int, committee_weight: int) -> int:
    """Device memory of one prepared committee (kept in the cache) plus the
    peak working memory of preparing it (MSM scratch, transform work)."""
    B, T, WT = batch_size, parties, committee_weight
    m = wb.transform_size_for(B)
    resident = m * 68 * 288 + B * T * G2B + m * G2B
    windows = 32
    segments = 16
    scratch = 2 * windows * WT * (2 + 8) + B * windows * segments * 2 * G2B + m * 2 * G2B + 2 * B * T * G2B
    return resident + scratch


@dataclass
class _Entry:
    pre: Optional[wb.DecryptionPrecomputation] = None
    ready: object = None  # torch.cuda.Event recorded after the preparation
    error: Optional[BaseException] = None
    done: threading.Event = field(default_factory=threading.Event)
    nbytes: int = 0


class CommitteeCache:
    """Prepared committees resident in HBM (LRU, bounded by bytes)."""

    def __init__(self, max_bytes: int):
        self.max_bytes = max_bytes
        self._lock = threading.Lock()
        self._entries: "collections.OrderedDict[bytes, _Entry]" = collections.OrderedDict()
        self._bytes = 0
        self.hits = 0
        self.misses = 0

    def get(self, dk: wb.PublicDecryptionKey, accepted: wb.AcceptedDecryptionShares):
        """Prepared committee for `accepted`, prepared on the calling thread's
        current stream if absent.  The caller's stream is ordered after the
        preparation."""
        torch = wb._t()
        key = wb.decryption_context_id(dk.setup_id(), accepted.batch_size, accepted.party_indices())
        with self._lock:
            entry = self._entries.get(key)
            owner = entry is None
            if owner:
                entry = _Entry()
                self._entries[key] = entry
                self.misses += 1
            else:
                self._entries.move_to_end(key)
                self.hits += 1
        if owner:
            try:
                entry.pre = wb.prepare_decryption(dk, accepted)
                ev = torch.cuda.Event()
                ev.record(torch.cuda.current_stream())
                entry.ready = ev
                entry.nbytes = sum(t.numel() for t in (entry.pre.kernel_lines, entry.pre.opening_keys,
                                                        entry.pre.transformed_kernel))
            except BaseException as exc:  # noqa: BLE001 -- handed to every waiter
                entry.error = exc
                with self._lock:
                    self._entries.pop(key, None)
            finally:
                entry.done.set()
            if entry.error is None:
                self._evict()
        else:
            entry.done.wait()
        if entry.error is not None:
            raise entry.error
        stream = torch.cuda.current_stream()
        stream.wait_event(entry.ready)
        for t in (entry.pre.kernel_lines, entry.pre.opening_keys, entry.pre.transformed_kernel):
            t.record_stream(stream)
        return entry.pre

    def _evict(self):
        with self._lock:
            self._bytes = sum(e.nbytes for e in self._entries.values())
            while self._bytes > self.max_bytes and len(self._entries) > 1:
                _, old = self._entries.popitem(last=False)
                self._bytes -= old.nbytes

    def clear(self):
        with self._lock:
            self._entries.clear()
            self._bytes = 0
            self.hits = self.misses = 0

    def __len__(self):
        return len(self._entries)


def decrypt_request(dk: wb.PublicDecryptionKey, ciphertexts, party_keys: Sequence[wb.PartySecretKey], rng,
                    cache: Optional[CommitteeCache] = None, device_output: bool = False):
    """One batch decryption: validate, committee partial decryptions, share
    acceptance, (cached) committee preparation, precomputation, opening."""
    batch = wb.validate_batch(dk, ciphertexts)
    shares = wb.partial_decrypt_many(party_keys, batch)
    accepted = wb.accept_decryption_shares(dk, batch, shares, rng)
    pre = cache.get(dk, accepted) if cache is not None else wb.prepare_decryption(dk, accepted)
    cross = wb.precompute_batch(pre, batch)
    return wb.open_batch(pre, accepted, batch, ciphertexts, cross, device_output=device_output)


@dataclass
class _Request:
    ciphertexts: object
    party_keys: Sequence[wb.PartySecretKey]
    seed: int
    need: int
    future: cf.Future
    submitted: float
    started: float = 0.0


class DecryptionServer:
    """Request loop with continuous batching over `slots` CUDA streams.

    submit() returns a Future of the request's result (one Optional[bytes]
    per slot, None where the ciphertext's proof failed).  Latency is measured
    from submit() to the result being available on the host."""

    def __init__(self, decryption_key: wb.PublicDecryptionKey, slots: int = 4,
                 hbm_budget_bytes: Optional[int] = None, cache_bytes: Optional[int] = None,
                 device: int = 0, cache_committees: bool = True):
        torch = wb._t()
        self.dk = decryption_key
        self.device = device
        if hbm_budget_bytes is None:
            free, _total = torch.cuda.mem_get_info(device)
            hbm_budget_bytes = free // 2
        self.budget = int(hbm_budget_bytes)
        self.cache = CommitteeCache(cache_bytes if cache_bytes is not None else self.budget // 4) \
            if cache_committees else None
        self._cv = threading.Condition()
        self._queue: "collections.deque[_Request]" = collections.deque()
        self._in_use = 0
        self._closed = False
        self.latencies: List[float] = []
        self.completed_ciphertexts = 0
        self.peak_in_flight = 0
        self.peak_bytes = 0
        self._in_flight = 0
        self._workers = [threading.Thread(target=self._work, args=(i,), daemon=True) for i in range(slots)]
        for w in self._workers:
            w.start()

    # ---------------------------------------------------------------- API
    def submit(self, ciphertexts, party_keys: Sequence[wb.PartySecretKey], seed: int = 0) -> cf.Future:
        B = len(ciphertexts)
        T = len(party_keys)
        need = request_bytes(B, T)
        # whether the committee will be cached is known only when the request
        # runs, so admission always reserves room for preparing it
        wt = sum(self.dk.party_weight(k.party_index) for k in party_keys)
        need_prep = preparation_bytes(B, T, wt)
        if need + need_prep > self.budget:
            raise MemoryError(f"request of {B} ciphertexts needs ~{need + need_prep} bytes, budget {self.budget}")
        fut: cf.Future = cf.Future()
        req = _Request(ciphertexts, list(party_keys), seed, need + need_prep, fut, time.perf_counter())
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._queue.append(req)
            self._cv.notify_all()
        return fut

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for w in self._workers:
            w.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def stats(self) -> dict:
        lat = sorted(self.latencies)

        def pct(p):
            if not lat:
                return None
            k = min(len(lat) - 1, max(0, int(round(p / 100.0 * (len(lat) - 1)))))
            return 1000.0 * lat[k]

        return {"requests": len(lat), "p50_ms": pct(50), "p99_ms": pct(99),
                "cache_hits": self.cache.hits if self.cache else 0,
                "cache_misses": self.cache.misses if self.cache else 0,
                "peak_in_flight": self.peak_in_flight, "peak_bytes": self.peak_bytes}

    # ------------------------------------------------------------ workers
    def _admit(self) -> Optional[_Request]:
        with self._cv:
            while True:
                if self._queue:
                    head = self._queue[0]
                    if self._in_use + head.need <= self.budget:
                        self._queue.popleft()
                        self._in_use += head.need
                        self.peak_bytes = max(self.peak_bytes, self._in_use)
                        self._in_flight += 1
                        self.peak_in_flight = max(self.peak_in_flight, self._in_flight)
                        return head
                elif self._closed:
                    return None
                self._cv.wait()

    def _release(self, req: _Request):
        with self._cv:
            self._in_use -= req.need
            self._in_flight -= 1
            self._cv.notify_all()

    def _work(self, slot: int):
        torch = wb._t()
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(device=self.device)
        while True:
            req = self._admit()
            if req is None:
                return
            req.started = time.perf_counter()
            try:
                with torch.cuda.stream(stream):
                    out = decrypt_request(self.dk, req.ciphertexts, req.party_keys,
                                          ChaCha20Rng.seed_from_u64(req.seed), self.cache)
                stream.synchronize()
                done = time.perf_counter()
                with self._cv:
                    self.latencies.append(done - req.submitted)
                    self.completed_ciphertexts += len(req.ciphertexts)
                req.future.set_result(out)
            except BaseException as exc:  # noqa: BLE001 -- reported through the future
                req.future.set_exception(exc)
            finally:
                self._release(req)


def run_concurrent(fn: Callable, items: Sequence, slots: int):
    """Runs fn(item) for every item on `slots` CUDA streams (one host thread
    each, items dealt round-robin).  Returns (outputs, device milliseconds
    from a start event that every stream waits on to the last stream's end
    event)."""
    torch = wb._t()
    streams = [torch.cuda.Stream() for _ in range(slots)]
    start = torch.cuda.Event(enable_timing=True)
    start.record(torch.cuda.current_stream())
    ends = [None] * slots
    outs = [None] * len(items)
    errors: List[BaseException] = []
    device = torch.cuda.current_device()

    def worker(w):
        try:
            torch.cuda.set_device(device)
            s = streams[w]
            s.wait_event(start)
            with torch.cuda.stream(s):
                for i in range(w, len(items), slots):
                    outs[i] = fn(items[i])
                e = torch.cuda.Event(enable_timing=True)
                e.record(s)
                ends[w] = e
        except BaseException as exc:  # noqa: BLE001
            errors.append(exc)

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(slots)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    torch.cuda.synchronize()
    ms = max(start.elapsed_time(e) for e in ends if e is not None)
    return outs, ms
