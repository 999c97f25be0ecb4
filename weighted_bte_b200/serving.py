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
overlap on the device.  Requests are admitted in arrival order.  A slot that
admits a request also takes the waiting requests of the same batch size and
committee (up to `max_group`, within the budget) and decrypts them as one
group: `decrypt_group`, where every GPU phase is one launch over all of
their batches (the batched form).

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
import struct
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _lib
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

    def obtain(self, key: bytes, build: Callable[[], tuple], count: bool = True):
        """The value cached under `key`, built by `build()` on the calling
        thread's current stream if absent.  build returns (value, tensors):
        the device tensors the value holds, which count against the budget.
        A thread that finds the value being built by another waits for it; the
        caller's stream is ordered after the build (a CUDA event)."""
        torch = wb._t()
        with self._lock:
            entry = self._entries.get(key)
            owner = entry is None
            if owner:
                entry = _Entry()
                self._entries[key] = entry
                if count:
                    self.misses += 1
            else:
                self._entries.move_to_end(key)
                if count:
                    self.hits += 1
        if owner:
            try:
                value, tensors = build()
                ev = torch.cuda.Event()
                ev.record(torch.cuda.current_stream())
                entry.pre, entry.ready = (value, list(tensors)), ev
                entry.nbytes = sum(t.numel() for t in tensors)
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
        value, tensors = entry.pre
        for t in tensors:
            t.record_stream(stream)
        return value

    def get(self, dk: wb.PublicDecryptionKey, accepted: wb.AcceptedDecryptionShares):
        """Prepared committee for `accepted`, prepared on the calling thread's
        current stream if absent.  The caller's stream is ordered after the
        preparation."""
        key = wb.decryption_context_id(dk.setup_id(), accepted.batch_size, accepted.party_indices())

        def build():
            pre = wb.prepare_decryption(dk, accepted)
            return pre, [pre.kernel_lines, pre.opening_keys, pre.opening_lines, pre.transformed_kernel]

        return self.obtain(key, build)

    def vk_tables(self, dk: wb.PublicDecryptionKey, batch_size: int, party_indices: Sequence[int]):
        """Fixed-base tables of the parties' verification keys at slots
        1..batch_size (wbte_wbtx_vk_tables), built once per party set and
        batch size on the calling thread's current stream; the share check of
        every later group of the same parties uses them."""
        key = b"vk-tables" + dk.setup_id() + struct.pack("<Q", batch_size) + b"".join(
            struct.pack("<q", j) for j in party_indices)

        def build():
            T = len(party_indices)
            tables = wb.empty_device(_lib.FIXED_TABLE_BYTES * T * batch_size)
            wb._ctx().call("wbte_wbtx_vk_tables", tables, dk.abi_key(), _lib.i64_array(party_indices), T, batch_size)
            return tables, [tables]

        return self.obtain(key, build, count=False)

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


class DecryptGraphs:
    """The batched decryption (wbte_wbtx_decrypt_many) replayed as captured
    CUDA graphs.  For each prepared committee, batch size and group size, a
    thread captures the call once into static device buffers; later groups of
    the same shape copy their inputs in and replay the graph, which launches
    the whole kernel sequence (transforms, Miller loops, final
    exponentiations, products) as one unit.  The call has no host-synchronous
    step when every buffer is on the device, so it captures as is; a warm-up
    call first fills the library's caches (twiddles, occupancy queries)."""

    def __init__(self):
        self._local = threading.local()
        self._lock = threading.Lock()
        self.captures = 0
        self.replays = 0
        self.kernels = {}  # shape -> kernels launched per replay

    def run(self, pre: wb.DecryptionPrecomputation, first, second, valid, sigma_dev, T: int, B: int, K: int):
        torch = wb._t()
        table = getattr(self._local, "table", None)
        if table is None:
            table = self._local.table = {}
        key = (pre.context_id, B, K, T)
        ent = table.get(key)
        if ent is None:
            ent = table[key] = self._capture(pre, T, B, K)
        ent["first"].copy_(first)
        ent["second"].copy_(second)
        ent["valid"].copy_(valid)
        ent["sigma"].copy_(sigma_dev)
        ent["graph"].replay()
        with self._lock:
            self.replays += 1
        return ent["out"].clone()

    def _capture(self, pre, T, B, K):
        torch = wb._t()
        st = {"first": wb.empty_device(G1B * B * K), "second": wb.empty_device(GTB * B * K),
              "valid": wb.empty_device(B * K), "sigma": wb.empty_device(G1B * T * K),
              "out": wb.empty_device(GTB * B * K)}
        for t in st.values():
            t.zero_()

        def call():
            wb._ctx().call("wbte_wbtx_decrypt_many", st["out"], pre.kernel_lines, pre.opening_keys,
                           pre.opening_lines, st["first"], st["second"], st["valid"], st["sigma"], T, B, K)

        call()  # warm-up outside the capture
        torch.cuda.current_stream().synchronize()
        lib = _lib.load()
        n0 = lib.wbte_thread_launch_count()
        g = torch.cuda.CUDAGraph()
        # Thread-local capture on a side stream: other threads keep launching,
        # copying and allocating on their own streams meanwhile.  (The
        # torch.cuda.graph context synchronizes the device and empties the
        # allocator cache first, which breaks another thread's capture.)
        cur = torch.cuda.current_stream()
        side = torch.cuda.Stream()
        side.wait_stream(cur)
        with torch.cuda.stream(side):
            g.capture_begin(capture_error_mode="thread_local")
            try:
                call()
            finally:
                g.capture_end()
        cur.wait_stream(side)
        with self._lock:
            self.kernels[(B, K, T)] = int(lib.wbte_thread_launch_count() - n0)
            self.captures += 1
        st["graph"] = g
        return st


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


def decrypt_group(dk: wb.PublicDecryptionKey, batches: Sequence, party_keys: Sequence[wb.PartySecretKey], rng,
                  cache: Optional[CommitteeCache] = None, device_output: bool = False,
                  graphs: Optional[DecryptGraphs] = None) -> List:
    """The batched form: K batches of one size, decrypted by one committee,
    with every GPU phase launched once for all K (the wbte_wbtx_*_many calls).
    Per batch the result is exactly `decrypt_request`'s: validation,
    transcripts, digests and the share-acceptance rules run per batch; a batch
    whose aggregate share check fails falls back to the per-share path alone.
    With `graphs`, the final decryption of each part is a replayed CUDA graph."""
    torch = wb._t()
    K = len(batches)
    if K == 0:
        return []
    B = len(batches[0])
    if any(len(b) != B for b in batches):
        raise ValueError("a group holds batches of one size")
    T = len(party_keys)
    validated = wb.validate_batches(dk, batches)
    for pk in party_keys:
        if pk.setup_id() != dk.setup_id():
            from . import errors as E

            raise E.MismatchedSetup()
    first = torch.cat([v.first_dev[: G1B * B] for v in validated])
    valid = torch.cat([v.valid_dev[:B] for v in validated])
    ctx = wb._ctx()
    sig = bytearray(G1B * T * K)
    ctx.call("wbte_wbtx_partial_decrypt_many", sig, first, B, b"".join(wb.fr_bytes(pk.secret_scalar()) for pk in party_keys),
             T, K)
    shares = [[wb.DecryptionShare(pk.party_index, bytes(sig[G1B * (b * T + j) : G1B * (b * T + j + 1)]),
                                  validated[b].digest(), pk.setup_id()) for j, pk in enumerate(party_keys)]
              for b in range(K)]
    screened = [wb.screen_shares(dk, validated[b], shares[b]) for b in range(K)]
    full = all(len(c) == T and not r for c, r in screened)
    if full and T > 0:
        from .rng import sample_nonzero

        challenges = [[sample_nonzero(rng) for _ in range(T)] for _ in range(K)]
        ok = np.zeros(K, dtype=np.int32)
        parties = [pk.party_index for pk in party_keys]
        tables = cache.vk_tables(dk, B, parties) if cache is not None else None
        ctx.call("wbte_wbtx_verify_shares_many", ok, dk.abi_key(), first, B, bytes(sig), _lib.i64_array(parties),
                 b"".join(wb.fr_bytes(c) for row in challenges for c in row), T, K, tables)
        accepted = [wb.finish_acceptance(dk, validated[b], *screened[b], bool(ok[b])) for b in range(K)]
    else:
        accepted = [wb.accept_decryption_shares(dk, validated[b], shares[b], rng) for b in range(K)]
    # a batch whose share check blamed a party keeps its own (smaller)
    # accepted committee: the batches are split by accepted committee and each
    # part is decrypted as one group, so one bad share costs one extra group,
    # not K single-batch decryptions
    parts: "collections.OrderedDict[tuple, List[int]]" = collections.OrderedDict()
    for b, a in enumerate(accepted):
        parts.setdefault(tuple(a.party_indices()), []).append(b)
    second_all = torch.cat([c.second[: GTB * B] if isinstance(c, wb.CiphertextBatch)
                            else wb.to_device(b"".join(x.second for x in c)) for c in batches])
    results: List = [None] * K
    for idx in parts.values():
        acc = [accepted[b] for b in idx]
        pre = cache.get(dk, acc[0]) if cache is not None else wb.prepare_decryption(dk, acc[0])
        Ta, Kp = acc[0].party_count(), len(idx)
        sigmas = b"".join(s.sigma for a in acc for s in a.shares())
        if Kp == K:
            f_p, v_p, s_p = first, valid, second_all
        else:
            f_p = torch.cat([first[G1B * B * b : G1B * B * (b + 1)] for b in idx])
            v_p = torch.cat([valid[B * b : B * (b + 1)] for b in idx])
            s_p = torch.cat([second_all[GTB * B * b : GTB * B * (b + 1)] for b in idx])
        # precompute_batch and open_batch of the part's batches, the cross terms
        # and the opening pairings sharing one hard final exponentiation per slot
        if graphs is not None:
            out = graphs.run(pre, f_p, s_p, v_p, wb.to_device(sigmas), Ta, B, Kp)
        else:
            out = wb.empty_device(GTB * B * Kp)
            ctx.call("wbte_wbtx_decrypt_many", out, pre.kernel_lines, pre.opening_keys, pre.opening_lines, f_p, s_p,
                     v_p, sigmas, Ta, B, Kp)
        if device_output:
            for q, b in enumerate(idx):
                results[b] = out[GTB * B * q : GTB * B * (q + 1)]
        else:
            host = wb.to_host(out, GTB * B * Kp)
            for q, b in enumerate(idx):
                results[b] = [host[GTB * (q * B + i) : GTB * (q * B + i + 1)] if validated[b].valid[i] else None
                              for i in range(B)]
    return results


class WbtxBackend:
    """How the server runs weighted_btx requests: memory estimate, grouping
    key, and the decryption of a group (one request alone, or several of
    one batch size and committee as one batched group)."""

    def __init__(self, decryption_key: wb.PublicDecryptionKey):
        self.dk = decryption_key

    def need(self, ciphertexts, party_keys) -> int:
        B, T = len(ciphertexts), len(party_keys)
        # whether the committee will be cached is known only when the request
        # runs, so admission always reserves room for preparing it
        wt = sum(self.dk.party_weight(k.party_index) for k in party_keys)
        return request_bytes(B, T) + preparation_bytes(B, T, wt)

    def group_key(self, ciphertexts, party_keys):
        return len(ciphertexts), tuple(k.party_index for k in party_keys)

    def run(self, group, rng, cache) -> list:
        if len(group) == 1:
            return [decrypt_request(self.dk, group[0].ciphertexts, group[0].party_keys, rng, cache)]
        return decrypt_group(self.dk, [r.ciphertexts for r in group], group[0].party_keys, rng, cache)


@dataclass
class _Request:
    ciphertexts: object
    party_keys: Sequence[wb.PartySecretKey]
    seed: int
    need: int
    future: cf.Future
    submitted: float
    key: object = None
    started: float = 0.0


class DecryptionServer:
    """Request loop with continuous batching over `slots` CUDA streams.

    submit() returns a Future of the request's result (for weighted_btx one
    Optional[bytes] per slot, None where the ciphertext's proof failed; a
    request the scheme rejects as a whole raises its error through the
    future).  Latency is measured from submit() to the result being
    available on the host.  `backend` selects the scheme (default: weighted_btx
    under `decryption_key`; wpfe_batched.WpfeBackend serves weighted_pfe);
    `cache` shares a committee cache between servers of the same keys."""

    def __init__(self, decryption_key: Optional[wb.PublicDecryptionKey] = None, slots: int = 4,
                 hbm_budget_bytes: Optional[int] = None, cache_bytes: Optional[int] = None,
                 device: Optional[int] = None, cache_committees: bool = True, max_group: int = 1, backend=None,
                 cache: Optional[CommitteeCache] = None):
        torch = wb._t()
        self.backend = backend if backend is not None else WbtxBackend(decryption_key)
        self.dk = decryption_key
        self.device = torch.cuda.current_device() if device is None else device
        # requests of one batch size and committee that wait together are
        # decrypted as one group (the batched form), up to max_group at a time
        self.max_group = max(1, int(max_group))
        if hbm_budget_bytes is None:
            free, _total = torch.cuda.mem_get_info(self.device)
            hbm_budget_bytes = free // 2
        self.budget = int(hbm_budget_bytes)
        if cache is not None:
            self.cache = cache  # shared with other servers of the same keys
        else:
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
    def submit(self, ciphertexts, party_keys: Sequence, seed: int = 0) -> cf.Future:
        need = self.backend.need(ciphertexts, party_keys)
        if need > self.budget:
            raise MemoryError(f"request of {len(ciphertexts)} ciphertexts needs ~{need} bytes, budget {self.budget}")
        fut: cf.Future = cf.Future()
        req = _Request(ciphertexts, list(party_keys), seed, need, fut, time.perf_counter(),
                       self.backend.group_key(ciphertexts, party_keys))
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
    @staticmethod
    def _group_key(req: _Request):
        return req.key

    def _admit(self) -> Optional[List[_Request]]:
        """Admit the head request once it fits the budget, then every waiting
        request of the same batch size and committee that still fits, up to
        max_group (requests keep their arrival order)."""
        with self._cv:
            while True:
                if self._queue:
                    head = self._queue[0]
                    if self._in_use + head.need <= self.budget:
                        group = [self._queue.popleft()]
                        key = self._group_key(head)
                        taken = head.need
                        rest = collections.deque()
                        while self._queue and len(group) < self.max_group:
                            r = self._queue.popleft()
                            if self._group_key(r) == key and self._in_use + taken + r.need <= self.budget:
                                group.append(r)
                                taken += r.need
                            else:
                                rest.append(r)
                        rest.extend(self._queue)
                        self._queue = rest
                        self._in_use += taken
                        self._in_flight += len(group)
                        self.peak_in_flight = max(self.peak_in_flight, self._in_flight)
                        self.peak_bytes = max(self.peak_bytes, self._in_use)
                        return group
                elif self._closed:
                    return None
                self._cv.wait()

    def _release(self, group: List[_Request]):
        with self._cv:
            for req in group:
                self._in_use -= req.need
            self._in_flight -= len(group)
            self._cv.notify_all()

    def _work(self, slot: int):
        torch = wb._t()
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(device=self.device)
        while True:
            group = self._admit()
            if group is None:
                return
            now = time.perf_counter()
            for req in group:
                req.started = now
            try:
                rng = ChaCha20Rng.seed_from_u64(group[0].seed)
                with torch.cuda.stream(stream):
                    outs = self.backend.run(group, rng, self.cache)
                stream.synchronize()
                done = time.perf_counter()
                with self._cv:
                    for req in group:
                        self.latencies.append(done - req.submitted)
                        self.completed_ciphertexts += len(req.ciphertexts)
                for req, out in zip(group, outs):
                    if isinstance(out, BaseException):
                        req.future.set_exception(out)
                    else:
                        req.future.set_result(out)
            except BaseException as exc:  # noqa: BLE001 -- reported through the futures
                for req in group:
                    if not req.future.done():
                        req.future.set_exception(exc)
            finally:
                self._release(group)


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
