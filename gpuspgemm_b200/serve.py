"""Served form: a continuous-batching request loop over device-resident operands.

Requests ``C = A * B`` (operands already on the device) arrive at any time.
Worker threads, each owning a library handle (its own side streams, scratch and
stream), repeatedly

1. size new arrivals on the device: NIP (intermediate products) of all of
   them with one launch and one host synchronisation (spgemm_get_nip_many); the
   binning phase's upper bound on the output,
   ``bytes(C) <= 4 (m + 1) + NIP * (4 + sizeof(value))``, is the request's
   share of the memory budget;
2. admit, oldest first: a request with ``NIP >= solo_nip`` runs alone on the
   plain path (its rows already fill every bin); smaller ones are taken in
   arrival order (passing over large ones, which the next free worker takes)
   while the budget, ``max_batch`` and the per-batch NIP cap ``batch_nip`` --
   which bounds a batch's duration, so a small request never waits long for
   the rest of its batch -- allow;
3. pack the small requests into block-diagonal operands and run them as ONE
   batched product (``spgemm_batch_*``), so rows of different requests share
   bins and kernels;
4. hand each request its own CSR result and release its share of the budget.

Workers wait on one condition variable that every arrival, every finished
sizing and every finished unit signals, and a free worker always takes the
next unit at once: with several workers a large product, medium products and
batches of small ones run side by side on the GPU, each on its worker's
stream.  The reference has no served or batched form; it multiplies one pair
per call (proposal.cuh:85-124).

The workers are Python threads: anything that holds the interpreter lock
stalls all of them.  A process serving requests should move its long-lived
objects out of the cyclic garbage collector's reach (``gc.freeze()`` after
start-up): a full collection over a pool of operands paused every worker for
~55 ms on a B200 host.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .api import DeviceCSR, Handle, PackedBatch, batch, get_nip_many, pack_batch, proposal


@dataclass
class Request:
    A: DeviceCSR
    B: DeviceCSR
    rid: int = 0
    t_arrival: float = 0.0
    t_admitted: float = 0.0
    t_done: float = 0.0
    bound_bytes: int = 0
    nip: int = 0
    sizing: bool = False
    result: DeviceCSR | None = None
    error: BaseException | None = None
    done: threading.Event = field(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


class SpgemmServer:
    """Continuous-batching SpGEMM server on one GPU.

    memory_budget: bytes of C bounds that may be in flight at once.
    max_batch:     most requests packed into one batched product.
    workers:       worker threads (handles), each with its own stream: units
                   of work run side by side on the GPU.
    solo_nip:      requests with at least this many intermediate products run
                   alone on the plain path.
    batch_nip:     most intermediate products of one batch.  The cap a batch
                   actually gets follows the backlog: the queued requests' NIP
                   shared over the workers, at least batch_nip_min.  A short
                   queue (light load) makes short batches, so a small request
                   does not wait long for the rest of its batch; a long one
                   (saturation) makes long batches, which amortise each
                   product's fixed cost over many requests.
    batch_cols:    most columns of a packed batch's B (the sum of its
                   members' B.n).
    size_chunk:    most arrivals a worker sizes in one call before it tries to
                   admit.
    """

    def __init__(self, memory_budget: int = 32 << 30, max_batch: int = 256, workers: int = 4,
                 device: int = 0, solo_nip: int = 4 << 20, batch_nip: int = 32 << 20,
                 batch_nip_min: int = 4 << 20, batch_cols: int = 1 << 20,
                 size_chunk: int = 256):
        import torch
        self._torch = torch
        self.device = device
        self.memory_budget = int(memory_budget)
        self.max_batch = int(max_batch)
        self.solo_nip = int(solo_nip)
        self.batch_nip = int(batch_nip)
        self.batch_nip_min = int(batch_nip_min)
        self.batch_cols = int(batch_cols)
        self.workers = int(workers)
        self.size_chunk = int(size_chunk)
        self._queue: deque[Request] = deque()
        self._cv = threading.Condition()
        self._in_flight_bytes = 0
        self._stop = False
        self._handles = [Handle(device) for _ in range(workers)]
        self._next_id = 0
        self.batches = 0
        self.batched_requests = 0
        # per batch: (worker, requests, t_admitted, t_launched, t_done), perf_counter s
        self.timeline: list[tuple[int, int, float, float, float]] = []
        self._threads = [threading.Thread(target=self._worker, args=(i, h), daemon=True)
                         for i, h in enumerate(self._handles)]
        for t in self._threads:
            t.start()

    # -- client side --------------------------------------------------------
    def submit(self, A: DeviceCSR, B: DeviceCSR, t_arrival: float | None = None) -> Request:
        """Queue C = A * B and return the Request; wait on req.done.  The
        request's admission bound is computed by a worker, on the device."""
        if A.n != B.m:
            raise ValueError("A.n must equal B.m")
        req = Request(A, B, t_arrival=time.perf_counter() if t_arrival is None else t_arrival,
                      bound_bytes=-1)
        with self._cv:
            req.rid = self._next_id
            self._next_id += 1
            self._queue.append(req)
            self._cv.notify_all()
        return req

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        for h in self._handles:
            h.close()

    # -- worker side --------------------------------------------------------
    def _admit(self) -> tuple[list[Request], bool]:
        """Take the next unit of work (call with the lock held): a large
        request alone (second value True), or small requests in arrival order
        under the budget, max_batch, the backlog-scaled NIP cap and
        batch_cols.  Unsized requests stop the
        scan, so admission order is arrival order.  A request larger than the
        whole budget runs when nothing else is in flight."""
        taken: list[Request] = []
        nip = 0
        cols = 0
        skipped = []
        backlog = sum(r.nip for r in self._queue if r.bound_bytes >= 0 and r.nip < self.solo_nip)
        cap = max(self.batch_nip_min, min(self.batch_nip, backlog // max(1, self.workers)))
        while self._queue and len(taken) < self.max_batch:
            r = self._queue[0]
            if r.bound_bytes < 0:
                break
            fits = self._in_flight_bytes + r.bound_bytes <= self.memory_budget
            if r.nip >= self.solo_nip:
                if taken:  # leave it for the next admission
                    skipped.append(self._queue.popleft())
                    continue
                if not fits and self._in_flight_bytes > 0:
                    break
                self._queue.popleft()
                self._in_flight_bytes += r.bound_bytes
                self._queue.extendleft(reversed(skipped))
                return [r], True
            if not fits and (taken or self._in_flight_bytes > 0):
                break
            if taken and (nip + r.nip > cap or cols + r.B.n > self.batch_cols):
                break
            self._queue.popleft()
            self._in_flight_bytes += r.bound_bytes
            nip += r.nip
            cols += r.B.n
            taken.append(r)
            if not fits:
                break
        self._queue.extendleft(reversed(skipped))
        return taken, False

    def _next(self) -> tuple[list[Request], list[Request], bool]:
        """Block until this worker has something to do (call with the lock
        held): requests to size, or a unit of work.  Returns (unsized, unit,
        solo); both lists empty means stop."""
        while True:
            if self._stop and not self._queue:
                return [], [], False
            unsized = []
            for r in self._queue:
                if r.bound_bytes < 0 and not r.sizing:
                    r.sizing = True
                    unsized.append(r)
                    if len(unsized) == self.size_chunk:
                        break
            if unsized:
                return unsized, [], False
            unit, solo = self._admit()
            if unit:
                return [], unit, solo
            self._cv.wait()

    def _worker(self, wid: int, handle: Handle) -> None:
        torch = self._torch
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(device=self.device)
        while True:
            with self._cv:
                unsized, reqs, solo = self._next()
            if not unsized and not reqs:
                return
            if unsized:
                # admission bounds of new arrivals: one sizing launch, on this
                # worker's stream; then this worker admits
                try:
                    nips = get_nip_many([(r.A, r.B) for r in unsized], handle, stream)
                except BaseException as e:  # an invalid pair fails the whole call
                    nips = [0] * len(unsized)
                    for r in unsized:
                        r.error = e
                for r, nip in zip(unsized, nips):
                    r.nip = nip
                    r.bound_bytes = 4 * (r.A.m + 1) + nip * (4 + r.A.val.element_size())
                with self._cv:
                    self._cv.notify_all()
                continue
            now = time.perf_counter()
            for r in reqs:
                r.t_admitted = now
            failed = [r for r in reqs if r.error is not None]
            reqs = [r for r in reqs if r.error is None]
            t_launch = now
            try:
                with torch.cuda.stream(stream):
                    if not reqs:
                        outs = []
                    elif solo or len(reqs) == 1:
                        t_launch = time.perf_counter()
                        outs = [proposal(reqs[0].A, reqs[0].B, handle, stream)]
                    else:
                        pb = pack_batch([(r.A, r.B) for r in reqs], share=True)
                        t_launch = time.perf_counter()
                        outs = batch(pb, handle, stream)
                    stream.synchronize()
                done = time.perf_counter()
                for r, c in zip(reqs, outs):
                    r.result = c
                    r.t_done = done
            except BaseException as e:  # report to every request of the batch
                done = time.perf_counter()
                for r in reqs:
                    r.error = e
                    r.t_done = done
            for r in failed:
                r.t_done = done
            reqs += failed
            self.timeline.append((wid, len(reqs), now, t_launch, done))
            with self._cv:
                self._in_flight_bytes -= sum(r.bound_bytes for r in reqs)
                self.batches += 1
                self.batched_requests += len(reqs)
                self._cv.notify_all()
            for r in reqs:
                r.done.set()


def latency_summary(reqs: list[Request]) -> dict:
    lat = np.array([r.latency for r in reqs]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}
