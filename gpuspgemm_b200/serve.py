"""Served form: a continuous-batching request loop over device-resident operands.

Requests ``C = A * B`` (operands already on the device) arrive at any time.
Worker threads, each owning a library handle (its own side streams, scratch and
memory pool), repeatedly

1. admit waiting requests, oldest first, while the outputs they may need fit
   the memory budget: the bound is the binning phase's upper bound on C,
   ``bytes(C) <= 4 (m + 1) + NIP * (4 + sizeof(value))`` (NIP = intermediate
   products, computed on the device when the request is submitted);
2. pack the admitted requests into block-diagonal operands and run them as ONE
   batched product (``spgemm_batch_*``), so rows of different requests share
   bins and kernels;
3. hand each request its own CSR result and release its share of the budget.

With two workers, a batch is packed and launched while the previous one is
still on the GPU, and requests that arrive meanwhile join the next batch: work
from different batches overlaps on the device.  The reference has no served or
batched form; it multiplies one pair per call (proposal.cuh:85-124).
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .api import DeviceCSR, Handle, PackedBatch, batch, get_nip, pack_batch


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
    workers:       worker threads (handles); 2 lets batches overlap.
    """

    def __init__(self, memory_budget: int = 32 << 30, max_batch: int = 256, workers: int = 2,
                 device: int = 0):
        import torch
        self._torch = torch
        self.device = device
        self.memory_budget = int(memory_budget)
        self.max_batch = int(max_batch)
        self._queue: deque[Request] = deque()
        self._cv = threading.Condition()
        self._in_flight_bytes = 0
        self._stop = False
        self._handles = [Handle(device) for _ in range(workers)]
        self._sizer = Handle(device)
        self._sizer_lock = threading.Lock()
        self._next_id = 0
        self.batches = 0
        self.batched_requests = 0
        self._threads = [threading.Thread(target=self._worker, args=(h,), daemon=True)
                         for h in self._handles]
        for t in self._threads:
            t.start()

    # -- client side --------------------------------------------------------
    def submit(self, A: DeviceCSR, B: DeviceCSR, t_arrival: float | None = None) -> Request:
        """Queue C = A * B.  Computes the request's NIP on the device (its
        admission bound) and returns the Request; wait on req.done."""
        if A.n != B.m:
            raise ValueError("A.n must equal B.m")
        with self._sizer_lock:
            nip = get_nip(A, B, self._sizer)
        s = A.val.element_size()
        req = Request(A, B, t_arrival=time.perf_counter() if t_arrival is None else t_arrival,
                      nip=nip, bound_bytes=4 * (A.m + 1) + nip * (4 + s))
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
        self._sizer.close()

    # -- worker side --------------------------------------------------------
    def _admit(self) -> list[Request]:
        """Oldest-first admission under the memory budget (call with the lock
        held).  A request larger than the whole budget runs alone."""
        taken: list[Request] = []
        while self._queue and len(taken) < self.max_batch:
            r = self._queue[0]
            fits = self._in_flight_bytes + r.bound_bytes <= self.memory_budget
            if not fits and (taken or self._in_flight_bytes > 0):
                break
            self._queue.popleft()
            self._in_flight_bytes += r.bound_bytes
            taken.append(r)
            if not fits:
                break
        return taken

    def _worker(self, handle: Handle) -> None:
        torch = self._torch
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream(device=self.device)
        while True:
            with self._cv:
                while not self._stop and not self._queue:
                    self._cv.wait()
                if self._stop and not self._queue:
                    return
                reqs = self._admit()
                if not reqs:
                    self._cv.wait(timeout=0.001)
                    continue
            now = time.perf_counter()
            for r in reqs:
                r.t_admitted = now
            try:
                with torch.cuda.stream(stream):
                    if len(reqs) == 1:
                        pb = PackedBatch(np.array([0, reqs[0].A.m], np.int32),
                                         np.array([0, reqs[0].B.m], np.int32),
                                         np.array([0, reqs[0].B.n], np.int32),
                                         reqs[0].A, reqs[0].B)
                    else:
                        pb = pack_batch([(r.A, r.B) for r in reqs])
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
