"""Decode serving: a device-resident compressed dataset answering a stream of region-of-interest
requests (extent, per-axis downsampling, tolerance).

Requests are queued as they arrive; whenever the GPU is free, the server takes the queued
requests in arrival order, as many as fit in its device-memory budget (the free HBM measured
when the server starts, less a reserve), and decodes them together with one
``Dataset.decode_batch`` call (one launch per level over the bricks of all of them). The
one-request-at-a-time mode decodes the head of the queue alone. Latency is the time from a
request's arrival to the end of the call that decoded it.

The reference decodes one request per call (Core/idx2Decode.cpp:326 Decode); this module is the
serving layer around the batched decode and has no counterpart there.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

BRICK_WORKSET = 33 * 33 * 33 * 8  # bytes of one decoded FP64 brick on the device


@dataclass
class Request:
    arrival: float                       # seconds after the start of the run
    first: Tuple[int, int, int]
    last: Tuple[int, int, int]
    downsampling: Tuple[int, int, int]
    tolerance: float
    out_bytes: int = 0                   # size of the output grid
    cost: int = 0                        # device bytes the request needs while decoded
    latency: Optional[float] = None


def output_dims(first, last, downsampling):
    """Output grid of an extent (Core/idx2Common.cpp:772 GetGrid): the first sample rounded
    down and the last rounded up to the stride 2^downsampling on each axis."""
    dims = []
    for f, l, d in zip(first, last, downsampling):
        s = 1 << d
        f0 = (f // s) * s
        l1 = ((l + s - 1) // s) * s
        dims.append((l1 - f0) // s + 1)
    return tuple(dims)


def request_cost(first, last, downsampling, elem_bytes, brick=32):
    """Output bytes plus the decoded bricks (FP64) the request keeps on the device: those of
    its finest decoded level, an upper bound on the coarser ones."""
    od = output_dims(first, last, downsampling)
    out_bytes = int(np.prod(od)) * elem_bytes
    nb = 1
    for f, l, d in zip(first, last, downsampling):
        span = max(1, ((l >> d) - (f >> d)) // brick + 2)
        nb *= span
    return out_bytes, out_bytes + nb * BRICK_WORKSET


def poisson_schedule(n: int, rate: float, dims: Sequence[int], seed: int = 0, side=(32, 512), ds=(0, 3),
                     tol=(1e-6, 1e-1), elem_bytes: int = 4) -> List[Request]:
    """n requests with exponential inter-arrival times (rate per second): each a box with sides
    uniform in `side` (clamped to the field) at a uniform position, per-axis downsampling
    uniform in `ds`, tolerance log-uniform in `tol`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        first, last = [], []
        for a in range(3):
            d = int(dims[a])
            s = min(int(rng.integers(side[0], side[1] + 1)), d)
            f = int(rng.integers(0, d - s + 1))
            first.append(f)
            last.append(f + s - 1)
        dsmp = tuple(int(rng.integers(ds[0], ds[1] + 1)) if dims[a] > 1 else 0 for a in range(3))
        tl = float(math.exp(rng.uniform(math.log(tol[0]), math.log(tol[1]))))
        ob, cost = request_cost(first, last, dsmp, elem_bytes)
        out.append(Request(t, tuple(first), tuple(last), dsmp, tl, ob, cost))
    return out


@dataclass
class RunStats:
    mode: str
    requests: int
    batches: int
    elapsed_s: float
    decoded_bytes: int
    p50_ms: float
    p99_ms: float
    mean_ms: float
    max_ms: float
    mean_batch: float
    max_queue: int
    rejected: int
    gpu_ms: float = 0.0

    def as_dict(self):
        return dict(self.__dict__)


class Server:
    """Batches queued requests under a device-memory budget and decodes them.

    decode: callable taking a list of Requests and decoding them (blocking); returns the GPU
    kernel milliseconds of the call (or 0). budget: device bytes the requests of one call may
    use. clock / sleep: injectable for tests."""

    def __init__(self, decode: Callable[[List[Request]], float], budget: int, max_batch: int = 256,
                 clock: Callable[[], float] = time.perf_counter, sleep: Callable[[float], None] = time.sleep):
        self.decode = decode
        self.budget = int(budget)
        self.max_batch = max_batch
        self.clock = clock
        self.sleep = sleep

    def admit(self, queue: List[Request]) -> List[Request]:
        """The longest arrival-order prefix of the queue that fits the budget (at least the
        head, which alone never exceeds it: larger requests are rejected on arrival)."""
        batch, used = [], 0
        for r in queue:
            if len(batch) >= self.max_batch or (batch and used + r.cost > self.budget):
                break
            batch.append(r)
            used += r.cost
        return batch

    def run(self, schedule: List[Request], batched: bool = True) -> RunStats:
        pending = sorted(schedule, key=lambda r: r.arrival)
        queue: List[Request] = []
        done: List[Request] = []
        rejected = 0
        batches = 0
        batch_sizes = []
        max_queue = 0
        gpu_ms = 0.0
        t0 = self.clock()
        i = 0
        while i < len(pending) or queue:
            now = self.clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                r = pending[i]
                i += 1
                if r.cost > self.budget:
                    rejected += 1  # would never fit: refused at admission
                    continue
                queue.append(r)
            max_queue = max(max_queue, len(queue))
            if not queue:
                if i < len(pending):
                    self.sleep(max(0.0, pending[i].arrival - (self.clock() - t0)))
                continue
            batch = self.admit(queue) if batched else queue[:1]
            del queue[:len(batch)]
            gpu_ms += float(self.decode(batch) or 0.0)
            t_done = self.clock() - t0
            for r in batch:
                r.latency = t_done - r.arrival
                done.append(r)
            batches += 1
            batch_sizes.append(len(batch))
        elapsed = self.clock() - t0
        lat = np.array([r.latency for r in done]) * 1e3 if done else np.zeros(1)
        return RunStats(mode="batched" if batched else "one-at-a-time", requests=len(done), batches=batches,
                        elapsed_s=elapsed, decoded_bytes=int(sum(r.out_bytes for r in done)),
                        p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                        mean_ms=float(lat.mean()), max_ms=float(lat.max()),
                        mean_batch=float(np.mean(batch_sizes)) if batch_sizes else 0.0, max_queue=max_queue,
                        rejected=rejected, gpu_ms=gpu_ms)


def dataset_decoder(ds) -> Callable[[List[Request]], float]:
    """The decode callable of a Server over a Dataset: one decode_batch call per batch, outputs
    on the device (released when the call returns)."""
    import torch

    def decode(batch: List[Request]) -> float:
        reqs = [{"first": r.first, "last": r.last, "downsampling": r.downsampling, "tolerance": r.tolerance}
                for r in batch]
        outs = ds.decode_batch(reqs, device_out=True)
        torch.cuda.synchronize()
        del outs
        return ds.last_kernel_ms

    return decode


def free_hbm_budget(reserve: int = 4 << 30, device: int = 0) -> int:
    """Free device memory now, less a reserve for the decoder's own workspace."""
    import torch
    free, _ = torch.cuda.mem_get_info(device)
    return max(0, int(free) - int(reserve))
