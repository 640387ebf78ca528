"""Device-resident continuous-batching service for KPM / MSD jobs.

Requests name a model (an operator set kept resident on the GPU), a job kind
(`"dos"`: Jackson-KPM DOS moments; `"msd"`: stepwise commutator MSD), the
number of moments, the number of random vectors and a seed.  The scheduler
admits a waiting request as soon as a slot and enough of the HBM budget are
free.  Each slot owns a CUDA stream and a host worker thread.  The engine
calls release the GIL, so the work of all admitted requests overlaps on the
device; a request that arrives while others run starts without waiting for
them to finish.  Latency is measured from arrival to result.  The results are
deterministic (fixed grids, fixed reduction orders): a request computes the
same numbers alone and in the mix.

Memory accounting: each model's H, S, velocity and engine set-up is charged
once when it is loaded.  Each job is charged its recurrence buffers (at most
six (N, b) blocks) while it runs, and the charge is released when it ends.  A
job is admitted only while the charges stay within the HBM budget and the
device reports the job's bytes free (cudaMemGetInfo), so an estimate that
falls short of real use delays admission instead of failing a job.
"""
from __future__ import annotations

import heapq
import queue
import threading
import time
from dataclasses import dataclass, field
from types import SimpleNamespace
from typing import Any

import numpy as np

from . import kpm


@dataclass(order=True)
class Request:
    arrival: float
    rid: int = field(compare=False)
    model: str = field(compare=False)
    kind: str = field(compare=False)        # "dos" | "msd"
    n_moments: int = field(compare=False)
    vectors: int = field(compare=False)
    seed: int = field(compare=False)
    times_fs: Any = field(compare=False, default=None)


@dataclass
class Result:
    rid: int
    arrival: float
    start: float
    end: float
    value: Any
    model: str
    kind: str
    footprint: int

    @property
    def latency(self):
        return self.end - self.arrival


class ResidentModel:
    """Operators of one model uploaded once; engines per precision."""

    def __init__(self, name, model, bounds, precision="mixed", energies=None, replicas=4):
        from .config import RunConfig
        from .operators import build_operators
        self.name = name
        self.n = model.n
        self.cfg = RunConfig(energy_eV=np.linspace(bounds[0] * .9, bounds[1] * .9, 101) if energies is None
                             else energies, time_fs=[0., 1.], spectral_bounds=bounds, axes=("x",),
                             include_vac=False, stochastic_method="stepwise", precision=precision,
                             moment_doubling=True, n_moments=256)
        self.ops = build_operators(model, self.cfg)
        self.bounds = bounds
        nnz = model.H.nnz + sum(v.nnz for v in model.velocity.values())
        self.footprint = int(nnz * 24 + model.n * 64)
        # engine replicas share the uploaded matrices; each serves one job at a time
        self.pool: "queue.Queue" = queue.Queue()
        engines = [self.ops.native] + [self.ops.native.replica() for _ in range(replicas - 1)]
        for eng in engines:
            self.pool.put(SimpleNamespace(native=eng, inner=eng.inner))

    def job_bytes(self, req):
        cols = req.vectors * (2 if req.kind == "msd" else 1)
        return int(6 * self.n * cols * 16)

    def run(self, req):
        import torch
        c, a = kpm.scaling(self.cfg)
        from .devstats import random_phases
        B = random_phases(self.n, req.seed, range(req.vectors))  # generated on the device
        ops = self.pool.get()
        try:
            if req.kind == "dos":
                mu = ops.native.moments(B, req.n_moments, c, a)
                return mu.cpu().numpy()
            from dataclasses import replace
            from .stochastic import stepwise_samples
            cfg = replace(self.cfg, n_moments=req.n_moments, time_fs=np.asarray(req.times_fs, float))
            dos, nums, _ = stepwise_samples(ops, cfg, B)
            return nums["msd_A2/commutator"]
        finally:
            self.pool.put(ops)


class Server:
    """Continuous-batching scheduler over `slots` streams and an HBM budget."""

    def __init__(self, models: dict, slots=8, hbm_budget_bytes=150 * 10 ** 9):
        self.models = models
        self.slots = slots
        self.budget = hbm_budget_bytes - sum(m.footprint for m in models.values())
        if self.budget <= 0:
            raise ValueError("resident models exceed the HBM budget")
        self.lock = threading.Condition()
        self.used = 0
        self.busy = 0
        self.pending_bytes = 0  # admitted, not yet started
        self.results: list[Result] = []
        self.errors: list[tuple[int, str]] = []

    def _device_has(self, need):
        """The budget is an account of estimates; admission also requires the
        device to have the job's bytes free right now (cudaMemGetInfo), less
        what admitted jobs that have not allocated yet may still take (memory
        cached by the allocator counts as free)."""
        import torch
        if self.busy == 0:
            return True  # nothing running could free more; the allocation itself decides
        free = torch.cuda.mem_get_info()[0] + torch.cuda.memory_reserved() - torch.cuda.memory_allocated()
        return free >= need + self.pending_bytes

    def _worker(self, work: "queue.Queue", stream):
        import torch
        with torch.cuda.stream(stream):
            while True:
                item = work.get()
                if item is None:
                    return
                req, admitted = item
                model = self.models[req.model]
                with self.lock:
                    self.pending_bytes -= model.job_bytes(req)
                try:
                    value = model.run(req)
                    end = time.perf_counter()
                    res = Result(req.rid, req.arrival, admitted, end, value, req.model, req.kind,
                                 model.job_bytes(req))
                    with self.lock:
                        self.results.append(res)
                except Exception as exc:  # noqa: BLE001
                    with self.lock:
                        self.errors.append((req.rid, f"{type(exc).__name__}: {exc}"))
                finally:
                    with self.lock:
                        self.used -= model.job_bytes(req)
                        self.busy -= 1
                        self.lock.notify_all()

    def serve(self, requests, t0=None):
        """Replay `requests` (arrival offsets in seconds from start) in real time;
        return the results ordered by request id."""
        import torch
        reqs = sorted(requests)
        work: "queue.Queue" = queue.Queue()
        streams = [torch.cuda.Stream() for _ in range(self.slots)]
        threads = [threading.Thread(target=self._worker, args=(work, s), daemon=True) for s in streams]
        for th in threads:
            th.start()
        start = time.perf_counter() if t0 is None else t0
        pending: list = []
        i = 0
        while i < len(reqs) or pending:
            now = time.perf_counter() - start
            while i < len(reqs) and reqs[i].arrival <= now:
                r = reqs[i]
                heapq.heappush(pending, (r.arrival, r.rid, r))
                i += 1
            with self.lock:
                admitted = False
                while pending and self.busy < self.slots:
                    r = pending[0][2]
                    need = self.models[r.model].job_bytes(r)
                    if need > self.budget:
                        heapq.heappop(pending)
                        self.errors.append((r.rid, "request exceeds the HBM budget"))
                        continue
                    if self.used + need > self.budget or not self._device_has(need):
                        break  # wait for memory (FIFO admission)
                    heapq.heappop(pending)
                    self.used += need
                    self.pending_bytes += need
                    self.busy += 1
                    # latency counts from the real arrival time
                    r2 = Request(start + r.arrival, r.rid, r.model, r.kind, r.n_moments, r.vectors, r.seed,
                                 r.times_fs)
                    work.put((r2, time.perf_counter()))
                    admitted = True
                if not admitted:
                    next_arrival = reqs[i].arrival - (time.perf_counter() - start) if i < len(reqs) else None
                    timeout = .05 if next_arrival is None else max(0., min(.05, next_arrival))
                    self.lock.wait(timeout)
        for _ in threads:
            work.put(None)
        for th in threads:
            th.join()
        return sorted(self.results, key=lambda r: r.rid)


def poisson_stream(rate, duration, models, seed=5, moments=(512, 1024, 2048), vectors=(8, 32), msd_fraction=0.,
                   times_fs=(0., 1., 2.)):
    """Poisson arrivals at `rate` per second for `duration` seconds over the
    model names, with M and R drawn uniformly from the given sets."""
    rng = np.random.default_rng(seed)
    t, out, rid = 0., [], 0
    names = sorted(models)
    while True:
        t += rng.exponential(1 / rate)
        if t > duration:
            break
        kind = "msd" if rng.random() < msd_fraction else "dos"
        out.append(Request(t, rid, names[rng.integers(len(names))], kind, int(rng.choice(moments)),
                           int(rng.choice(vectors)), int(rng.integers(1 << 30)),
                           list(times_fs) if kind == "msd" else None))
        rid += 1
    return out


def latency_summary(results):
    lat = np.array([r.latency for r in results])
    busy = np.array([r.end - r.start for r in results])
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_service_s": float(busy.mean()) if len(busy) else None}
