"""Serving form: continuous batching of beam solves on one GPU.

Requests (a beam, a law, a loading rate) arrive over time. The server admits
a request as soon as it has arrived and its device memory fits the HBM
budget, keeps every admitted solve resident on the device, and advances all
of them together with one persistent batch launch per chunk of steps (a
captured CUDA graph while the membership holds). After each chunk it reads
every member's per-step reaction, retires solves that have finished (load
fallen to `post_peak` of its peak after the peak, or the step cap reached),
frees their memory and admits waiting requests. New requests therefore join
while others are still running, and their work overlaps on the device.

`run_sequential` is the baseline: the same requests, one plain solve at a
time in arrival order, on the same GPU.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Any
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import beam as B
from .batch import Batch
from .solver import Solver

LAWKW = {
    "linear": dict(law="linear", sc=2e-3),
    "bilinear": dict(law="bilinear", s0=1e-4, sc=2e-3),
    "trilinear": dict(law="trilinear", s0=1e-4, s1=3e-4, sc=2e-3),
    "exponential": dict(law="exponential", s0=1e-4, sc=2e-3),
}


@dataclasses.dataclass
class Request:
    id: int
    arrival: float              # seconds after the start of the run
    inp: Any                    # beam arrays (beam.build), or a callable that builds them on admission
    law: str
    rate: float                 # prescribed displacement per step (m)
    max_steps: int
    post_peak: float = 0.8      # stop once |load| <= post_peak * peak after the peak
    sizes: tuple | None = None  # (nodes, bonds, per-bond sc) when inp is built on admission

    def counts(self) -> tuple:
        """(nodes, bonds, per-bond critical stretch) without building the arrays."""
        if isinstance(self.inp, dict):
            return int(self.inp["nNodes"]), int(self.inp["nBonds"]), "sc" in self.inp
        return self.sizes

    def arrays(self) -> dict:
        """The beam arrays (built now when the request holds a builder): a
        stream of large solves then keeps only admitted requests' arrays on
        the host, and only until their solvers exist."""
        return self.inp if isinstance(self.inp, dict) else self.inp()


@dataclasses.dataclass
class Result:
    id: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    peak: float
    peak_step: int
    bond_updates: float
    reactions: np.ndarray

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def device_bytes_estimate(inp: dict, per_bond_sc: bool) -> int:
    """Upper estimate of a solver's device memory (bond streams, damage state,
    per-bond sc, node arrays) used for admission before the solver exists."""
    nD = 2 * int(inp["nBonds"])
    return int(nD * (7 + 8 + (8 if per_bond_sc else 0)) * 1.15 + int(inp["nNodes"]) * 320 + (1 << 20))


class _Track:
    """Peak tracking of one solve from its per-step reactions."""

    def __init__(self, req: Request):
        self.req = req
        self.peak = 0.0
        self.peak_step = 0
        self.steps = 0
        self.hist: list[np.ndarray] = []

    def skip(self, n: int) -> None:
        """Steps run without a kept reaction (schedule trials of the autotuner)."""
        self.hist.append(np.full(n, np.nan))
        self.steps += n

    def update(self, r: np.ndarray) -> bool:
        """Append a chunk of reactions; True when the solve is finished."""
        if r.size == 0:
            return self.steps >= self.req.max_steps
        self.hist.append(r)
        a = np.abs(r)
        k = int(np.argmax(a))
        if a[k] > self.peak:
            self.peak, self.peak_step = float(a[k]), self.steps + k + 1
        self.steps += len(r)
        after = a[max(0, self.peak_step - (self.steps - len(r))):]   # this chunk's steps after the peak
        dropped = self.peak > 0 and after.size > 0 and float(after.min()) <= self.req.post_peak * self.peak
        return dropped or self.steps >= self.req.max_steps


def _new_solver(req: Request, precision: str, device: int) -> Solver:
    return Solver(req.arrays(), device=device, scheme="adr", rate=req.rate, precision=precision,
                  **LAWKW[req.law])


def run_batched(requests: list[Request], *, hbm_budget: float = 150e9, precision: str = "fp64",
                chunk: int = 100, device: int = 0, tune: bool = True,
                builders: int = 2) -> tuple[list[Result], dict]:
    """Continuous batching. Solvers of arrived requests are built by worker
    threads (host layout and upload) while the GPU steps the batch; a request
    is admitted when its estimated device memory fits the budget. Returns the
    results and run statistics."""
    pending = sorted(requests, key=lambda r: r.arrival)
    batch = Batch(precision, device)
    pool = ThreadPoolExecutor(max_workers=builders)
    creating: list = []                 # (request, future, estimate)
    active: list = []                   # (request, solver, track, admitted, bytes)
    results: list[Result] = []
    used = reserved = 0
    launches = 0
    peak_members = 0
    tuned = False
    t0 = time.perf_counter()
    try:
        while pending or active or creating:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                r = pending[0]
                nn, nb, sc = r.counts()
                est = device_bytes_estimate({"nNodes": nn, "nBonds": nb}, sc)
                if (active or creating) and used + reserved + est > hbm_budget:
                    break                   # wait for a solve to finish
                creating.append((r, pool.submit(_new_solver, r, precision, device), est))
                reserved += est
                pending.pop(0)
            for item in list(creating):
                r, fut, est = item
                if fut.done() or not active:
                    s = fut.result()
                    nbytes = int(s.info()["device_bytes"])
                    batch.add(s)
                    used += nbytes
                    reserved -= est
                    active.append((r, s, _Track(r), time.perf_counter() - t0, nbytes))
                    creating.remove(item)
            if not active:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.05)))
                continue
            peak_members = max(peak_members, len(active))
            if tune and not tuned and len(active) > 1:
                batch.tune(max(1, chunk // 16))   # trials run real steps of every member
                tuned = True
            batch.step(chunk)
            launches += 1
            done = []
            for item in active:
                r, s, tr, ta, nbytes = item
                got = (s.next_step - 1) - tr.steps
                if got > chunk:
                    tr.skip(got - chunk)
                if tr.update(s.reaction(chunk)):
                    done.append(item)
            tnow = time.perf_counter() - t0
            for item in done:
                r, s, tr, ta, nbytes = item
                batch.remove(s)
                s.close()
                used -= nbytes
                active.remove(item)
                results.append(Result(r.id, r.arrival, ta, tnow, tr.steps, tr.peak, tr.peak_step,
                                      float(r.counts()[1]) * tr.steps, np.concatenate(tr.hist)))
    finally:
        pool.shutdown(wait=True)
        batch.close()
    wall = time.perf_counter() - t0
    return results, dict(wall=wall, launches=launches, peak_members=peak_members)


def run_sequential(requests: list[Request], *, precision: str = "fp64", chunk: int = 100,
                   device: int = 0) -> tuple[list[Result], dict]:
    """Baseline: one solve at a time in arrival order (same chunking and stop rule)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    results = []
    t0 = time.perf_counter()
    for r in pending:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        ta = time.perf_counter() - t0
        s = _new_solver(r, precision, device)
        tr = _Track(r)
        while True:
            s.step(chunk)
            if tr.update(s.reaction(chunk)):
                break
        s.close()
        results.append(Result(r.id, r.arrival, ta, time.perf_counter() - t0, tr.steps, tr.peak,
                              tr.peak_step, float(r.counts()[1]) * tr.steps, np.concatenate(tr.hist)))
    return results, dict(wall=time.perf_counter() - t0)


def summary(results: list[Result], stats: dict) -> dict:
    lat = np.array([r.latency for r in results])
    bu = sum(r.bond_updates for r in results)
    return dict(solves=len(results), wall_s=stats["wall"],
                solves_per_hour=3600.0 * len(results) / stats["wall"],
                p50_latency_s=float(np.percentile(lat, 50)), p99_latency_s=float(np.percentile(lat, 99)),
                bond_updates_per_s=bu / stats["wall"], **{k: v for k, v in stats.items() if k != "wall"})
