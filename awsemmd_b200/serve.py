"""Request loop of the serving mode: MD requests (annealing or structure
prediction runs) arrive over time, are admitted onto one GPU while earlier
ones are still running (continuous batching), and return their final
coordinates and per-term energies.

Admission is by the serving handle's fixed memory: the handle allocates its
residue, request and memory-record capacities once (the HBM budget) and
`admit` answers None while a request does not fit; the loop keeps such a
request (and everything behind it, first come first served) waiting until a
collect frees room.  Latency of a request = completion time - arrival time,
both on the loop's wall clock.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the stream starts
    chain: dict     # synth.chain_arrays layout
    nsteps: int
    t_start: float = 600.0
    t_stop: float = 300.0
    seed: int = 1


@dataclass
class Completed:
    rid: int
    arrival: float
    admitted: float
    finished: float
    n_res: int
    nsteps: int
    x: np.ndarray = field(repr=False, default=None)
    energies: np.ndarray = field(repr=False, default=None)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def poisson_arrivals(n: int, rate: float, rng: np.random.Generator) -> np.ndarray:
    """Arrival times of a Poisson process with `rate` requests per second."""
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def log_uniform_lengths(n: int, lo: int, hi: int, rng: np.random.Generator) -> np.ndarray:
    """Chain lengths log-uniform in [lo, hi]."""
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=n))).astype(int).clip(lo, hi)


def run_stream(server, requests: list, chunk: int = 50, clock=time.perf_counter, sleep=time.sleep,
               keep_state: bool = True) -> list:
    """Serve `requests` in real time on `server` (an AwsemServer or anything
    with its admit / advance / progress / collect methods).  Between GPU
    chunks of `chunk` steps the loop admits every arrived request that fits,
    first come first served, and collects every finished one (a request that
    finishes inside a chunk stays frozen; its completion time is the chunk's
    end).  When the server can prepare
    requests on the host (AwsemServer.prepare), a worker thread prepares each
    request as it arrives while the GPU advances the others, and admission
    only places the prepared request."""
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    active = {}  # slot -> (request, admitted time)
    done = []
    prep = {}  # rid -> future of the prepared request
    pool = ThreadPoolExecutor(max_workers=1) if hasattr(server, "prepare") else None
    t0 = clock()
    try:
        while pending or active:
            now = clock() - t0
            if pool is not None:  # prepare every request that has arrived
                for r in pending:
                    if r.arrival > now:
                        break
                    if r.rid not in prep:
                        prep[r.rid] = pool.submit(server.prepare, r.chain, r.seed)
            while pending and pending[0].arrival <= now:
                r = pending[0]
                if pool is not None:
                    fut = prep[r.rid]
                    if not fut.done() and active:
                        break  # keep the GPU busy; admit it after the next chunk
                    what = fut.result()
                else:
                    what = r.chain
                slot = server.admit(what, r.nsteps, r.t_start, r.t_stop, r.seed)
                if slot is None:
                    if not active:
                        raise ValueError(f"request {r.rid} ({int(r.chain['n_res'])} residues) does not fit the "
                                         "empty serving handle")
                    break  # first come first served: later arrivals wait behind it
                pending.popleft()
                if pool is not None:
                    prep.pop(r.rid).result().free()
                active[slot] = (r, now)
            if not active:
                if pending and pending[0].arrival > clock() - t0:
                    sleep(max(0.0, pending[0].arrival - (clock() - t0)))
                continue
            # fixed chunks: a request that finishes inside one stays frozen
            # until its end, and stopping at every completion would leave the
            # GPU idle at each of them
            server.advance(chunk)
            now = clock() - t0
            for slot in [s for s in active if (lambda p: p[0] >= p[1])(server.progress(s))]:
                r, adm = active.pop(slot)
                x, _, e = server.collect(slot)
                done.append(Completed(r.rid, r.arrival, adm, now, int(r.chain["n_res"]), r.nsteps,
                                      x if keep_state else None, e if keep_state else None))
    finally:
        if pool is not None:
            pool.shutdown(wait=True)
            for fut in prep.values():
                fut.result().free()
    return done


def stream_stats(done: list) -> dict:
    """p50 / p99 latency, makespan and aggregate residue-steps/s of a served stream."""
    lat = np.array([d.latency for d in done])
    t_first = min(d.arrival for d in done)
    t_last = max(d.finished for d in done)
    work = float(sum(d.n_res * d.nsteps for d in done))
    return {"requests": len(done), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": t_last - t_first,
            "residue_steps": work, "residue_steps_per_s": work / max(t_last - t_first, 1e-9)}


def fifo_latencies(arrivals: np.ndarray, service: np.ndarray) -> np.ndarray:
    """Completion latencies of one-at-a-time service in arrival order (a
    single FIFO server): start = max(arrival, previous finish)."""
    out = np.empty(len(arrivals))
    free = 0.0
    for k in np.argsort(arrivals, kind="stable"):
        start = max(arrivals[k], free)
        free = start + service[k]
        out[k] = free - arrivals[k]
    return out


def plan_capacities(forcefield: dict, budget_bytes: float, precision: str = "mixed", records_per_residue: float = 420.0,
                    mean_request_residues: float = 277.0, device: int = 0) -> dict:
    """Capacities of a serving handle whose device allocation fits
    `budget_bytes`: the cost of a residue and of a memory record are read
    from the allocations of three small probe handles, and the residue
    capacity is what the budget holds at `records_per_residue` records each
    (the uniform-coefficient table; a mixed-coefficient stream needs 25%
    more per record in the mixed form)."""
    from .engine import AwsemServer

    def size(res, rec, req):
        with AwsemServer(forcefield, res, req, rec, precision, device) as s:
            return s.usage()["device_bytes"]

    b0 = size(8192, 0, 64)
    per_res = (size(16384, 0, 64) - b0) / 8192.0
    per_rec = (size(8192, 1 << 20, 64) - b0) / float(1 << 20)
    per_req = (size(8192, 0, 64 + 4096) - b0) / 4096.0
    fixed = b0 - 8192 * per_res - 64 * per_req
    req_per_res = 4.0 / mean_request_residues  # request slots: four times the mean concurrency the residues allow
    # 0.1% kept back for the rounding of residues to groups and records to stripes
    usable = 0.999 * budget_bytes - fixed
    max_res = int(usable / (per_res + records_per_residue * per_rec + req_per_res * per_req))
    max_res -= max_res % 32
    return {"max_residues": max_res, "max_memory_records": int(max_res * records_per_residue),
            "max_requests": max(64, int(req_per_res * max_res)),
            "bytes_per_residue": per_res, "bytes_per_record": per_rec, "bytes_per_request": per_req}
