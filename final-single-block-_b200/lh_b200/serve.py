"""Serving loop: simulation requests admitted by HBM budget and advanced
together with continuous batching.

Requests arrive over time (e.g. a Poisson stream).  The server keeps every
admitted instance's state resident on the device in one :class:`Batch`;
between RK3 steps it admits waiting requests while the HBM budget allows,
advances all live instances in shared launches, and retires instances the
moment they reach their step count (their memory then admits the next
requests).  Progress is tracked on the host (each live instance advances by
exactly the steps the batch takes while it is a member), so no device
round trip decides completion.  Results are the final states and the
time-to-completion of every request.

Host work stays off the device's critical path: initial states of arrived
requests are built by a worker thread while the device steps the live
instances, and the batch uploads an admission on a stream of its own while
queued steps run (it synchronises only to rebuild its step graph).

``run_plain`` runs the same requests one at a time through the
single-instance :class:`Engine` -- the drop-in path -- on the same arrival
clock, for comparison.
"""
from __future__ import annotations

import math
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from .capi import Batch, Desc, Engine, LHError, LH_EDEVICE, LH_ENOMEM
from .state import grids, perturbed_laminar, re_from_retau


@dataclass
class Request:
    rid: int
    desc: Desc
    seed: int
    nsteps: int
    arrival: float = 0.0  # seconds after the start of the run
    # filled by the server
    admitted: float = math.nan
    finished: float = math.nan
    result: dict | None = None
    error: str | None = None  # set when the simulation diverged (non-finite state)

    @property
    def work(self) -> float:
        """grid-point substeps of the request"""
        return self.desc.points() * 3.0 * self.nsteps


def poisson_stream(n: int, rate: float, rng: np.random.Generator, grid_choices, ny_choices,
                   retau=(100.0, 550.0), steps=(200, 5000), dt=(5e-4, 2e-3), base_seed: int = 20260005,
                   cfl: float | None = None):
    """Requests with Poisson arrivals, grids and Re_tau drawn as the serving config describes.
    Every request runs at a fixed dt drawn from `dt`; with `cfl` it runs in
    the reference's CFL mode at that number instead (its input deck uses 0.7).
    The CFL rule sees only the x and z velocities (the reference never
    assigns dthetavi, so its wall-normal term is infinite), and laminar
    starts at Re_tau above ~400 run thousands of steps with a dt that breaks
    the wall-normal limit: the oracle itself diverges on them even at CFL
    0.25, while a fixed dt of 2e-4..5e-4 stays stable.""" 
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        N = int(rng.choice(grid_choices))
        ny = int(rng.choice(ny_choices))
        rt = float(rng.uniform(*retau))
        ns = int(round(math.exp(rng.uniform(math.log(steps[0]), math.log(steps[1])))))
        dtr = float(rng.uniform(*dt))
        if cfl is None:
            d = Desc(Nx=N, Nz=N, ny=ny, Re=re_from_retau(rt), dt_mode=1, dt=dtr)
        else:
            d = Desc(Nx=N, Nz=N, ny=ny, Re=re_from_retau(rt), dt_mode=0, CFL=cfl)
        out.append(Request(k, d, base_seed + 1000 * k, max(1, ns), t))
    return out


def initial_state(req: Request):
    yu, yv = grids(req.desc)
    return perturbed_laminar(req.desc, req.seed, yu, yv)


@dataclass
class ServeStats:
    wall: float
    requests: int
    work: float
    p50: float
    p99: float
    mean_live: float
    max_live: int
    rejected_at_peak: int = 0
    ttc: list = field(default_factory=list)

    @property
    def throughput(self) -> float:
        return self.work / self.wall if self.wall > 0 else 0.0


def serve(requests, hbm_budget: int, max_chunk: int = 50, keep_results: bool = True,
          time_scale: float = 1.0, clock=time.perf_counter, batch_factory=Batch,
          state_fn=None, prefetch: int = 4) -> ServeStats:
    """Continuous batching over `requests` (sorted by arrival).

    time_scale < 1 compresses the arrival times (a faster replay of the
    stream); the reported time-to-completion is in real seconds.  Up to
    `prefetch` arrived requests have their initial states built ahead by
    worker threads while the device steps (0: built on the scheduling thread
    at admission); admission itself is unchanged: every arrived request that
    fits the budget joins before the next step.
    batch_factory/state_fn default to the device batch and the synthetic
    initial state; tests substitute host fakes to check the scheduling.
    """
    reqs = sorted(requests, key=lambda r: r.arrival)
    state_fn = state_fn or initial_state
    b = batch_factory(hbm_budget)
    pool = ThreadPoolExecutor(max_workers=2) if prefetch > 0 else None
    pending: dict[int, object] = {}  # rid -> future of the initial state
    queue: list[Request] = []
    live: dict[int, tuple[Request, int]] = {}  # slot -> (request, remaining steps)
    nxt = 0
    t0 = clock()
    live_samples = []
    done = 0

    def state_of(r: Request, block: bool):
        if pool is None:
            return state_fn(r)
        f = pending.get(r.rid)
        if f is None:
            f = pending[r.rid] = pool.submit(state_fn, r)
        if not block and not f.done():
            return None
        return f.result()

    try:
        while done < len(reqs):
            now = clock() - t0
            while nxt < len(reqs) and reqs[nxt].arrival * time_scale <= now:
                queue.append(reqs[nxt])
                nxt += 1
            if pool is not None:
                for r in queue[:prefetch]:
                    if r.rid not in pending:
                        pending[r.rid] = pool.submit(state_fn, r)
            # admit every arrived request in arrival order while memory allows
            # (a state the worker has started is waited for: it costs no more
            # than building it here, and the worker builds the next ones while
            # the device steps)
            while queue:
                r = queue[0]
                st = state_of(r, block=True)
                try:
                    slot = b.add(r.desc, *st)
                except LHError as e:
                    if e.code == LH_ENOMEM and live:
                        break  # wait for a retirement
                    raise
                pending.pop(r.rid, None)
                r.admitted = clock() - t0
                live[slot] = (r, r.nsteps)
                queue.pop(0)
            if not live:
                # idle until the next arrival
                if nxt < len(reqs):
                    wait = reqs[nxt].arrival * time_scale - (clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                continue
            k = min(max_chunk, min(rem for _, rem in live.values()))
            b.step(k)
            live_samples.append(len(live))
            finished = []
            for slot, (r, rem) in list(live.items()):
                rem -= k
                if rem == 0:
                    finished.append(slot)
                live[slot] = (r, rem)
            if finished:
                b.synchronize()
                tf = clock() - t0
                for slot in finished:
                    r, _ = live.pop(slot)
                    if hasattr(b, "scalars"):
                        # a diverged simulation (non-finite state) is retired with
                        # its error, as a server answers a failed request
                        try:
                            b.scalars(slot)
                        except LHError as err:
                            if err.code != LH_EDEVICE:
                                raise
                            r.error = "non-finite state"
                    if keep_results and r.error is None:
                        r.result = b.download(slot)
                    r.finished = tf
                    b.remove(slot)
                    done += 1
        b.synchronize()
    finally:
        if pool is not None:
            pool.shutdown(wait=True, cancel_futures=True)
    wall = clock() - t0
    ttc = [r.finished - r.arrival * time_scale for r in reqs]
    b.close()
    return ServeStats(wall=wall, requests=len(reqs), work=sum(r.work for r in reqs),
                      p50=float(np.percentile(ttc, 50)), p99=float(np.percentile(ttc, 99)),
                      mean_live=float(np.mean(live_samples)) if live_samples else 0.0,
                      max_live=max(live_samples) if live_samples else 0, ttc=ttc)


def run_plain(requests, keep_results: bool = True, clock=time.perf_counter, time_scale: float = 1.0) -> float:
    """The drop-in path: each request alone through the single-instance engine,
    in arrival order, none started before its arrival (the same clock as
    :func:`serve`, so the two wall times compare like for like).

    Returns the wall time; states go to ``request.result``, completion times
    to ``request.finished``."""
    t0 = clock()
    for r in sorted(requests, key=lambda q: q.arrival):
        wait = r.arrival * time_scale - (clock() - t0)
        if wait > 0:
            time.sleep(wait)
        e = Engine(r.desc)
        e.upload(*initial_state(r))
        e.step(r.nsteps)
        try:
            e.synchronize()
        except LHError as err:
            if err.code != LH_EDEVICE:
                raise
            r.error = "non-finite state"
        if keep_results and r.error is None:
            r.result = e.download()
        r.finished = clock() - t0
        e.close()
    return clock() - t0
