"""Serving: a request loop over one resident store and several resident banks.

A request is one segment to analyse with one of the server's banks (its own duration, bank
size and seed).  Each worker is a child context (exm_ctx_create_sharing) that borrows the
parent's resident tables and holds one bank and one workspace on its own CUDA stream, in its
own host thread (the ctypes calls release the GIL), so requests of different banks and
segments run on the device at the same time.

Admission is continuous: whenever a worker finishes, the scheduler admits the oldest queued
request that has an idle worker for its bank, or whose bank can get a new worker within the
HBM budget (the workspace a worker needs is first estimated from its bank's shape), up to a
worker limit; once a worker of a bank has run, the bank's measured workspace replaces the estimate.
Every worker uses the same gather launch shape, so a request's result does not depend
on what else is running (bitwise).  Requests on the device at once get stream priorities in the
order they started, so the oldest one's gather leads and the others fill its gaps.
"""

import threading
import time
from collections import deque
from concurrent.futures import Future

import numpy as np

from . import _lib
from .pe import prepare
from .segments import read_segments
from .store import upload_store


def workspace_bytes(nm, n_time, n_nodes, n_lags, nfreq, nwalk):
    """device bytes one worker's workspace takes for a bank of nm templates (as exm_pe_intrinsic
    sizes it): FFT and trajectories, selection, tap descriptors, partial sums, bank copies"""
    nmc = min(nm, 8192)
    per_lag = nmc * nwalk * 20
    rc = max(1, min(n_lags, (8 << 30) // max(per_lag, 1)))
    b = 2 * nmc * n_time * (16 + 8 + 4)                  # FFT buffer + trajectories + ln|z| residuals
    b += max(nmc * n_time, nm * 1024 + 4096) * 4 + nm * 1024 * 4
    b += nmc * nwalk * 4 + rc * 48 * (nmc + 1) * 4 + rc * per_lag
    b += (n_nodes + 1) * n_lags * nm * 8 + nm * 8 * 12 + nm * nfreq * 8
    b += 2 * nm * n_time * 16 // max(1, nm // max(nmc, 1))  # cuFFT work area (about one buffer)
    return int(b * 1.05) + (64 << 20)


class Scheduler:
    """admission by workspace budget; no device work (the server drives it)

    workers: key -> list of worker ids; a new worker for key costs cost(key) bytes.  A request whose
    bank has no worker may evict idle workers of banks with no queued requests to get budget or a
    worker slot; a request whose bank has workers, all busy, gets another only from free budget and
    slots, else it waits for one of them."""

    def __init__(self, budget, cost, max_workers):
        self.budget, self.cost, self.max_workers = int(budget), cost, int(max_workers)
        self.used = 0
        self.workers = {}       # key -> list of worker ids
        self.busy = set()
        self.next_id = 0
        self.queue = deque()

    def n_workers(self):
        return sum(len(v) for v in self.workers.values())

    def push(self, item, key):
        self.queue.append((item, key))

    def _take_worker(self, key):
        mine = self.workers.get(key, [])
        for w in mine:
            if w not in self.busy:
                return w, False, []
        c = self.cost(key)
        evicted = []
        # make room by closing idle workers of other banks (never a busy one) -- only for a bank that has
        # no worker at all: a bank whose workers are busy waits for one, since opening a worker (context,
        # workspace, FFT plans, graph capture) costs more than a segment
        while mine == [] and (self.used + c > self.budget or self.n_workers() >= self.max_workers):
            w = self._evict_one(key)
            if w is None:
                break
            evicted.append(w)
        if self.n_workers() < self.max_workers and self.used + c <= self.budget:
            w = self.next_id
            self.next_id += 1
            self.workers.setdefault(key, []).append(w)
            self.used += c
            return w, True, evicted
        return None, False, evicted

    def _evict_one(self, key_needed):
        waiting = {k for _, k in self.queue}
        for key, ws in self.workers.items():
            if key == key_needed or key in waiting:   # a worker whose bank has queued work stays
                continue
            for w in ws:
                if w not in self.busy:
                    ws.remove(w)
                    self.used -= self.cost(key)
                    return w
        return None

    def admit(self):
        """the oldest admissible queued item: (item, key, worker id, new worker?, evicted worker ids),
        or (None, None, None, False, evicted worker ids) when nothing can start now"""
        evicted_all = []
        for i, (item, key) in enumerate(self.queue):
            w, new, ev = self._take_worker(key)
            evicted_all += ev
            if w is not None:
                del self.queue[i]
                self.busy.add(w)
                return item, key, w, new, evicted_all
        return None, None, None, False, evicted_all

    def release(self, w):
        self.busy.discard(w)

    def forget(self, w):
        """drop worker w (one that could not be opened): its slot and budget are free again"""
        self.busy.discard(w)
        for key, ws in self.workers.items():
            if w in ws:
                ws.remove(w)
                self.used -= self.cost(key)
                return

    def recost(self, key, new_cost, set_cost):
        """replace key's per-worker cost (an estimate by a measured figure); set_cost(key, c) updates the
        table self.cost reads, and the budget in use follows for key's live workers"""
        old = self.cost(key)
        set_cost(key, int(new_cost))
        self.used += (int(new_cost) - old) * len(self.workers.get(key, []))


class _Worker:
    def __init__(self, parent, bank, store, prior, ymin, graph=False):
        # the context may take what the device has (the scheduler keeps the sum within its budget)
        self.ctx = _lib.Context(share_store_of=parent)
        self.ctx.set_graph(graph)
        self.priority = 0
        self.prio_range = self.ctx.set_priority(0)     # (greatest, least)
        self.bank = bank.clone_for(self.ctx)
        prepare(self.bank, store, prior, ymin)

    def prioritise(self, rank):
        """stream priority for a request that starts while `rank` others are on the device: the
        oldest request leads (greatest priority), later ones fill its gaps"""
        greatest, least = self.prio_range
        p = min(least, greatest + rank)
        if p != self.priority:
            self.ctx.set_priority(p)
            self.priority = p

    def run(self, segments, row, seed, n_loud, n_random):
        seg = read_segments(segments, [row])       # as pe_intrinsic(rows=[row]) reads it
        return self.ctx.pe_intrinsic(seg["d_H"], seg["d_L"], seg["sig2_H"], seg["sig2_L"],
                                     np.array([seed + row], np.int64), n_loud, n_random)

    def close(self):
        self.ctx.close()


class Request:
    __slots__ = ("rid", "key", "segments", "row", "seed", "t_arrival", "t_start", "t_done", "future")

    def __init__(self, rid, key, segments, row=0, seed=0, t_arrival=None):
        self.rid, self.key, self.segments, self.row, self.seed = rid, key, segments, row, seed
        self.t_arrival = time.perf_counter() if t_arrival is None else t_arrival
        self.t_start = self.t_done = None
        self.future = Future()


class Server:
    """continuous-batching request loop on one GPU

    store   the node tables (resident once, on the parent context)
    banks   dict key -> exmarg_b200.MassBank (each kept resident on its workers)
    graph   workers replay each segment as one captured CUDA graph (exm_ctx_set_graph)
    """

    def __init__(self, store, banks, device=0, hbm_budget=None, max_workers=4, prior="volume", ymin=0.1267,
                 n_loud=1024, n_random=1024, graph=False):
        self.parent = _lib.context(device)
        upload_store(store, self.parent)
        self.store, self.banks = store, banks
        self.prior, self.ymin, self.n_loud, self.n_random = prior, ymin, n_loud, n_random
        self.graph = graph
        spec = store.tables[0].shape if store.tables[0] is not None else store.spec.shape
        n_lags = spec[0]
        nwalk = lambda b: (n_loud + n_random) if n_loud > 0 else b.n_time
        self.cost = {k: workspace_bytes(b.u.size, b.n_time, len(store.tables), n_lags, b.W.shape[1], nwalk(b))
                     for k, b in banks.items()}
        if hbm_budget is None:
            free, _ = _lib.device_memory(device)
            hbm_budget = int(0.85 * free)
        self.sched = Scheduler(hbm_budget, lambda k: self.cost[k], max_workers)
        self.measured = set()
        self.n_created = self.n_evicted = 0   # workers opened and closed for budget (diagnostics)
        self.running = set()            # workers with a request on the device
        self.workers = {}
        self.lock = threading.Condition()
        self.done = []
        self._threads = []
        self._stop = False

    def _worker_for(self, wid, key):
        if wid not in self.workers:
            self.workers[wid] = _Worker(self.parent, self.banks[key], self.store, self.prior, self.ymin, self.graph)
            self.n_created += 1
        return self.workers[wid]

    def _run(self, req, wid):
        try:
            w = self.workers[wid]
            with self.lock:
                rank = len(self.running)
                self.running.add(wid)
            w.prioritise(rank)
            req.t_start = time.perf_counter()
            lnl, lnb = w.run(req.segments, req.row, req.seed, self.n_loud, self.n_random)
            req.t_done = time.perf_counter()
            used = w.ctx.bytes
            req.future.set_result((lnl[0], float(lnb[0])))
        except BaseException as e:   # the request fails, the server goes on
            req.t_done = time.perf_counter()
            used = None
            req.future.set_exception(e)
        with self.lock:
            self.running.discard(wid)
            if used is not None and req.key not in self.measured:   # the estimate gives way to the measured size
                self.measured.add(req.key)
                self.sched.recost(req.key, used, self.cost.__setitem__)
            self.sched.release(wid)
            self.done.append(req)
            self.lock.notify_all()

    def _dispatch(self):
        """admit what can run now; returns the number admitted"""
        n = 0
        while True:
            with self.lock:
                req, key, wid, new, evicted = self.sched.admit()
            for e in evicted:   # idle workers of other banks, closed to free their budget
                w = self.workers.pop(e, None)
                if w is not None:
                    w.close()
                    self.n_evicted += 1
            if req is None:
                return n
            if new:
                try:
                    self._worker_for(wid, key)
                except Exception as e:   # the worker could not open (e.g. device memory): its request fails
                    with self.lock:
                        self.sched.forget(wid)
                    req.t_done = time.perf_counter()
                    req.future.set_exception(e)
                    with self.lock:
                        self.done.append(req)
                        self.lock.notify_all()
                    continue
            t = threading.Thread(target=self._run, args=(req, wid), daemon=True)
            t.start()
            self._threads.append(t)
            n += 1

    def submit(self, req):
        with self.lock:
            self.sched.push(req, req.key)
        self._dispatch()
        return req.future

    def serve(self, requests, arrivals=None):
        """submit requests at their arrival offsets (seconds from now; None: all at once) and wait for
        every result.  returns the requests (with their times and futures)"""
        t0 = time.perf_counter()
        pending = list(requests)
        offs = [0.0] * len(pending) if arrivals is None else list(arrivals)
        i = 0
        while i < len(pending) or any(not r.future.done() for r in pending):
            now = time.perf_counter() - t0
            while i < len(pending) and offs[i] <= now:
                pending[i].t_arrival = t0 + offs[i]
                with self.lock:
                    self.sched.push(pending[i], pending[i].key)
                i += 1
            self._dispatch()
            with self.lock:
                wait = (offs[i] - (time.perf_counter() - t0)) if i < len(pending) else 0.05
                self.lock.wait(timeout=max(0.0005, min(wait, 0.05)))
        for t in self._threads:
            t.join()
        self._threads = []
        return pending

    def close(self):
        for w in self.workers.values():
            w.close()
        self.workers = {}


def latency_stats(requests):
    """arrival-to-result latency percentiles, throughput over the served window, and the service time
    (start to result) apart from the queueing"""
    done = [r for r in requests if r.t_done is not None]
    lat = np.array([r.t_done - r.t_arrival for r in done])
    svc = np.array([r.t_done - r.t_start for r in done if r.t_start is not None])
    t0 = min(r.t_arrival for r in requests)
    t1 = max(r.t_done for r in done)
    return {"requests": len(lat), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "segments_per_s": len(lat) / (t1 - t0),
            "service_ms_p50": float(np.percentile(svc, 50) * 1e3) if svc.size else None,
            "service_ms_max": float(svc.max() * 1e3) if svc.size else None}
