"""A request loop for many concurrent dUCC drivers on one GPU.

VQE, PQE and ADAPT drivers of 10-26 qubits send energy and energy+gradient
evaluations of their current amplitudes; each driver's problem (Hamiltonian,
compiled Pauli-exponential programs) is registered once and stays on the
device.  One serving thread owns the loop:

* **continuous batching** - requests of one problem and kind that are waiting
  when a CUDA stream frees up go out together as one graph-captured evaluator
  run (a batch of parameter rows, padded to a power of two); requests that
  arrive while others are on the GPU join the next batch of their problem;
* **overlap** - up to ``streams`` batches (of different problems or of the
  same one) are in flight at once, each on its own stream with its own
  evaluator, so their kernels share the device;
* **admission against an HBM budget** - every evaluator's device bytes are
  counted; a batch is admitted only when its evaluator fits in the budget
  (idle evaluators are released oldest first to make room), otherwise its
  requests wait for running batches to finish and free memory;
* **latency accounting** - each request's time from submission to the moment
  its results are back on the host, reported as p50 / p99 beside throughput.

Every row of a batch is computed independently of the other rows, so a
request's result is the same alone and in any mix, up to the summation order
of reductions whose chunking depends on the batch width (energies agree to
1e-12 and better).
"""

import collections
import math
import queue
import threading
import time
from concurrent.futures import Future

import numpy as np

from ._lib import check, lib
from .ucc import DUCC, Evaluator

__all__ = ["Server"]


class _Req:
    __slots__ = ("key", "params", "mode", "t_submit", "future")

    def __init__(self, key, params, mode):
        self.key = key
        self.params = params
        self.mode = mode
        self.t_submit = time.perf_counter()
        self.future = Future()


class _Slot:
    """An evaluator with its pinned host buffers (one batch at a time)."""

    def __init__(self, ducc, bucket):
        import torch
        self.ev = Evaluator(ducc, bucket)
        self.bucket = bucket
        self.bytes = self.ev.device_bytes
        self.h_par = torch.empty((bucket, ducc.nparam), dtype=torch.float64).pin_memory()
        self.h_en = torch.empty(bucket, dtype=torch.float64).pin_memory()
        self.h_gr = torch.empty((bucket, ducc.nparam), dtype=torch.float64).pin_memory()
        self.d_par, self.d_en, self.d_gr = self.ev.tensors()
        self.last_used = time.perf_counter()


class _Batch:
    __slots__ = ("slot", "reqs", "stream", "event", "mode", "key", "t_launch")


class Server:
    """Serve dUCC energy / gradient requests of registered problems.

    ``hbm_budget`` bytes bound the evaluators' device memory; ``max_batch``
    bounds the rows of one run; ``streams`` bounds the batches in flight.
    """

    def __init__(self, hbm_budget=150e9, max_batch=256, streams=4, device=0):
        self.hbm_budget = float(hbm_budget)
        self.max_batch = int(max_batch)
        self.nstreams = int(streams)
        self.device = int(device)
        self._problems = {}
        self._inbox = queue.SimpleQueue()
        self._waiting = collections.OrderedDict()  # (key, mode) -> deque of _Req
        self._idle = {}                           # (key, bucket) -> [ _Slot ]
        self._live_bytes = 0
        self._peak_bytes = 0
        self._inflight = []
        self._free_streams = []
        self._thread = None
        self._stop = threading.Event()
        self._lock = threading.Lock()
        self._lat = []
        self._done = 0
        self._batches = 0
        self._rows = 0
        self._t0 = None
        self._t_last = None
        self._error = None

    # ---- problems ----------------------------------------------------------
    def register(self, key, ducc):
        """Make a compiled problem (a qforte_b200.ucc.DUCC) servable."""
        if key in self._problems:
            raise ValueError(f"problem {key!r} already registered")
        self._problems[key] = ducc

    def register_problem(self, key, hamiltonian, pool, tops, ref, pool_type=None):
        self.register(key, DUCC(hamiltonian, pool, tops, ref, pool_type))

    def _bucket_cap(self, ducc):
        """The widest batch whose evaluator stays within half the budget."""
        per_row = 2 * 16 * (1 << ducc.nqubit) + 24 * ducc.nparam
        cap = int(0.5 * self.hbm_budget // max(per_row, 1))
        if cap < 1:
            raise ValueError("one state of this problem exceeds half the HBM budget")
        return min(self.max_batch, 1 << int(math.floor(math.log2(cap))))

    # ---- client side -------------------------------------------------------
    def submit(self, key, params, with_grad=True):
        """Queue one evaluation; the future resolves to (energy, gradient or None)."""
        if key not in self._problems:
            raise KeyError(f"unknown problem {key!r}")
        p = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
        if p.shape[0] != self._problems[key].nparam:
            raise ValueError(f"expected {self._problems[key].nparam} parameters, got {p.shape[0]}")
        r = _Req(key, p, 1 if with_grad else 0)
        if self._error is not None:
            r.future.set_exception(RuntimeError(f"server failed: {self._error}"))
            return r.future
        self._inbox.put(r)
        return r.future

    # ---- lifecycle ---------------------------------------------------------
    def start(self):
        if self._thread is not None:
            return self
        self._stop.clear()
        self._thread = threading.Thread(target=self._loop, name="qfb-serving", daemon=True)
        self._thread.start()
        return self

    def stop(self):
        """Finish every submitted request, then end the loop."""
        if self._thread is None:
            return
        self._stop.set()
        self._thread.join()
        self._thread = None

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    def reset_stats(self):
        """Forget the latencies and counts so far (after a warm-up)."""
        with self._lock:
            self._lat = []
            self._done = self._batches = self._rows = 0
            self._t0 = self._t_last = None
            self._peak_bytes = self._live_bytes

    def stats(self):
        with self._lock:
            lat = np.array(self._lat) * 1e3
            span = (self._t_last - self._t0) if self._t0 is not None and self._t_last else 0.0
            out = {"completed": self._done, "batches": self._batches,
                   "mean_batch_rows": self._rows / max(self._batches, 1),
                   "peak_device_bytes": self._peak_bytes, "hbm_budget": self.hbm_budget,
                   "throughput_per_s": self._done / span if span > 0 else None}
        if lat.size:
            out["latency_ms"] = {"p50": float(np.percentile(lat, 50)),
                                 "p99": float(np.percentile(lat, 99)),
                                 "mean": float(lat.mean()), "max": float(lat.max())}
        return out

    # ---- the loop ----------------------------------------------------------
    def _loop(self):
        import torch
        try:
            torch.cuda.set_device(self.device)
            self._free_streams = [torch.cuda.Stream() for _ in range(self.nstreams)]
            while True:
                got = self._drain()
                done = self._complete()
                launched = self._launch()
                if self._stop.is_set() and not self._inflight and not self._waiting \
                        and self._inbox.empty():
                    break
                if not (got or done or launched):
                    if self._inflight:
                        time.sleep(20e-6)
                    else:
                        try:
                            r = self._inbox.get(timeout=0.005)
                            self._enqueue(r)
                        except queue.Empty:
                            pass
        except BaseException as e:  # fail every pending request loudly
            self._error = repr(e)
            for b in self._inflight:
                for r in b.reqs:
                    if not r.future.done():
                        r.future.set_exception(e)
            for dq in self._waiting.values():
                for r in dq:
                    r.future.set_exception(e)
            while not self._inbox.empty():
                self._inbox.get().future.set_exception(e)
            raise
        finally:
            self._release_all()

    def _enqueue(self, r):
        if self._t0 is None:
            self._t0 = r.t_submit
        k = (r.key, r.mode)
        dq = self._waiting.get(k)
        if dq is None:
            dq = self._waiting[k] = collections.deque()
        dq.append(r)

    def _drain(self):
        n = 0
        while True:
            try:
                r = self._inbox.get_nowait()
            except queue.Empty:
                return n
            self._enqueue(r)
            n += 1

    def _complete(self):
        n = 0
        still = []
        for b in self._inflight:
            if not b.event.query():
                still.append(b)
                continue
            s = b.slot
            en = s.h_en.numpy()
            gr = s.h_gr.numpy() if b.mode else None
            now = time.perf_counter()
            for i, r in enumerate(b.reqs):
                r.future.set_result((float(en[i]), gr[i].copy() if gr is not None else None))
                with self._lock:
                    self._lat.append(now - r.t_submit)
                    self._done += 1
            with self._lock:
                self._t_last = now
            s.last_used = now
            self._idle.setdefault((b.key, s.bucket), []).append(s)
            self._free_streams.append(b.stream)
            n += 1
        self._inflight = still
        return n

    def _slot_for(self, key, bucket, may_create):
        lst = self._idle.get((key, bucket))
        if lst:
            return lst.pop()
        if not may_create:
            return None
        ducc = self._problems[key]
        need = 2 * 16 * (1 << ducc.nqubit) * bucket
        while self._live_bytes + need > self.hbm_budget:
            if not self._evict_one():
                return None
        s = _Slot(ducc, bucket)
        self._live_bytes += s.bytes
        if self._live_bytes > self.hbm_budget:  # the estimate was short: give it back
            self._live_bytes -= s.bytes
            del s
            return None
        self._peak_bytes = max(self._peak_bytes, self._live_bytes)
        return s

    def _evict_one(self):
        best = None
        for k, lst in self._idle.items():
            for s in lst:
                if best is None or s.last_used < best[1].last_used:
                    best = (k, s)
        if best is None:
            return False
        self._idle[best[0]].remove(best[1])
        self._live_bytes -= best[1].bytes
        del best
        return True

    def _release_all(self):
        for lst in self._idle.values():
            lst.clear()
        self._idle.clear()
        self._live_bytes = 0

    def _launch(self):
        import torch
        n = 0
        blocked_oldest = False
        while self._free_streams and self._waiting:
            # the problem whose oldest request has waited longest goes first
            order = sorted(self._waiting.items(), key=lambda kv: kv[1][0].t_submit)
            started = False
            for (key, mode), dq in order:
                ducc = self._problems[key]
                take = min(len(dq), self._bucket_cap(ducc))
                bucket = 1 << int(math.ceil(math.log2(take))) if take > 1 else 1
                # while the oldest problem waits for memory, others may only
                # reuse evaluators that already exist
                slot = self._slot_for(key, bucket, may_create=not blocked_oldest)
                if slot is None:
                    blocked_oldest = True
                    continue
                reqs = [dq.popleft() for _ in range(take)]
                if not dq:
                    del self._waiting[(key, mode)]
                self._start(slot, key, mode, reqs)
                started = True
                n += 1
                break
            if not started:
                break
        return n

    def _start(self, slot, key, mode, reqs):
        import torch
        stream = self._free_streams.pop()
        P = slot.h_par.numpy()
        for i, r in enumerate(reqs):
            P[i] = r.params
        if len(reqs) < slot.bucket:
            P[len(reqs):] = reqs[-1].params
        with torch.cuda.stream(stream):
            check(lib().qfb_set_stream(stream.cuda_stream), "qfb_set_stream")
            slot.d_par.copy_(slot.h_par, non_blocking=True)
            slot.ev.run(mode)
            slot.h_en.copy_(slot.d_en, non_blocking=True)
            if mode:
                slot.h_gr.copy_(slot.d_gr, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        b = _Batch()
        b.slot, b.reqs, b.stream, b.event, b.mode, b.key = slot, reqs, stream, ev, mode, key
        b.t_launch = time.perf_counter()
        self._inflight.append(b)
        self._batches += 1
        self._rows += len(reqs)
