"""A request loop for many concurrent dUCC drivers on one GPU.

VQE, PQE and ADAPT drivers of 10-26 qubits send energy and energy+gradient
evaluations of their current amplitudes; each driver's problem (Hamiltonian,
compiled Pauli-exponential programs) is registered once and stays on the
device.  One serving thread owns the loop:

* **packing** - requests of every problem small enough for the compact
  shared-memory evaluator (up to ~16 qubits), energy and energy+gradient
  alike, go out together in ONE launch (``ucc.Pack``: one CTA per request,
  whatever its problem), so a mix of small problems shares launches instead
  of each problem waiting for its own;
* **continuous batching** - requests of a larger problem and kind that are
  waiting when a CUDA stream frees up go out together as one graph-captured
  evaluator run (a batch of parameter rows, padded to a power of two);
  requests that arrive while others are on the GPU join the next launch;
* **overlap** - up to ``streams`` batches (of different problems or of the
  same one) are in flight at once, each on its own stream with its own
  evaluator, so their kernels share the device; at most one of them belongs
  to a problem of ``heavy_qubits`` or more, so long evaluations never slow
  each other down;
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
from .ucc import DUCC, Evaluator, Pack

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


class _PackSlot:
    """A Pack with its pinned host buffers (one launch at a time)."""

    def __init__(self, pack):
        import torch
        self.pack = pack
        C, MP = pack.capacity, pack.maxparam
        self.h_items = torch.zeros((C, 2), dtype=torch.int32).pin_memory()
        self.h_par = torch.zeros((C, MP), dtype=torch.float64).pin_memory()
        self.h_en = torch.empty(C, dtype=torch.float64).pin_memory()
        self.h_gr = torch.empty((C, MP), dtype=torch.float64).pin_memory()
        self.d_items, self.d_par, self.d_en, self.d_gr = pack.tensors()


class _Batch:
    __slots__ = ("slot", "reqs", "stream", "event", "mode", "key", "t_launch", "pack")


class Server:
    """Serve dUCC energy / gradient requests of registered problems.

    ``hbm_budget`` bytes bound the evaluators' device memory; ``max_batch``
    bounds the rows of one run; ``streams`` bounds the batches in flight.
    """

    def __init__(self, hbm_budget=150e9, max_batch=256, streams=4, device=0, pack=True,
                 heavy_qubits=22):
        self.hbm_budget = float(hbm_budget)
        self.max_batch = int(max_batch)
        self.nstreams = int(streams)
        self.device = int(device)
        self.pack = bool(pack)
        # problems of at least this many qubits take tens of milliseconds a
        # batch: at most one such batch runs at a time, so two never share the
        # GPU and stretch each other's latency, while smaller work overlaps it
        self.heavy_qubits = int(heavy_qubits)
        self._pack_of = {}      # key -> (group, member index) for packed problems
        self._pack_free = []    # per group: idle _PackSlot objects
        self._pack_bytes = 0    # device bytes the packs hold
        self._repack = queue.SimpleQueue()  # registrations waiting for the packs to be rebuilt
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
        """Make a compiled problem (a qforte_b200.ucc.DUCC) servable.  With
        packing on, a problem that fits the compact shared-memory evaluator
        joins the packs: on a running server the call returns once the loop
        has rebuilt them (between launches), so every request of the problem
        takes the packed path."""
        if key in self._problems:
            raise ValueError(f"problem {key!r} already registered")
        self._problems[key] = ducc
        if self.pack and self._thread is not None and self._thread.is_alive():
            done = threading.Event()
            self._repack.put(done)
            while not done.wait(0.05):
                if self._error is not None:
                    raise RuntimeError(f"server failed: {self._error}")

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

    # ---- packing -------------------------------------------------------------
    def _build_packs(self):
        """One pack group per state storage (real / complex) over the
        registered problems that take the compact shared-memory path, with a
        pack per stream; their device bytes count against the budget."""
        self._live_bytes -= self._pack_bytes
        self._pack_bytes = 0
        self._pack_free, self._pack_of = [], {}
        if not self.pack:
            return
        groups = {}
        for key, ducc in list(self._problems.items()):
            ev = ducc.evaluator(1)
            if ev.path == 2:
                groups.setdefault(ev.real_states, []).append(key)
        for keys in groups.values():
            g = len(self._pack_free)
            slots = []
            for _ in range(self.nstreams):
                pk = Pack([self._problems[k] for k in keys], capacity=self.max_batch)
                # the members' evaluators are shared by the group's packs
                need = pk.pack_bytes if slots else pk.device_bytes
                if self._live_bytes + need > self.hbm_budget:
                    break
                self._live_bytes += need
                self._pack_bytes += need
                slots.append(_PackSlot(pk))
            if not slots:
                continue
            self._pack_free.append(slots)
            for i, k in enumerate(keys):
                self._pack_of[k] = (g, i)
        self._peak_bytes = max(self._peak_bytes, self._live_bytes)

    def _launch_packs(self):
        """One packed launch per pack group with waiting requests and a free
        pack and stream: the group's oldest requests first, energy and
        gradient requests of every problem together."""
        import torch
        n = 0
        for g, free in enumerate(self._pack_free):
            if not free or not self._free_streams:
                continue
            queues = [(k, dq) for k, dq in self._waiting.items() if k[0] in self._pack_of
                      and self._pack_of[k[0]][0] == g]
            if not queues:
                continue
            queues.sort(key=lambda kv: kv[1][0].t_submit)
            ps = free.pop()
            cap = ps.pack.capacity
            reqs = []
            for k, dq in queues:
                while dq and len(reqs) < cap:
                    reqs.append(dq.popleft())
                if not dq:
                    del self._waiting[k]
                if len(reqs) == cap:
                    break
            items, par = ps.h_items.numpy(), ps.h_par.numpy()
            for i, r in enumerate(reqs):
                items[i, 0] = self._pack_of[r.key][1]
                items[i, 1] = r.mode
                par[i, :r.params.shape[0]] = r.params
            m = len(reqs)
            stream = self._free_streams.pop()
            with torch.cuda.stream(stream):
                check(lib().qfb_set_stream(stream.cuda_stream), "qfb_set_stream")
                ps.d_items[:m].copy_(ps.h_items[:m], non_blocking=True)
                ps.d_par[:m].copy_(ps.h_par[:m], non_blocking=True)
                ps.pack.launch(m)
                ps.h_en[:m].copy_(ps.d_en[:m], non_blocking=True)
                if any(r.mode for r in reqs):
                    ps.h_gr[:m].copy_(ps.d_gr[:m], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(stream)
            b = _Batch()
            b.slot, b.reqs, b.stream, b.event, b.mode, b.key = None, reqs, stream, ev, -1, g
            b.pack = ps
            b.t_launch = time.perf_counter()
            self._inflight.append(b)
            self._batches += 1
            self._rows += m
            n += 1
        return n

    # ---- the loop ----------------------------------------------------------
    def _loop(self):
        import torch
        try:
            torch.cuda.set_device(self.device)
            self._free_streams = [torch.cuda.Stream() for _ in range(self.nstreams)]
            self._build_packs()
            while True:
                got = self._drain()
                done = self._complete()
                if not self._repack.empty() and not any(b.pack for b in self._inflight):
                    self._build_packs()  # problems registered while running
                    while not self._repack.empty():
                        self._repack.get().set()
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
            if b.pack is not None:
                ps = b.pack
                en, gr = ps.h_en.numpy(), ps.h_gr.numpy()
                now = time.perf_counter()
                for i, r in enumerate(b.reqs):
                    g = gr[i, :r.params.shape[0]].copy() if r.mode else None
                    r.future.set_result((float(en[i]), g))
                    with self._lock:
                        self._lat.append(now - r.t_submit)
                        self._done += 1
                with self._lock:
                    self._t_last = now
                self._pack_free[b.key].append(ps)
                self._free_streams.append(b.stream)
                n += 1
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
        self._pack_free = []
        self._pack_of = {}
        self._pack_bytes = 0
        self._live_bytes = 0
        while not self._repack.empty():
            self._repack.get().set()

    def _launch(self):
        import torch
        n = self._launch_packs()
        blocked_oldest = False
        while self._free_streams and self._waiting:
            # the problem whose oldest request has waited longest goes first
            order = sorted(((k, dq) for k, dq in self._waiting.items() if k[0] not in self._pack_of),
                           key=lambda kv: kv[1][0].t_submit)
            heavy_busy = any(b.pack is None and self._problems[b.key].nqubit >= self.heavy_qubits
                             for b in self._inflight)
            started = False
            for (key, mode), dq in order:
                ducc = self._problems[key]
                if heavy_busy and ducc.nqubit >= self.heavy_qubits:
                    continue
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
        b.pack = None
        b.t_launch = time.perf_counter()
        self._inflight.append(b)
        self._batches += 1
        self._rows += len(reqs)
