"""Device-resident compiled objects and the host-side packing that feeds them.

* ``DeviceSum``  -- a grouped Pauli sum (qfb_sum): a QubitOperator, or a pool
  of them (one result segment per pool entry).
* ``DeviceProg`` -- a Pauli-exponential program (qfb_prog): an ordered list
  of exp(i phi_k P_k) with phi_k = scale_k * params[param_k].
* ``pack_gates`` -- gates to the qfb_gate array layout.

Compiled objects are cached by content (the packed arrays' digest), so
calling ``direct_op_exp_val(H)`` in a loop compiles and uploads H once.
"""

import ctypes
import hashlib
from collections import OrderedDict

import numpy as np

from . import _lib
from ._lib import GATE_DTYPE, PAULI_DTYPE, check, lib, ptr

__all__ = ["DeviceSum", "DeviceProg", "pack_gates", "sum_from_terms", "prog_from_strings"]


class DeviceSum:
    """Owner of a qfb_sum handle."""

    __slots__ = ("h", "nterms", "ngroups", "nsegment", "maxbit", "__weakref__")

    def __init__(self, coeffs, xs, zs, segments=None, nsegment=1):
        coeffs = np.ascontiguousarray(coeffs, dtype=np.complex128)
        n = coeffs.shape[0]
        pa = np.empty(n, dtype=PAULI_DTYPE)
        pa["x"] = np.asarray(xs, dtype=np.uint64)
        pa["z"] = np.asarray(zs, dtype=np.uint64)
        seg = None
        if segments is not None:
            seg = np.ascontiguousarray(segments, dtype=np.int32)
        h = ctypes.c_void_p()
        check(lib().qfb_sum_create(ptr(pa), ptr(coeffs), None if seg is None else ptr(seg), n,
                                   int(nsegment), ctypes.byref(h)), "qfb_sum_create")
        self.h = h
        self.nterms = n
        self.nsegment = int(nsegment)
        ng = ctypes.c_int64(0)
        check(lib().qfb_sum_info(h, None, ctypes.byref(ng), None))
        self.ngroups = ng.value
        m = 0
        if n:
            m = int(np.bitwise_or.reduce(pa["x"] | pa["z"]))
        self.maxbit = m.bit_length()

    def __del__(self):
        try:
            if self.h:
                lib().qfb_sum_destroy(self.h)
                self.h = None
        except Exception:
            pass


class DeviceProg:
    """Owner of a qfb_prog handle."""

    __slots__ = ("h", "nstrings", "nsteps", "nparam", "maxbit", "__weakref__")

    def __init__(self, xs, zs, scale, param, nparam):
        n = len(scale)
        pa = np.empty(n, dtype=PAULI_DTYPE)
        pa["x"] = np.asarray(xs, dtype=np.uint64)
        pa["z"] = np.asarray(zs, dtype=np.uint64)
        sc = np.ascontiguousarray(scale, dtype=np.float64)
        pr = np.ascontiguousarray(param, dtype=np.int32)
        h = ctypes.c_void_p()
        check(lib().qfb_prog_create(ptr(pa), ptr(sc), ptr(pr), n, int(nparam), ctypes.byref(h)),
              "qfb_prog_create")
        self.h = h
        self.nstrings = n
        self.nparam = int(nparam)
        ns = ctypes.c_int64(0)
        check(lib().qfb_prog_info(h, None, ctypes.byref(ns), None))
        self.nsteps = ns.value
        m = int(np.bitwise_or.reduce(pa["x"] | pa["z"])) if n else 0
        self.maxbit = m.bit_length()

    def __del__(self):
        try:
            if self.h:
                lib().qfb_prog_destroy(self.h)
                self.h = None
        except Exception:
            pass


class _LRU:
    def __init__(self, cap):
        self.cap = cap
        self.d = OrderedDict()

    def get(self, k):
        v = self.d.get(k)
        if v is not None:
            self.d.move_to_end(k)
        return v

    def put(self, k, v):
        self.d[k] = v
        self.d.move_to_end(k)
        while len(self.d) > self.cap:
            self.d.popitem(last=False)


_SUMS = _LRU(64)
_PROGS = _LRU(64)


def _digest(*arrays):
    h = hashlib.blake2b(digest_size=16)
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.digest()


def sum_from_terms(terms, segments=None, nsegment=1):
    """[(coeff, x, z)] (+ per-term segment) -> cached DeviceSum."""
    n = len(terms)
    c = np.fromiter((t[0] for t in terms), dtype=np.complex128, count=n)
    x = np.fromiter((t[1] for t in terms), dtype=np.uint64, count=n)
    z = np.fromiter((t[2] for t in terms), dtype=np.uint64, count=n)
    seg = None if segments is None else np.asarray(segments, dtype=np.int32)
    key = _digest(c, x, z, np.zeros(0) if seg is None else seg, np.array([nsegment]))
    ds = _SUMS.get(key)
    if ds is None:
        ds = DeviceSum(c, x, z, seg, nsegment)
        _SUMS.put(key, ds)
    return ds


def prog_from_strings(xs, zs, scale, param, nparam, cache=True):
    xs = np.asarray(xs, dtype=np.uint64)
    zs = np.asarray(zs, dtype=np.uint64)
    scale = np.asarray(scale, dtype=np.float64)
    param = np.asarray(param, dtype=np.int32)
    if not cache:
        return DeviceProg(xs, zs, scale, param, nparam)
    key = _digest(xs, zs, scale, param, np.array([nparam]))
    dp = _PROGS.get(key)
    if dp is None:
        dp = DeviceProg(xs, zs, scale, param, nparam)
        _PROGS.put(key, dp)
    return dp


def pack_gates(gates):
    arr = np.zeros(len(gates), dtype=GATE_DTYPE)
    for k, g in enumerate(gates):
        arr[k]["target"] = g.target()
        arr[k]["control"] = g.control()
        arr[k]["mat"] = g.matrix()
    return arr


def gate_plan(gates, nqubit):
    """(tile runs, one-gate passes, bytes read and written) of applying
    ``gates`` (Gate objects) to one ``nqubit`` state under the current tile
    shape; host only."""
    arr = pack_gates(gates)
    w, s, b = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
    check(lib().qfb_gates_plan(arr.ctypes.data if len(arr) else None, len(arr), int(nqubit),
                               ctypes.byref(w), ctypes.byref(s), ctypes.byref(b)),
          "qfb_gates_plan")
    return w.value, s.value, b.value


def gate_phases(gates, nqubit):
    """(register phases, gate operations) of the tile runs of ``gates`` on one
    ``nqubit`` state under the current tile shape; host only."""
    arr = pack_gates(gates)
    p, o = ctypes.c_int64(), ctypes.c_int64()
    check(lib().qfb_gates_phases(arr.ctypes.data if len(arr) else None, len(arr), int(nqubit),
                                 ctypes.byref(p), ctypes.byref(o)), "qfb_gates_phases")
    return p.value, o.value


def gate_fused_plan(gates, nqubit, complex64=False):
    """(phases, segments, matrix entries) of the fused form of the tile runs
    of ``gates`` on one ``nqubit`` state under the current tile shape, every
    phase checked as the device reads it (ValueError on a failed check); host
    only."""
    arr = pack_gates(gates)
    p, s, e = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
    check(lib().qfb_gates_fused_plan(arr.ctypes.data if len(arr) else None, len(arr), int(nqubit),
                                     1 if complex64 else 0, ctypes.byref(p), ctypes.byref(s),
                                     ctypes.byref(e)), "qfb_gates_fused_plan")
    return p.value, s.value, e.value


def gates_config(tile_bits=0, low_bits=3, reg_bits=0, dense=0, fused=None):
    """Process-wide shape of gate runs: tile_bits 0 (default) or 4-12 for
    register-blocked shared-memory tiles, -1 for one pass per gate; reg_bits 0
    for the default register bits per thread; dense 5 or 6 to fuse runs on at
    most that many qubits into dense unitaries applied on the FP64 tensor
    cores instead (states of 10 qubits and more); fused True / False to apply
    each tile phase as fused 8 x 8 matrices on the FP64 tensor cores / its
    gates one by one (None: fused for states larger than L2)."""
    check(lib().qfb_gates_config(int(tile_bits), int(low_bits)), "qfb_gates_config")
    check(lib().qfb_gates_regs(int(reg_bits)), "qfb_gates_regs")
    check(lib().qfb_gates_dense(int(dense)), "qfb_gates_dense")
    check(lib().qfb_gates_fused(2 if fused is None else 1 if fused else 0), "qfb_gates_fused")
