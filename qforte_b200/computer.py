"""``Computer``: the state-vector engine, resident in HBM.

The drop-in for QForte's ``Computer`` (computer.h:22-185, bound at
bindings.cc:149-191): same constructor, same methods, same results; the
complex128 amplitudes live on the GPU and every operation is a libqfb.so
kernel.  Reference behaviours kept on purpose:

* ``apply_operator`` applies each term's circuit in gate order (the last gate
  acts leftmost), exactly as computer.cc:80-91 does, also for circuits that
  are not canonical;
* ``direct_op_exp_val`` is <psi| apply_operator(O) psi> (the shipped serial
  build, computer.cc:753-771);
* ``direct_pauli_circ_exp_val`` reproduces get_pauli_permuted_idx
  (computer.cc:850-935) bit for bit, including its sign convention for Y;
* ``direct_gate_exp_val`` leaves the gate applied to the state and returns 0,
  which is what computer.cc:937-954 does (it reads the zeroed scratch vector).
"""

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check, cplx, lib, ptr
from .circuit import Circuit
from .device import DeviceProg, pack_gates, prog_from_strings, sum_from_terms
from .gate import Gate, make_gate
from .pauli import ipow_mul
from .qubit_basis import QubitBasis
from .qubit_operator import QubitOperator, to_string

__all__ = ["Computer", "ComputerC64", "inner_product", "prepare_computer_from_circuit",
           "prepare_computer_from_gates", "add_gate_to_computer", "set_sampling_seed"]


_SEED = [int.from_bytes(__import__("os").urandom(8), "little")]


# ---- objects of the reference's own module (duck typing) -------------------
# The entry points below also take the reference's pybind Gate, Circuit,
# QubitOperator and QubitOpPool (bindings.cc:193-218 and the classes around
# them): a gate is rebuilt from gate_id(), target(), control() and
# parameter() by make_gate, the same construction as the reference's
# (make_gate.cc:18-235); circuits, operators and pools from gates() and
# terms().  So a caller may keep the reference's object model and swap in
# this Computer alone.


def _as_gate(g):
    if isinstance(g, Gate):
        return g
    p = g.parameter() if g.has_parameter() else None
    # the adjoint of a parameter-free gate that is not its own inverse is
    # labelled adj(label) (gate.cc:172-177): rebuild the gate, then take it
    label, depth = g.gate_id(), 0
    while label.startswith("adj(") and label.endswith(")"):
        label, depth = label[4:-1], depth + 1
    out = make_gate(label, g.target(), g.control(), 0.0 if p is None else float(p))
    for _ in range(depth):
        out = out.adjoint()
    return out


def _as_circuit(c):
    if isinstance(c, Circuit):
        return c
    out = Circuit()
    for g in c.gates():
        out.add(_as_gate(g))
    return out


def _as_operator(qo):
    if isinstance(qo, QubitOperator):
        return qo
    out = QubitOperator()
    for coeff, circ in qo.terms():
        out.add(complex(coeff), _as_circuit(circ))
    return out


def _as_pool(pool):
    from .sq_op_pool import QubitOpPool
    if isinstance(pool, QubitOpPool):
        return pool
    out = QubitOpPool()
    for coeff, op in pool.terms():
        out.add(complex(coeff), _as_operator(op))
    return out


def set_sampling_seed(seed):
    """Start the process-wide seed sequence of Computer's measurement draws
    (the reference's draws are unseeded; equal seeds here give equal draws)."""
    _SEED[0] = int(seed) & ((1 << 64) - 1)


def _next_seed():
    s = _SEED[0]
    _SEED[0] = (s + 0xD1B54A32D192ED03) & ((1 << 64) - 1)
    return s


def _new_state(nqubit, nbatch=1):
    h = ctypes.c_void_p()
    check(lib().qfb_state_create(int(nqubit), int(nbatch), ctypes.byref(h)), "qfb_state_create")
    return h


# ---------------------------------------------------------------------------
# circuit plans: runs of gates and fused Pauli-exponential segments
# ---------------------------------------------------------------------------


class _Plan:
    __slots__ = ("ops", "nqubit_needed")

    def __init__(self, ops, nq):
        self.ops = ops
        self.nqubit_needed = nq


def _plan_for(circ):
    plan = circ._plan
    if plan is not None:
        return plan
    gates = circ._gates()
    segs = sorted(circ._pexp or [], key=lambda s: s[0])
    ops = []
    pos = 0
    run_strings = []

    def flush_strings():
        if run_strings:
            xs = [s[0] for s in run_strings]
            zs = [s[1] for s in run_strings]
            th = [s[2] for s in run_strings]
            dp = DeviceProg(np.array(xs, dtype=np.uint64), np.array(zs, dtype=np.uint64),
                            np.array(th), np.zeros(len(th), dtype=np.int32), 1)
            ops.append(("p", dp))
            run_strings.clear()

    def flush_gates(a, b):
        if b > a:
            flush_strings()
            ops.append(("g", pack_gates(gates[a:b])))

    for (s, e, x, z, th) in segs:
        if s < pos:  # overlapping annotation: ignore it, the gates stay
            continue
        flush_gates(pos, s)
        run_strings.append((x, z, th))
        pos = e
    flush_gates(pos, len(gates))
    flush_strings()
    plan = _Plan(ops, circ.num_qubits())
    circ._plan = plan
    return plan


class Computer:
    """A quantum computer with ``nqubits`` qubits in the state |0...0>, or a
    deep copy of another Computer (``Computer(other)``)."""

    def __init__(self, nqubits, print_threshold=1.0e-6):
        self._h = None
        if isinstance(nqubits, Computer):
            other = nqubits
            self._n = other._n
            self._thr = other._thr
            self._h = _new_state(self._n)
            check(lib().qfb_state_copy(self._h, other._h), "Computer copy")
        else:
            n = int(nqubits)
            if n < 1:
                raise ValueError(f"Computer needs at least one qubit, got {n}")
            self._n = n
            self._thr = float(print_threshold)
            self._h = _new_state(n)
        self._timings = []

    def __del__(self):
        try:
            if self._h:
                lib().qfb_state_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # ---- basic properties ------------------------------------------------
    def get_nqubit(self):
        return self._n

    def get_nbasis(self):
        return 1 << self._n

    def _swap_in(self, h):
        old = self._h
        self._h = h
        lib().qfb_state_destroy(old)

    def device_ptr(self):
        return lib().qfb_state_device_ptr(self._h)

    def tensor(self):
        """The amplitudes as a torch complex128 CUDA tensor sharing this
        Computer's memory (valid while the Computer lives)."""
        import torch

        n = 1 << self._n

        class _Iface:
            __cuda_array_interface__ = {"shape": (n, 2), "typestr": "<f8",
                                        "data": (int(self.device_ptr()), False), "version": 2}

        return torch.view_as_complex(torch.as_tensor(_Iface(), device="cuda"))

    # ---- state setting / reading (computer.cc:40-54, bindings.cc:172-187) ---
    def reset(self):
        check(lib().qfb_state_reset(self._h))

    def null_state(self):
        check(lib().qfb_state_null(self._h))

    def set_state(self, state):
        idx = np.array([b.index() if isinstance(b, QubitBasis) else int(b) for b, _ in state],
                       dtype=np.uint64)
        val = np.array([complex(c) for _, c in state], dtype=np.complex128)
        check(lib().qfb_state_set_basis(self._h, 0, ptr(idx), ptr(val), len(state)))

    def set_coeff_vec(self, c_vec):
        a = np.ascontiguousarray(np.asarray(c_vec, dtype=np.complex128).reshape(-1))
        check(lib().qfb_state_upload(self._h, 0, ptr(a), a.shape[0]))

    set_coeff_vec_from_numpy = set_coeff_vec

    def get_coeff_array(self):
        out = np.empty(1 << self._n, dtype=np.complex128)
        check(lib().qfb_state_download(self._h, 0, ptr(out), out.shape[0]))
        return out

    def get_coeff_vec(self):
        return self.get_coeff_array().tolist()

    def coeff(self, basis):
        idx = basis.index() if isinstance(basis, QubitBasis) else int(basis)
        out = np.zeros(1, dtype=np.complex128)
        check(lib().qfb_state_get_amp(self._h, 0, idx, ptr(out)))
        return complex(out[0])

    def get_timings(self):
        return list(self._timings)

    def clear_timings(self):
        self._timings.clear()

    # ---- gates and circuits (computer.cc:93-128) --------------------------
    def _check_qubits(self, nq):
        if nq > self._n:
            raise ValueError(f"circuit acts on qubit {nq - 1} of a {self._n}-qubit Computer")

    def apply_circuit(self, qc):
        qc = _as_circuit(qc)
        plan = _plan_for(qc)
        self._check_qubits(plan.nqubit_needed)
        one = np.ones(1)
        for kind, obj in plan.ops:
            if kind == "g":
                check(lib().qfb_apply_gates(self._h, ptr(obj), obj.shape[0]), "apply_circuit")
            else:
                check(lib().qfb_prog_apply(obj.h, self._h, ptr(one), 1, 1), "apply_circuit")

    apply_circuit_safe = apply_circuit

    def apply_gate(self, qg):
        qg = _as_gate(qg)
        self._check_qubits(max(qg.target(), qg.control()) + 1)
        arr = pack_gates([qg])
        check(lib().qfb_apply_gates(self._h, ptr(arr), 1), "apply_gate")

    apply_gate_safe = apply_gate

    def apply_constant(self, a):
        check(lib().qfb_scale(self._h, cplx(a)))

    # ---- operators (computer.cc:80-91, :753-848) ---------------------------
    def apply_operator(self, qo):
        qo = _as_operator(qo)
        pt = qo._pauli_terms(applied=True)
        if pt is not None:
            ds = sum_from_terms(pt)
            self._check_qubits(ds.maxbit)
            h = _new_state(self._n)
            try:
                check(lib().qfb_sum_apply(ds.h, h, self._h), "apply_operator")
            except Exception:
                lib().qfb_state_destroy(h)
                raise
            self._swap_in(h)
            return
        # terms with general gates: copy, apply the circuit, scale, accumulate
        acc = _new_state(self._n)
        tmp = _new_state(self._n)
        try:
            check(lib().qfb_state_null(acc))
            for c, circ in qo.terms():
                check(lib().qfb_state_copy(tmp, self._h))
                t = Computer.__new__(Computer)
                t._h, t._n, t._thr, t._timings = tmp, self._n, self._thr, []
                t.apply_circuit(circ)
                t._h = None
                check(lib().qfb_axpy(acc, cplx(c), tmp))
        except Exception:
            lib().qfb_state_destroy(acc)
            raise
        finally:
            lib().qfb_state_destroy(tmp)
        self._swap_in(acc)

    def _expval_terms(self, terms, segments=None, nsegment=1):
        ds = sum_from_terms(terms, segments, nsegment)
        self._check_qubits(ds.maxbit)
        out = np.zeros(nsegment, dtype=np.complex128)
        check(lib().qfb_sum_expval(ds.h, self._h, self._h, ptr(out)), "expectation value")
        return out

    def direct_op_exp_val(self, qo):
        qo = _as_operator(qo)
        pt = qo._pauli_terms(applied=True)
        if pt is not None:
            return complex(self._expval_terms(pt)[0])
        tmp = Computer(self)
        tmp.apply_operator(qo)
        return inner_product(self, tmp)

    def direct_oppl_exp_val(self, qopl):
        qopl = _as_pool(qopl)
        return self._pool_expvals(qopl, range(len(qopl)))

    def direct_idxd_oppl_exp_val(self, qopl, idxs):
        qopl = _as_pool(qopl)
        return self._pool_expvals(qopl, list(idxs))

    def _pool_expvals(self, qopl, idxs):
        pool = qopl.terms()
        terms, seg = [], []
        for k, i in enumerate(idxs):
            pt = pool[i][1]._pauli_terms(applied=True)
            if pt is None:
                return [self.direct_op_exp_val(pool[i][1]) * pool[i][0] for i in idxs]
            terms.extend(pt)
            seg.extend([k] * len(pt))
        if not idxs:
            return []
        vals = self._expval_terms(terms, seg, len(idxs))
        return [complex(vals[k]) * pool[i][0] for k, i in enumerate(idxs)]

    def direct_oppl_exp_val_w_mults(self, qopl, mults):
        qopl = _as_pool(qopl)
        pool = qopl.terms()
        terms, seg = [], []
        for k, (pc, op) in enumerate(pool):
            for l, (c, circ) in enumerate(op.terms()):
                m = circ._applied_pauli_masks()
                if m is None:
                    return self._w_mults_generic(pool, mults)
                x, z, e = m
                terms.append((ipow_mul(complex(mults[l]) * pc * c, e), x, z))
                seg.append(k)
        if not pool:
            return []
        return [complex(v) for v in self._expval_terms(terms, seg, len(pool))]

    def _w_mults_generic(self, pool, mults):
        out = []
        for pc, op in pool:
            r = 0j
            for l, (c, circ) in enumerate(op.terms()):
                r += complex(mults[l]) * pc * c * self.direct_circ_exp_val(circ)
            out.append(r)
        return out

    def direct_circ_exp_val(self, qc):
        qc = _as_circuit(qc)
        m = qc._applied_pauli_masks()
        if m is not None:
            x, z, e = m
            return complex(self._expval_terms([(ipow_mul(1.0 + 0j, e), x, z)])[0])
        tmp = Computer(self)
        tmp.apply_circuit(qc)
        return inner_product(self, tmp)

    def direct_pauli_circ_exp_val(self, qc):
        qc = _as_circuit(qc)
        xs, ys, zs = [], [], []
        for g in qc.gates():
            lab = g.gate_id()
            if lab == "Z":
                zs.append(g.target())
            elif lab == "X":
                xs.append(g.target())
            elif lab == "Y":
                ys.append(g.target())
            else:
                raise RuntimeError("Not a valid pauli gate!")
        xm = 0
        for q in xs:
            xm ^= 1 << q
        # phase constant and effective z mask of get_pauli_permuted_idx
        cur = xm
        const = 0
        zeff = 0
        for q in ys:
            const += (cur >> q) & 1
            zeff ^= 1 << q
            cur ^= 1 << q
        for q in zs:
            const += (cur >> q) & 1
            zeff ^= 1 << q
        X = cur  # xm ^ ym
        K = ipow_mul(1.0 + 0j, len(ys))
        if const & 1:
            K = -K
        if bin(X & zeff).count("1") & 1:
            K = -K
        c = ipow_mul(K, -bin(X & zeff).count("1"))
        return complex(self._expval_terms([(c, X, zeff)])[0])

    def direct_gate_exp_val(self, qg):
        qg = _as_gate(qg)
        self.apply_gate(qg)
        return 0j

    # ---- measurement helpers (computer.cc:135-315) --------------------------
    def _rotated_copy(self, qc):
        rot = Circuit()
        for g in qc.gates():
            t = g.target()
            lab = g.gate_id()
            if lab == "X":
                rot.add_gate(make_gate("H", t, t))
            elif lab == "Y":
                rot.add_gate(make_gate("Rx", t, t, math.pi / 2))
        tmp = Computer(self)
        tmp.apply_circuit(rot)
        return tmp

    def perfect_measure_circuit(self, qc):
        qc = _as_circuit(qc)
        zm = 0
        for g in qc.gates():
            zm ^= 1 << g.target()
        tmp = self._rotated_copy(qc)
        return float(tmp._expval_terms([(1.0 + 0j, 0, zm)])[0].real)

    def sample(self, n_measurements, seed=None):
        """Basis indices of ``n_measurements`` draws from |c_i|^2 (libqfb's
        seeded sampler, qfb_state_sample; ``seed`` None takes the next seed of
        the process-wide sequence, see ``set_sampling_seed``)."""
        n = int(n_measurements)
        out = np.empty(n, dtype=np.uint64)
        if n:
            check(lib().qfb_state_sample(self._h, 0, _next_seed() if seed is None else int(seed),
                                         n, ptr(out)), "sample")
        return out

    def measure_circuit(self, qc, n_measurements):
        """computer.cc:135-183: rotate X / Y measured qubits to Z on a copy,
        draw basis states, return the product of the measured qubits' +-1."""
        qc = _as_circuit(qc)
        tmp = self._rotated_copy(qc)
        idx = tmp.sample(n_measurements)
        del tmp
        zm = 0
        for g in qc.gates():
            zm ^= 1 << g.target()
        bits = np.zeros(len(idx), dtype=np.uint64)
        for q in range(self._n):
            if (zm >> q) & 1:
                bits ^= (idx >> np.uint64(q)) & np.uint64(1)
        return (1.0 - 2.0 * bits.astype(np.float64)).tolist()

    def measure_readouts(self, qc, n_measurements):
        """computer.cc:213-259: the measured qubits' bits of each draw."""
        qc = _as_circuit(qc)
        tmp = self._rotated_copy(qc)
        idx = tmp.sample(n_measurements)
        del tmp
        tg = [g.target() for g in qc.gates()]
        return [[int((int(i) >> t) & 1) for t in tg] for i in idx]

    def measure_z_readouts_fast(self, na, nb, n_measurements):
        """computer.cc:185-211: bits na..nb of each draw, no rotation."""
        idx = self.sample(n_measurements)
        return [[int((int(i) >> l) & 1) for l in range(na, nb + 1)] for i in idx]

    # ---- printing / comparison ----------------------------------------------
    def str(self):
        c = self.get_coeff_array()
        lines = ["Computer("]
        for i in np.nonzero(np.abs(c) >= self._thr)[0]:
            lines.append(to_string(c[i]) + " " + QubitBasis(int(i)).str(self._n))
        lines.append(")")
        return "\n".join(lines)

    __str__ = str
    __repr__ = str

    def __eq__(self, other):
        if not isinstance(other, Computer):
            return NotImplemented
        if self._n != other._n:
            return False
        return bool(np.array_equal(self.get_coeff_array(), other.get_coeff_array()))

    __hash__ = None


def inner_product(a, b):
    """<a|b> (computer.cc:975-980)."""
    out = np.zeros(1, dtype=np.complex128)
    check(lib().qfb_vdot(a._h, b._h, ptr(out)), "inner_product")
    return complex(out[0])


def prepare_computer_from_circuit(nqubit, circuit):
    qc = Computer(nqubit)
    qc.apply_circuit(circuit)
    return qc


def prepare_computer_from_gates(nqubits, gates):
    qc = Computer(nqubits)
    for g in gates:
        qc.apply_gate(g)
    return qc


def add_gate_to_computer(gate, computer):
    qc = Computer(computer)
    qc.apply_gate(gate)
    return qc


class ComputerC64:
    """A complex64 state for gate-sweep throughput (qfb_c64_*): the gate path
    of Computer.apply_circuit with FP32 arithmetic and half the bytes per
    amplitude.  Not a drop-in for the reference's Computer (complex128 only)
    and never used where results are compared with it."""

    def __init__(self, nqubits):
        self._n = int(nqubits)
        h = ctypes.c_void_p()
        check(lib().qfb_c64_create(self._n, ctypes.byref(h)), "qfb_c64_create")
        self._h = h

    def get_nqubit(self):
        return self._n

    def reset(self):
        check(lib().qfb_c64_reset(self._h), "qfb_c64_reset")

    def set_coeff_vec(self, c_vec):
        v = np.ascontiguousarray(c_vec, dtype=np.complex64)
        if v.shape != (1 << self._n,):
            raise ValueError(f"expected {1 << self._n} amplitudes, got {v.shape}")
        check(lib().qfb_c64_upload(self._h, ptr(v), v.size), "qfb_c64_upload")

    def get_coeff_array(self):
        out = np.empty(1 << self._n, dtype=np.complex64)
        check(lib().qfb_c64_download(self._h, ptr(out), out.size), "qfb_c64_download")
        return out

    def apply_circuit(self, qc):
        """The circuit's gates (gates beyond the state raise ValueError)."""
        qc = _as_circuit(qc)
        arr = pack_gates(qc.gates())
        check(lib().qfb_c64_apply_gates(self._h, arr.ctypes.data if len(arr) else None, len(arr)),
              "qfb_c64_apply_gates")

    def norm2(self):
        out = ctypes.c_double()
        check(lib().qfb_c64_norm2(self._h, ctypes.byref(out)), "qfb_c64_norm2")
        return out.value

    def __del__(self):
        try:
            if self._h:
                lib().qfb_c64_destroy(self._h)
                self._h = None
        except Exception:
            pass

