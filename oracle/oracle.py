"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for the state-vector hot path.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` /
``--impl reference`` legs import this module, and only as the checker or the
timed CPU baseline.  The product package (``qforte_b200``) never imports it.

It restates, on plain term lists, the reference algorithms that drive QForte's
``Computer``:

* gate matrices and angle normalisation      ``make_gate.cc:7-235``
* gate adjoint (conjugate transpose)          ``gate.cc:135-179``
* exp(c P) as a gate circuit                  ``utils/exponentiate.py:9-87``
* first-order Trotter product                 ``utils/trotterization.py:10-57``
* dUCC energy (``measure_energy``)            ``abc/algorithm.py:309-334``
* adjoint dUCC gradient (``measure_gradient``)``abc/uccvqeabc.py:122-251``
* ADAPT pool gradients (``measure_gradient3``)``abc/uccvqeabc.py:253-283``

and runs the state-vector arithmetic in ``sv_oracle.c`` (the C restatement of
``computer.cc``).  Parity is pinned: ``tests/test_oracle_pins.py`` checks this
module against golden vectors produced by the compiled reference
(``tests/golden/make_golden.py``) and against the reference's own test values.

A Pauli term is ``(coeff, [(pauli, qubit), ...])`` with the Pauli letters in
circuit order; a gate is ``(target, control, mat4x4)``.
"""

import cmath
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libqfb_oracle.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            subprocess.run(["make", "-s", "-C", _HERE, "port"], check=True)
        lib = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        i32p = ctypes.POINTER(ctypes.c_int32)
        i64p = ctypes.POINTER(ctypes.c_int64)
        lib.ora_apply_gates.argtypes = [dp, ctypes.c_int, ctypes.c_int64, i32p, i32p, dp]
        lib.ora_apply_gate.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        lib.ora_scale.argtypes = [dp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.ora_dot.argtypes = [dp, dp, ctypes.c_int, dp]
        lib.ora_apply_operator.argtypes = [dp, ctypes.c_int, ctypes.c_int64, dp, i64p, i32p,
                                           i32p, dp]
        _lib = lib
    return _lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# --------------------------------------------------------------------------
# gates (make_gate.cc)
# --------------------------------------------------------------------------

ONE_QUBIT = ("X", "Y", "Z", "H", "R", "Rx", "Ry", "Rz", "V", "S", "T", "I")
TWO_QUBIT = ("A", "cX", "CNOT", "acX", "aCNOT", "cY", "cZ", "cR", "cV", "cRz", "SWAP")


def normalize_angle(angle, period):
    """make_gate.cc:7-16 (std::fmod, then fold into [-period/2, period/2])."""
    angle = math.fmod(angle, period)
    if angle < -period / 2:
        angle += period
    elif angle > period / 2:
        angle -= period
    return angle


def make_gate(kind, target, control=None, parameter=0.0):
    """Return (target, control, 4x4 complex matrix) as make_gate.cc:18-235 builds it."""
    if control is None:
        control = target
    m = np.zeros((4, 4), dtype=np.complex128)
    j = 1j
    p = float(parameter)
    if target == control:
        if kind == "X":
            m[0, 1] = m[1, 0] = 1.0
        elif kind == "Y":
            m[0, 1], m[1, 0] = -j, j
        elif kind == "Z":
            m[0, 0], m[1, 1] = 1.0, -1.0
        elif kind == "H":
            c = 1.0 / math.sqrt(2.0)
            m[0, 0] = m[0, 1] = m[1, 0] = c
            m[1, 1] = -c
        elif kind == "R":
            p = normalize_angle(p, 2 * math.pi)
            m[0, 0], m[1, 1] = 1.0, cmath.exp(j * p)
        elif kind == "Rx":
            p = normalize_angle(p, 4 * math.pi)
            a, b = math.cos(0.5 * p), j * math.sin(0.5 * p)
            m[0, 0], m[0, 1], m[1, 0], m[1, 1] = a, -b, -b, a
        elif kind == "Ry":
            p = normalize_angle(p, 4 * math.pi)
            a, b = math.cos(0.5 * p), math.sin(0.5 * p)
            m[0, 0], m[0, 1], m[1, 0], m[1, 1] = a, -b, b, a
        elif kind == "Rz":
            p = normalize_angle(p, 4 * math.pi)
            m[0, 0], m[1, 1] = cmath.exp(-j * 0.5 * p), cmath.exp(j * 0.5 * p)
        elif kind == "V":
            a, b = 0.5 + 0.5j, 0.5 - 0.5j
            m[0, 0], m[0, 1], m[1, 0], m[1, 1] = a, b, b, a
        elif kind == "S":
            m[0, 0], m[1, 1] = 1.0, j
        elif kind == "T":
            m[0, 0], m[1, 1] = 1.0, (1.0 + j) / math.sqrt(2.0)
        elif kind == "I":
            m[0, 0] = m[1, 1] = 1.0
        else:
            raise ValueError(f"make_gate(): type = {kind} is not a valid quantum gate type")
        return (target, control, m)
    m[0, 0] = m[1, 1] = m[2, 2] = m[3, 3] = 1.0
    if kind == "A":
        p = normalize_angle(p, 2 * math.pi)
        c, s = math.cos(p), math.sin(p)
        m[1, 1], m[1, 2], m[2, 1], m[2, 2] = c, s, s, -c
    elif kind in ("cX", "CNOT"):
        m[2, 2] = m[3, 3] = 0.0
        m[2, 3] = m[3, 2] = 1.0
    elif kind in ("acX", "aCNOT"):
        m[0, 0] = m[1, 1] = 0.0
        m[0, 1] = m[1, 0] = 1.0
    elif kind == "cY":
        m[2, 2] = m[3, 3] = 0.0
        m[2, 3], m[3, 2] = -j, j
    elif kind == "cZ":
        m[3, 3] = -1.0
    elif kind == "cR":
        p = normalize_angle(p, 2 * math.pi)
        m[3, 3] = cmath.exp(j * p)
    elif kind == "cV":
        a, b = 0.5 + 0.5j, 0.5 - 0.5j
        m[2, 2], m[2, 3], m[3, 2], m[3, 3] = a, b, b, a
    elif kind == "cRz":
        p = normalize_angle(p, 4 * math.pi)
        m[2, 2], m[3, 3] = cmath.exp(-j * 0.5 * p), cmath.exp(j * 0.5 * p)
    elif kind == "SWAP":
        m[1, 1] = m[2, 2] = 0.0
        m[1, 2] = m[2, 1] = 1.0
    else:
        raise ValueError(f"make_gate(): type = {kind} is not a valid quantum gate type")
    return (target, control, m)


def gate_adjoint(g):
    """Conjugate transpose of the stored matrix (gate.cc:137-147)."""
    t, c, m = g
    return (t, c, m.conj().T.copy())


def circuit_adjoint(gates):
    """Circuit::adjoint (circuit.cc:98-105): adjoint gates in reverse order."""
    return [gate_adjoint(g) for g in reversed(gates)]


def pauli_gates(term):
    """Gate list of a Pauli circuit [(letter, qubit), ...] in circuit order."""
    return [make_gate(p, q, q) for p, q in term]


# --------------------------------------------------------------------------
# exp(c P) and Trotter products (utils/exponentiate.py, utils/trotterization.py)
# --------------------------------------------------------------------------


def exponentiate_pauli_string(coefficient, term):
    """utils/exponentiate.py:9-87 -> (gates, phase)."""
    coefficient = complex(coefficient)
    if abs(coefficient.real) > 1.0e-14:
        raise ValueError(
            f"exponentiate_pauli_string() called with a real coefficient {coefficient}")
    if len(term) == 0:
        return [], cmath.exp(coefficient)
    to_z, cx = [], []
    prev_target = None
    max_target = None
    for pid, target in term:
        if pid == "X":
            to_z.append(make_gate("H", target, target))
        elif pid == "Y":
            to_z.append(make_gate("Rx", target, target, math.pi / 2))
        elif pid == "I":
            continue
        if prev_target is not None:
            cx.append(make_gate("cX", target, prev_target))
        prev_target = target
        max_target = target
    z_rot = make_gate("Rz", max_target, max_target, -2.0 * coefficient.imag)
    gates = to_z + cx + [z_rot] + circuit_adjoint(cx) + circuit_adjoint(to_z)
    return gates, 1.0


def trotterize(terms, factor=1.0):
    """utils/trotterization.py:27-35 (trotter_number = trotter_order = 1)."""
    gates = []
    phase = 1.0
    for coeff, term in terms:
        g, p = exponentiate_pauli_string(factor * complex(coeff), term)
        gates.extend(g)
        phase *= p
    return gates, phase


# --------------------------------------------------------------------------
# the state (computer.cc restated in sv_oracle.c)
# --------------------------------------------------------------------------


def _pack_gates(gates):
    n = len(gates)
    targets = np.array([g[0] for g in gates], dtype=np.int32)
    controls = np.array([g[1] for g in gates], dtype=np.int32)
    mats = np.zeros((max(n, 1), 4, 4), dtype=np.complex128)
    for k, g in enumerate(gates):
        mats[k] = g[2]
    return targets, controls, mats


class State:
    """A complex128 state vector driven by the C restatement of ``Computer``."""

    def __init__(self, nqubit, coeffs=None):
        self.nqubit = int(nqubit)
        if coeffs is None:
            self.psi = np.zeros(1 << self.nqubit, dtype=np.complex128)
            self.psi[0] = 1.0
        else:
            self.psi = np.array(coeffs, dtype=np.complex128).copy()

    def copy(self):
        return State(self.nqubit, self.psi)

    def apply_gates(self, gates):
        if not gates:
            return
        t, c, m = _pack_gates(gates)
        i32p = ctypes.POINTER(ctypes.c_int32)
        _load().ora_apply_gates(_dptr(self.psi), self.nqubit, len(gates),
                                t.ctypes.data_as(i32p), c.ctypes.data_as(i32p), _dptr(m))

    def apply_constant(self, a):
        a = complex(a)
        _load().ora_scale(_dptr(self.psi), self.nqubit, a.real, a.imag)

    def apply_operator(self, terms):
        """``terms``: [(coeff, [gate, ...]), ...] with arbitrary gates per term."""
        coeffs = np.array([complex(c) for c, _ in terms] or [0j], dtype=np.complex128)
        offsets = np.zeros(len(terms) + 1, dtype=np.int64)
        flat = []
        for k, (_, gates) in enumerate(terms):
            flat.extend(gates)
            offsets[k + 1] = len(flat)
        t, c, m = _pack_gates(flat)
        i32p = ctypes.POINTER(ctypes.c_int32)
        _load().ora_apply_operator(_dptr(self.psi), self.nqubit, len(terms), _dptr(coeffs),
                                   offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                   t.ctypes.data_as(i32p), c.ctypes.data_as(i32p), _dptr(m))

    def apply_pauli_operator(self, pterms):
        self.apply_operator([(c, pauli_gates(t)) for c, t in pterms])

    def dot(self, other):
        """<self|other> (computer.cc:975-980)."""
        out = np.zeros(2)
        _load().ora_dot(_dptr(self.psi), _dptr(other.psi), self.nqubit, _dptr(out))
        return complex(out[0], out[1])

    def direct_op_exp_val(self, pterms):
        """Serial direct_op_exp_val (computer.cc:753-771): <psi| apply_operator(H) psi>."""
        sig = self.copy()
        sig.apply_pauli_operator(pterms)
        return self.dot(sig)


# --------------------------------------------------------------------------
# algorithm drivers (abc/algorithm.py, abc/uccvqeabc.py)
# --------------------------------------------------------------------------


def sample_indices(psi, seed, nshots):
    """Seeded sampling of basis indices from |c_i|^2, the CPU restatement of
    the device sampler (the draws of Computer::measure_circuit,
    computer.cc:135-315, whose own generator is unseeded): weights
    trunc(|c|^2 2^56), exact integer prefix sums, SplitMix64 draw u_k of the
    seed, r_k = floor(u_k T / 2^64), sample = first index whose inclusive
    prefix exceeds r_k."""
    psi = np.asarray(psi, dtype=np.complex128)
    p = psi.real * psi.real + psi.imag * psi.imag
    w = (p * 2.0 ** 56).astype(np.uint64)
    cum = np.cumsum(w, dtype=np.uint64)
    T = int(cum[-1])
    M = (1 << 64) - 1
    r = np.empty(nshots, dtype=np.uint64)
    for k in range(nshots):
        z = (int(seed) + (k + 1) * 0x9E3779B97F4A7C15) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        z ^= z >> 31
        r[k] = (z * T) >> 64
    return np.searchsorted(cum, r, side="right").astype(np.uint64)


def refprep(ref):
    """utils/state_prep.py:5-11: X on every occupied spin-orbital."""
    return [make_gate("X", j, j) for j, occ in enumerate(ref) if occ]


def ansatz_terms(kops, amps, drop_tol=1.0e-12):
    """Terms of A = sum_mu t_mu K_mu in pool order (sq_op_pool.cc:97-104).

    ``kops[mu]`` is the ordered term list of K_mu (already simplified and
    ordered as ``get_qubit_operator('commuting_grp_lex')`` leaves it);
    ``simplify`` drops products with |t c| <= 1e-12 (qubit_operator.cc:166-171).
    """
    out = []
    for t, K in zip(amps, kops):
        for c, term in K:
            v = complex(c) * t
            if abs(v) > drop_tol:
                out.append((v, term))
    return out


def prepare_state(nqubit, ref, kops, amps):
    """Uprep then U(t) (abc/algorithm.py:271-288, abc/ansatz.py:73-82)."""
    st = State(nqubit)
    st.apply_gates(refprep(ref))
    gates, phase = trotterize(ansatz_terms(kops, amps))
    if phase != 1.0:
        raise ValueError("Encountered phase change")
    st.apply_gates(gates)
    return st


def energy(nqubit, ref, kops, amps, hterms):
    """measure_energy (abc/algorithm.py:309-334), fast path."""
    st = prepare_state(nqubit, ref, kops, amps)
    return st.direct_op_exp_val(hterms).real, st


def measure_gradient(nqubit, ref, kops, amps, hterms, kops_grad=None, kops_unrot=None):
    """Adjoint dUCC gradient, abc/uccvqeabc.py:122-251 (non-compact, trotter_number 1).

    ``kops_grad[mu]`` is K_mu as ``jw_transform`` returns it times the pool
    coefficient (term order of the gradient loop); defaults to ``kops``.
    ``kops_unrot[mu]`` are the strings whose Trotter product un-applies U_mu:
    K_mu itself for particle-hole pools (:228-230, the default), the ansatz's
    component excitations for spin-adapted pools (:208-224).
    """
    kg = kops if kops_grad is None else kops_grad
    ku = kg if kops_unrot is None else kops_unrot
    M = len(amps)
    grads = np.zeros(M)
    psi = prepare_state(nqubit, ref, kops, amps)
    sig = psi.copy()
    sig.apply_pauli_operator(hterms)
    tmp = psi.copy()
    tmp.apply_pauli_operator(kg[M - 1])
    grads[M - 1] = 2.0 * sig.dot(tmp).real
    for mu in reversed(range(M - 1)):
        umu, pmu = trotterize(ku[mu + 1], factor=-amps[mu + 1])
        sig.apply_gates(umu)
        psi.apply_gates(umu)
        tmp = psi.copy()
        tmp.apply_pauli_operator(kg[mu])
        grads[mu] = 2.0 * sig.dot(tmp).real
    return grads


def pqe_residuals(nqubit, ref, kops, amps, hterms, excited_dets):
    """UCCNPQE.get_residual_vector (ucc/uccnpqe.py:249-292): Uprep, U(t), H,
    U(t)^dagger (the adjoint circuit), then coeff[I] * phase for each excited
    determinant (I, phase)."""
    st = State(nqubit)
    st.apply_gates(refprep(ref))
    gates, phase = trotterize(ansatz_terms(kops, amps))
    if phase != 1.0:
        raise ValueError("Encountered phase change")
    st.apply_gates(gates)
    st.apply_pauli_operator(hterms)
    st.apply_gates(circuit_adjoint(gates))
    out = []
    for I, ph in excited_dets:
        r = st.psi[int(I)] * ph
        if abs(r.imag) > 1.0e-12:
            raise ValueError("residual has imaginary component")
        out.append(r.real)
    return np.array(out)


def measure_gradient3(nqubit, ref, kops, amps, hterms, pool_kops):
    """ADAPT pool gradients 2 Re <H psi| K_mu psi>, abc/uccvqeabc.py:253-283."""
    psi = prepare_state(nqubit, ref, kops, amps)
    sig = psi.copy()
    sig.apply_pauli_operator(hterms)
    out = np.zeros(len(pool_kops))
    for mu, K in enumerate(pool_kops):
        tmp = psi.copy()
        tmp.apply_pauli_operator(K)
        out[mu] = 2.0 * sig.dot(tmp).real
    return out


# --------------------------------------------------------------------------
# the compiled reference, importable in the build container only
# --------------------------------------------------------------------------


# The reference's Python sources: $QFORTE_REF_SRC, else the build container's copy.
REF_SRC_DEFAULT = os.environ.get("QFORTE_REF_SRC", "/root/reference/src/qforte")


def load_reference(ref_src=REF_SRC_DEFAULT):
    """Import the reference package with its compiled module from oracle/_ref.

    The package's Python sources are used where they lie; its extension
    module ``qforte.qforte`` is the one ``make -C oracle ref`` built (searched
    first: the sources hold a placeholder ``qforte.py`` of the same name).  Returns
    the package, or raises ImportError when either part is missing.
    """
    import importlib.util
    import sys

    if "qforte" in sys.modules and hasattr(sys.modules["qforte"], "Computer"):
        return sys.modules["qforte"]
    ext_dir = os.path.join(_HERE, "_ref", "qforte")
    init = os.path.join(ref_src, "__init__.py")
    if not (os.path.isdir(ext_dir) and os.path.exists(init)):
        raise ImportError("reference sources or compiled module not present")
    spec = importlib.util.spec_from_file_location(
        "qforte", init, submodule_search_locations=[ext_dir, ref_src])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qforte"] = mod
    try:
        spec.loader.exec_module(mod)
    except Exception:
        del sys.modules["qforte"]
        raise
    return mod


def load_reference_engine():
    """Import only the compiled engine module (works without the Python sources)."""
    import importlib.util
    import glob
    import sys

    if "qforte" in sys.modules and hasattr(sys.modules["qforte"], "Computer"):
        return sys.modules["qforte"]
    hits = glob.glob(os.path.join(_HERE, "_ref", "qforte", "qforte*.so"))
    if not hits:
        raise ImportError("oracle/_ref/qforte/qforte*.so not built")
    spec = importlib.util.spec_from_file_location("qforte", hits[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules["qforte"] = mod
    return mod


# --------------------------------------------------------------------------
# timing the compiled reference on a bounded sample (bench.py's CPU legs)
# --------------------------------------------------------------------------


def ref_pauli_circuit(qf, term):
    c = qf.Circuit()
    for l, q in term:
        c.add(qf.gate(l, q, q))
    return c


def ref_operator(qf, terms):
    op = qf.QubitOperator()
    for c, term in terms:
        op.add(complex(c), ref_pauli_circuit(qf, term))
    return op


def ref_exponential(qf, coefficient, term):
    """utils/exponentiate.py:9-87 with the reference's own gate factory."""
    coefficient = complex(coefficient)
    to_z, cx = qf.Circuit(), qf.Circuit()
    prev, mx = None, None
    for l, q in term:
        if l == "X":
            to_z.add(qf.gate("H", q, q))
        elif l == "Y":
            to_z.add(qf.gate("Rx", q, q, math.pi / 2))
        if prev is not None:
            cx.add(qf.gate("cX", q, prev))
        prev = mx = q
    out = qf.Circuit()
    out.add(to_z)
    out.add(cx)
    out.add(qf.gate("Rz", mx, mx, -2.0 * coefficient.imag))
    out.add(cx.adjoint())
    out.add(to_z.adjoint())
    return out


def ref_trotter(qf, terms, factor=1.0):
    circ = qf.Circuit()
    for c, term in terms:
        circ.add(ref_exponential(qf, factor * complex(c), term))
    return circ


def ref_pqe_sample(qf, nqubit, ref, kops_fwd, amps, hterms, h_sample):
    """Time one UCCNPQE.get_residual_vector of the compiled reference
    (uccnpqe.py:249-292) on a bounded sample: refprep and U(t) as gates, then
    apply_operator on ``h_sample`` of the H terms scaled to all of them, then
    U(t)^dagger as gates and the coefficient read-back.  Returns seconds per
    residual vector."""
    import time

    t0 = time.perf_counter()
    qc = qf.Computer(nqubit)
    prep = qf.Circuit()
    for j, occ in enumerate(ref):
        if occ:
            prep.add(qf.gate("X", j, j))
    qc.apply_circuit(prep)
    U = ref_trotter(qf, ansatz_terms(kops_fwd, amps))
    qc.apply_circuit(U)
    t_u = time.perf_counter() - t0
    hs = ref_operator(qf, hterms[:h_sample])
    t0 = time.perf_counter()
    qc.apply_operator(hs)
    t_h = (time.perf_counter() - t0) * len(hterms) / max(1, min(h_sample, len(hterms)))
    t0 = time.perf_counter()
    qc.apply_circuit(U.adjoint())
    qc.get_coeff_vec()
    t_ud = time.perf_counter() - t0
    return t_u + t_h + t_ud, {"t_U": t_u, "t_H": t_h, "t_Udagger": t_ud}


def ref_eval_sample(qf, nqubit, ref, kops_fwd, kops_grad, amps, hterms, h_sample, m_sample):
    """Time one dUCC energy + adjoint gradient of the compiled reference on a
    bounded sample and return the per-evaluation seconds it implies.

    Timed exactly as the reference's drivers run (serial build):
      t_U      refprep + U(t) as gates on a fresh Computer   (measure_energy)
      t_H      apply_operator on ``h_sample`` of the H terms, scaled to all of
               them; an evaluation applies H twice (direct_op_exp_val, sigma)
      t_sweep  ``m_sample`` reverse-sweep steps of measure_gradient (un-apply
               U_mu from sigma and psi, copy, apply_operator(K_mu), two
               get_coeff_vec + vdot), scaled to all parameters
    """
    import time

    M = len(amps)
    t0 = time.perf_counter()
    qc = qf.Computer(nqubit)
    prep = qf.Circuit()
    for j, occ in enumerate(ref):
        if occ:
            prep.add(qf.gate("X", j, j))
    qc.apply_circuit(prep)
    qc.apply_circuit(ref_trotter(qf, ansatz_terms(kops_fwd, amps)))
    t_u = time.perf_counter() - t0
    hs = ref_operator(qf, hterms[:h_sample])
    t0 = time.perf_counter()
    sig = qf.Computer(qc)
    sig.apply_operator(hs)
    t_h = (time.perf_counter() - t0) * len(hterms) / max(1, min(h_sample, len(hterms)))
    ks = [ref_operator(qf, k) for k in kops_grad]
    m_s = max(1, min(m_sample, M - 1))
    t0 = time.perf_counter()
    for mu in range(M - 2, M - 2 - m_s, -1):
        umu = ref_trotter(qf, kops_grad[mu + 1], -amps[mu + 1])
        sig.apply_circuit(umu)
        qc.apply_circuit(umu)
        tmp = qf.Computer(qc)
        tmp.apply_operator(ks[mu])
        np.vdot(sig.get_coeff_vec(), tmp.get_coeff_vec())
    t_sweep = (time.perf_counter() - t0) * M / m_s
    return t_u + 2.0 * t_h + t_sweep, {"t_U": t_u, "t_H": t_h, "t_sweep": t_sweep}


def _ref_eval_worker(args):
    """One spawned worker of ref_eval_parallel: imports the compiled reference
    itself and times one sample evaluation."""
    nqubit, ref, kops_fwd, kops_grad, amps, hterms, h_sample, m_sample = args
    qf = load_reference_engine()
    return ref_eval_sample(qf, nqubit, ref, kops_fwd, kops_grad, amps, hterms, h_sample,
                           m_sample)


def host_cores():
    """The host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def ref_eval_parallel(nqubit, ref, kops_fwd, kops_grad, rows, hterms, h_sample, m_sample,
                      workers):
    """ref_eval_sample on ``workers`` host cores at once: the evaluations of a
    batch are independent, so the shipped serial build runs one per core, in
    processes started with ``spawn`` (safe after CUDA was initialised in the
    parent).  Worker w evaluates ``rows[w % len(rows)]``.  Returns (evaluations
    per second of all workers together, per-worker seconds per evaluation,
    wall seconds of the sample, per-worker parts)."""
    import multiprocessing as mp
    import time

    args = [(nqubit, list(ref), kops_fwd, kops_grad, list(map(float, rows[w % len(rows)])),
             hterms, h_sample, m_sample) for w in range(workers)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        out = pool.map(_ref_eval_worker, args, chunksize=1)
    wall = time.perf_counter() - t0
    per = [t for t, _ in out]
    return sum(1.0 / t for t in per), per, wall, [p for _, p in out]


def ref_gate_sample(qf, nqubit, spec, ngates):
    """Seconds per gate of the compiled reference's Computer.apply_circuit
    (computer.cc:93-114) on the first ``ngates`` gates of ``spec`` [(kind,
    target, control, parameter)], from |0...0> (the first gates of the sweep
    act on a fresh state, as in the reference's own use)."""
    import time

    circ = qf.Circuit()
    for k, t, c, p in spec[:ngates]:
        circ.add(qf.gate(k, int(t), int(c), float(p)))
    qc = qf.Computer(nqubit)
    t0 = time.perf_counter()
    qc.apply_circuit(circ)
    return (time.perf_counter() - t0) / ngates
