"""Quantum imaginary time evolution (QITE) and its Lanczos step on the device state.

Follows ``ite/qite.py``: ``QITE.run`` (:125-174), ``build_expansion_pool``
(:214-254), ``build_S`` (:256-276), ``build_sparse_S_b`` (:278-303),
``build_b`` (:305-326), ``do_qite_step`` (:328-373), ``evolve`` (:375-437) and
``do_qlanczos`` (:444-491), with ``maths/eigsolve.py:canonical_geig_solve``.

The reference forms b and S from a Computer copy, one ``apply_operator`` and one
host readback of the whole state per expansion operator, then vdots on the host.
Here the state stays in HBM and both come from segmented expectation values
(``qfb_sum_expval``): each (segment, x-mask) group reads the state once for all
of its terms, and the only data crossing to the host are the results.

* b_I = Re(-i c_I / sqrt(1 - 2 db E) <psi| sigma_I H |psi>): H psi is formed
  once (``qfb_sum_apply``), then <psi| P |H psi> for every distinct Pauli
  string P of the operators, one result segment each, with bra psi and ket
  H psi.
* S_IJ = Re <sigma_I psi | sigma_J psi> = Re <psi| sigma_I^dag sigma_J |psi>:
  a product of two Pauli strings is one Pauli string times a power of i
  (``pauli_mul``, exact), so S needs <psi| P |psi> once per distinct product
  string, and each pair I < J combines them with its coefficients on the
  host.  S_II = 1 as in the reference (a Pauli string squares to one).

The evolution step exp(A), A = -i db sum_I x_I sigma_I, is trotterized as in the
reference and applied through ``Computer.apply_circuit``, which runs Pauli
exponentials as fused streaming passes.  Lanczos vectors stay on the device as
state copies; their overlaps are device inner products.
"""

import numpy as np
from scipy import linalg

from ._lib import check, lib, ptr
from .circuit import Circuit
from .computer import Computer, inner_product
from .device import sum_from_terms
from .gate import gate
from .pauli import ipow_mul, pauli_mul
from .qubit_operator import QubitOperator
from .sq_op_pool import QubitOpPool, SQOpPool
from .utils import build_refprep, trotterize

__all__ = ["QITE", "canonical_geig_solve", "qite_b", "qite_S"]


# qfb_sum_expval takes at most 65,535 (segment, x-mask) groups per call; a
# call never holds more terms than that, so never more groups
_MAX_TERMS_PER_CALL = 65535


def _segment_runs(segments, limit=_MAX_TERMS_PER_CALL):
    """Split term indices [0, n) into runs [lo, hi) of at most ``limit`` terms
    that end on segment boundaries (``segments`` non-decreasing)."""
    n = len(segments)
    runs = []
    lo = 0
    while lo < n:
        hi = min(n, lo + limit)
        if hi < n:
            while hi > lo and segments[hi] == segments[hi - 1]:
                hi -= 1
            if hi == lo:
                raise ValueError(f"one QITE matrix element has more than {limit} terms")
        runs.append((lo, hi))
        lo = hi
    return runs


def _segment_expvals(bra, ket, terms, segments, nsegment, limit=_MAX_TERMS_PER_CALL):
    """out[g] = sum over the terms of segment g of c <bra| P(x, z) |ket> on the
    device (qfb_sum_expval), one call per run of whole segments of at most
    ``limit`` terms."""
    out = np.zeros(nsegment, dtype=np.complex128)
    for lo, hi in _segment_runs(segments, limit):
        s0 = segments[lo]
        ns = segments[hi - 1] - s0 + 1
        ds = sum_from_terms(terms[lo:hi], [g - s0 for g in segments[lo:hi]], ns)
        bra._check_qubits(ds.maxbit)
        part = np.zeros(ns, dtype=np.complex128)
        check(lib().qfb_sum_expval(ds.h, bra._h, ket._h, ptr(part)), "QITE expectation values")
        out[s0:s0 + ns] = part
    return out


def _op_terms(qo):
    """[(c, x, z)] of the operator apply_operator applies; every QITE expansion
    operator is a Pauli string with a coefficient."""
    pt = qo._pauli_terms(applied=True)
    if pt is None:
        raise ValueError("QITE expansion operators must be Pauli strings")
    return pt


def _distinct_string_expvals(bra, ket, strings):
    """<bra| P(x, z) |ket> for every distinct (x, z) of ``strings``, one
    result segment each: returns ({(x, z): value})."""
    keys = list(dict.fromkeys(strings))
    vals = _segment_expvals(bra, ket, [(1.0, x, z) for x, z in keys], list(range(len(keys))),
                            len(keys))
    return dict(zip(keys, vals))


def qite_b(qc, hamiltonian, sig_ops, sig_coeffs, db, energy):
    """build_b (ite/qite.py:305-326): b_I = Re(-i c_I <psi| sigma_I H |psi>) /
    sqrt(1 - 2 db E).  H psi is formed once; <psi| P |H psi> is read once per
    distinct Pauli string P among the operators' terms."""
    prefactor = -1.0j / np.sqrt(1 - 2 * db * energy)
    hpsi = Computer(qc)
    hpsi.apply_operator(hamiltonian)
    ops = [_op_terms(op) for op in sig_ops]
    ev = _distinct_string_expvals(qc, hpsi, [(x, z) for pt in ops for _, x, z in pt])
    vals = np.array([sum(complex(c) * ev[(x, z)] for c, x, z in pt) for pt in ops],
                    dtype=np.complex128)
    b = prefactor * np.asarray(sig_coeffs, dtype=np.complex128) * vals
    return np.real(b)


def qite_S(qc, sig_ops):
    """build_S (ite/qite.py:256-276) over the given operators: S_II = 1 and
    S_IJ = S_JI = Re <sigma_I psi | sigma_J psi> for I != J.  Each product of
    two terms' Pauli strings is one string times a power of i, so
    <sigma_I psi | sigma_J psi> = sum_ab conj(c_a) c_b i^e <psi| P_ab |psi>,
    and <psi| P |psi> is read once per distinct product string P (for
    single-string operators on n qubits: at most 4^n reads, not NI^2 / 2)."""
    n = len(sig_ops)
    S = np.eye(n)
    if n < 2:
        return S
    ops = [_op_terms(op) for op in sig_ops]
    # (i, j) -> [(coefficient, (x, z))] of sigma_i^dag sigma_j
    prods = {}
    for i in range(n):
        for j in range(i):
            lst = []
            for ca, xa, za in ops[i]:
                ca = complex(ca).conjugate()
                for cb, xb, zb in ops[j]:
                    x, z, e = pauli_mul(xa, za, xb, zb)
                    lst.append((ipow_mul(ca * complex(cb), e), (x, z)))
            prods[(i, j)] = lst
    ev = _distinct_string_expvals(qc, qc, [k for lst in prods.values() for _, k in lst])
    for (i, j), lst in prods.items():
        S[i, j] = S[j, i] = np.real(sum(c * ev[k] for c, k in lst))
    return S


def _sorted_idxs(values):
    """Indices of ``values`` by increasing real part, ties in input order
    (helper/idx_org.py:sorted_largest_idxs with use_real=True, rev=False)."""
    return sorted(range(len(values)), key=lambda i: np.real(values[i]))


def canonical_geig_solve(S, H, print_mats=False, sort_ret_vals=False):
    """Generalised eigenproblem H C = S C e by canonical orthogonalisation
    (maths/eigsolve.py:canonical_geig_solve): eigenvalues of S at or below
    1e-15 are dropped, the first columns of S's eigenvectors are scaled by the
    kept eigenvalues' inverse square roots, exactly as the reference pairs them."""
    threshold = 1e-15
    s, U = linalg.eig(S)
    s_prime = []
    for sii in s:
        if np.imag(sii) > 1e-12:
            raise ValueError("S may not be hermetian, large imag. eval component.")
        if np.real(sii) > threshold:
            s_prime.append(np.real(sii))
    X_prime = np.zeros((len(s), len(s_prime)), dtype=complex)
    for j in range(len(s_prime)):
        X_prime[:, j] = U[:, j] / np.sqrt(s_prime[j])
    H_prime = X_prime.conj().T.dot(H).dot(X_prime)
    e_prime, C_prime = linalg.eig(H_prime)
    if not sort_ret_vals:
        return e_prime, X_prime.dot(C_prime)
    order = _sorted_idxs(e_prime)
    sorted_e = np.array([e_prime[k] for k in order], dtype=complex)
    sorted_C = C_prime[:, order]
    sorted_X = X_prime[:, order]
    return sorted_e, sorted_X.dot(sorted_C)


class QITE:
    """QITE on the drop-in Computer (ite/qite.py:24-491).

    ``system`` supplies ``hamiltonian`` (a QubitOperator) and ``hf_reference``
    unless ``reference`` is given.  ``run`` takes the reference's arguments and
    leaves the same attributes: ``_Ekb`` (energy per step), ``_Egs``,
    ``_Egs_lanczos`` (with ``do_lanczos``), ``_NI``, ``_n_classical_params``,
    ``_n_cnot`` and ``_n_pauli_trm_measures``.
    """

    def __init__(self, system, reference=None, trotter_number=1, verbose=False):
        self._sys = system
        self._ref = list(system.hf_reference if reference is None else reference)
        self._nqb = len(self._ref)
        self._qb_ham = system.hamiltonian
        self._trotter_number = trotter_number
        self._verbose = verbose
        self._Uprep = Circuit(build_refprep(self._ref))

    def run(self, beta=1.0, db=0.2, expansion_type="SD", sparseSb=True, b_thresh=1.0e-6,
            x_thresh=1.0e-10, do_lanczos=False, lanczos_gap=2):
        self._beta = beta
        self._db = db
        self._nbeta = int(beta / db) + 1
        self._expansion_type = expansion_type
        self._sparseSb = sparseSb
        self._total_phase = 1.0 + 0.0j
        self._Uqite = Circuit()
        self._b_thresh = b_thresh
        self._x_thresh = x_thresh
        self._n_classical_params = 0
        self._n_cnot = self._Uprep.get_num_cnots()
        self._n_pauli_trm_measures = 0
        self._do_lanczos = do_lanczos
        self._lanczos_gap = lanczos_gap

        qc_ref = Computer(self._nqb)
        qc_ref.apply_circuit(self._Uprep)
        self._Ekb = [np.real(qc_ref.direct_op_exp_val(self._qb_ham))]

        self.build_expansion_pool()
        self.evolve()
        if self._do_lanczos:
            self.do_qlanczos()
        return self._Egs

    def get_gs_energy(self):
        return self._Egs

    # ---- the expansion operators (ite/qite.py:214-254) ------------------------
    def build_expansion_pool(self):
        self._sig = QubitOpPool()
        if self._expansion_type == "complete_qubit":
            if self._nqb > 6:
                raise ValueError("Using complete qubits expansion will result in a very "
                                 "large number of terms!")
            self._sig.fill_pool("complete_qubit", self._nqb)
        elif self._expansion_type == "cqoy":
            self._sig.fill_pool("cqoy", self._nqb)
        elif self._expansion_type in {"SD", "GSD", "SDT", "SDTQ", "SDTQP", "SDTQPH"}:
            P = SQOpPool()
            P.set_orb_spaces(self._ref)
            P.fill_pool(self._expansion_type)
            sig_temp = P.get_qubit_operator("commuting_grp_lex", False)
            # only strings with an odd number of Y survive (real H and states:
            # the other b elements are imaginary and vanish); coefficients are
            # dropped, every operator enters with 1
            for _, rho in sig_temp.terms():
                temp_rho = Circuit()
                nygates = 0
                for g in rho.gates():
                    temp_rho.add(gate(g.gate_id(), g.target(), g.control()))
                    if g.gate_id() == "Y":
                        nygates += 1
                if nygates % 2 == 1:
                    rho_op = QubitOperator()
                    rho_op.add(1.0, temp_rho)
                    self._sig.add(1.0, rho_op)
        else:
            raise ValueError("Invalid expansion type specified.")
        self._NI = len(self._sig.terms())

    # ---- one imaginary-time step (ite/qite.py:256-373) -------------------------
    def build_b(self):
        self._n_pauli_trm_measures += len(self._qb_ham.terms()) * self._NI
        terms = self._sig.terms()
        return qite_b(self._qc, self._qb_ham, [op for _, op in terms], [c for c, _ in terms],
                      self._db, self._Ekb[-1])

    def build_S(self):
        self._n_pauli_trm_measures += int(self._NI * (self._NI + 1) * 0.5)
        return qite_S(self._qc, [op for _, op in self._sig.terms()])

    def build_sparse_S_b(self, b):
        idx_sparse = [i for i, bi in enumerate(b) if np.abs(bi) > self._b_thresh]
        b_sparse = [b[i] for i in idx_sparse]
        n = len(idx_sparse)
        self._n_pauli_trm_measures += int(n * (n + 1) * 0.5)
        terms = self._sig.terms()
        S = qite_S(self._qc, [terms[i][1] for i in idx_sparse])
        return idx_sparse, S, np.real(b_sparse)

    def do_qite_step(self):
        btot = self.build_b()
        A = QubitOperator()
        if self._sparseSb:
            sp_idxs, S, btot = self.build_sparse_S_b(btot)
        else:
            S = self.build_S()
            sp_idxs = list(range(self._NI))
        x = np.real(linalg.lstsq(S, btot)[0]) if len(btot) else np.zeros(0)
        terms = self._sig.terms()
        for i, spi in enumerate(sp_idxs):
            if np.abs(x[i]) > self._x_thresh:
                A.add(-1.0j * self._db * x[i], terms[spi][1].terms()[0][1])
                self._n_classical_params += 1
        eiA_kb, phase1 = trotterize(A, trotter_number=self._trotter_number)
        self._total_phase *= phase1
        self._Uqite.add(eiA_kb)
        self._qc.apply_circuit(eiA_kb)
        self._Ekb.append(np.real(self._qc.direct_op_exp_val(self._qb_ham)))
        self._n_cnot += eiA_kb.get_num_cnots()

    def _lanczos_push(self):
        self._lanczos_vecs.append(Computer(self._qc))
        h = Computer(self._qc)
        h.apply_operator(self._qb_ham)
        self._Hlanczos_vecs.append(h)

    def evolve(self):
        self._Uqite.add(self._Uprep)
        self._qc = Computer(self._nqb)
        self._qc.apply_circuit(self._Uqite)
        if self._do_lanczos:
            self._lanczos_vecs, self._Hlanczos_vecs = [], []
            self._lanczos_push()
        if self._verbose:
            print(f"{'beta':>7}{'E(beta)':>18}{'N(params)':>14}{'N(CNOT)':>18}{'N(measure)':>20}")
            print(f" {0.0:7.3f}    {self._Ekb[0]:+15.9f}    {self._n_classical_params:8}"
                  f"        {self._n_cnot:10}        {self._n_pauli_trm_measures:12}")
        for kb in range(1, self._nbeta):
            self.do_qite_step()
            if self._do_lanczos and kb % self._lanczos_gap == 0:
                self._lanczos_push()
            if self._verbose:
                print(f" {kb * self._db:7.3f}    {self._Ekb[kb]:+15.9f}    "
                      f"{self._n_classical_params:8}        {self._n_cnot:10}        "
                      f"{self._n_pauli_trm_measures:12}")
        self._Egs = self._Ekb[-1]

    # ---- quantum Lanczos over the stored states (ite/qite.py:444-491) ---------
    def do_qlanczos(self):
        n = len(self._lanczos_vecs)
        h_mat = np.zeros((n, n), dtype=complex)
        s_mat = np.zeros((n, n), dtype=complex)
        self._lanczos_energies = []
        for m in range(n):
            for k in range(m + 1):
                h_mat[m][k] = inner_product(self._lanczos_vecs[m], self._Hlanczos_vecs[k])
                h_mat[k][m] = np.conj(h_mat[m][k])
                s_mat[m][k] = inner_product(self._lanczos_vecs[m], self._lanczos_vecs[k])
                s_mat[k][m] = np.conj(s_mat[m][k])
            evals, _ = canonical_geig_solve(s_mat[:m + 1, :m + 1], h_mat[:m + 1, :m + 1],
                                            sort_ret_vals=True)
            self._lanczos_energies.append(np.real(evals[0]))
        self._Egs_lanczos = evals[0]
