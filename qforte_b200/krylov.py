"""Single-reference quantum Krylov diagonalisation (SRQK, NTSRQK) on the device state.

Follows ``qkd/srqk.py``: ``SRQK.run`` (:46-61) and ``build_qk_mats_fast``
(:103-204); ``qkd/nt_srqk.py`` (``NTSRQK``: the basis from exact time
evolution, ``utils/exp_ops.py``); and the generalised eigenproblem of
``abc/qsdabc.py:common_run`` (:87-115).

The Krylov basis is omega_m = U_m |Phi>, U_m the reference's circuit for
exp(-i m dt H) (``trotterize`` with the run's Trotter number, then the global
phase it returns), built afresh for every m exactly as the reference builds it,
so the Trotter error is the reference's.  The reference copies each omega_m and
H omega_m to the host and takes vdots there; here both stay in HBM as states
(the Trotter circuits run as fused Pauli-exponential passes, H omega_m by
``qfb_sum_apply``) and S_mn = <omega_m|omega_n>, H_mn = <omega_m|H|omega_n> are
device inner products (``qfb_vdot``): only the (s+1)^2 matrix elements reach
the host.
"""

import math

import numpy as np

from ._lib import check, cplx, lib
from .circuit import Circuit
from .computer import Computer, inner_product
from .qite import canonical_geig_solve
from .utils import build_refprep, trotterize

__all__ = ["SRQK", "NTSRQK", "evolve_exact", "fill_krylov_row"]


def _axpy(dst, a, src):
    """dst += a * src on the device (qfb_axpy)."""
    check(lib().qfb_axpy(dst._h, cplx(a), src._h), "axpy")


def _norm1(hamiltonian):
    """Sum of |c| over the terms: a bound on the spectral norm of H."""
    return sum(abs(complex(c)) for c, _ in hamiltonian.terms())


def evolve_exact(qc, hamiltonian, t, max_order=60):
    """A new Computer holding exp(-i t H) psi (psi = qc's state, left as it
    is), by a scaled Taylor series on the device: t is cut into substeps with
    |t| sum|c| / nsub <= 1/2, and in each substep the terms (-i h H)^k / k! psi
    (one qfb_sum_apply each) are added until two in a row fall below 2^-53 of
    the sum's norm.  Stands in for scipy's expm_multiply on the sparse matrix
    of H (utils/exp_ops.py:30-33)."""
    out = Computer(qc)
    if t == 0.0:
        return out
    nsub = max(1, math.ceil(abs(t) * _norm1(hamiltonian) / 0.5))
    h = t / nsub
    eps = 2.0 ** -53
    for _ in range(nsub):
        term = Computer(out)
        small = 0
        for k in range(1, max_order + 1):
            term.apply_operator(hamiltonian)
            term.apply_constant(-1.0j * h / k)
            _axpy(out, 1.0, term)
            tn = abs(inner_product(term, term)) ** 0.5
            an = abs(inner_product(out, out)) ** 0.5
            small = small + 1 if tn <= eps * an else 0
            if small == 2:
                break
        else:
            raise RuntimeError("evolve_exact: Taylor series did not converge")
    return out


def fill_krylov_row(S, H, states, hstates, m):
    """Row m of S_mn = <omega_m|omega_n> and H_mn = <omega_m|H omega_n> for
    n <= m, the mirror elements by conjugation (qkd/srqk.py:160-165)."""
    for k in range(m + 1):
        H[m][k] = inner_product(states[m], hstates[k])
        H[k][m] = np.conj(H[m][k])
        S[m][k] = inner_product(states[m], states[k])
        S[k][m] = np.conj(S[m][k])


class SRQK:
    """SRQK on the drop-in Computer (qkd/srqk.py:22-204).

    ``system`` supplies ``hamiltonian`` (a QubitOperator) and ``hf_reference``
    unless ``reference`` is given.  ``run`` leaves the reference's attributes:
    ``_S``, ``_Hbar``, ``_Scond``, ``_eigenvalues``, ``_eigenvectors``,
    ``_Egs``, ``_Ets``, ``_n_classical_params``, ``_n_cnot`` and
    ``_n_pauli_trm_measures``.
    """

    def __init__(self, system, reference=None, trotter_number=1, verbose=False):
        self._sys = system
        self._ref = list(system.hf_reference if reference is None else reference)
        self._nqb = len(self._ref)
        self._qb_ham = system.hamiltonian
        self._Nl = len(self._qb_ham.terms())
        self._trotter_number = trotter_number
        self._verbose = verbose
        self._Uprep = Circuit(build_refprep(self._ref))

    def run(self, s=3, dt=0.5, target_root=0, diagonalize_each_step=True):
        self._s = s
        self._nstates = s + 1
        self._dt = dt
        self._target_root = target_root
        self._diagonalize_each_step = diagonalize_each_step
        self._n_classical_params = 0
        self._n_cnot = 0
        self._n_pauli_trm_measures = 0
        self.common_run()
        return self._Egs

    def get_gs_energy(self):
        return self._Egs

    def get_ts_energy(self):
        return self._Ets

    def get_qk_eigenvalues(self):
        return self._eigenvalues

    def get_qk_eigenvectors(self):
        return self._eigenvectors

    def build_qk_mats(self):
        """build_qk_mats_fast (qkd/srqk.py:103-204): the basis states and H on
        them stay on the device; returns (S, H)."""
        self._omega_lst, homega = [], []
        self._step_energies = []
        S = np.zeros((self._nstates, self._nstates), dtype=complex)
        H = np.zeros((self._nstates, self._nstates), dtype=complex)
        for m in range(self._nstates):
            Um = Circuit(self._Uprep)
            phase1 = 1.0
            if m > 0:
                fact = (0.0 - 1.0j) * m * self._dt
                expn_op1, phase1 = trotterize(self._qb_ham, factor=fact,
                                              trotter_number=self._trotter_number)
                Um.add(expn_op1)
            qc = Computer(self._nqb)
            qc.apply_circuit(Um)
            qc.apply_constant(phase1)
            self._omega_lst.append(qc)
            hq = Computer(qc)
            hq.apply_operator(self._qb_ham)
            homega.append(hq)
            fill_krylov_row(S, H, self._omega_lst, homega, m)
            if self._diagonalize_each_step:
                k = m + 1
                evals, _ = canonical_geig_solve(S[:k, :k], H[:k, :k], sort_ret_vals=True)
                self._step_energies.append(np.real(evals[min(self._target_root, k - 1)]))
                if self._verbose:
                    print(f" {np.linalg.cond(S[:k, :k]):7.2e}    {self._step_energies[-1]:+15.9f}")
        self._n_classical_params = self._nstates
        self._n_cnot = 2 * Um.get_num_cnots()
        # the Hadamard-test measurements the reference counts (qkd/srqk.py:196-202)
        self._n_pauli_trm_measures = self._nstates * self._Nl
        self._n_pauli_trm_measures += self._nstates * (self._nstates - 1) * self._Nl
        self._n_pauli_trm_measures += self._nstates * (self._nstates - 1)
        return S, H

    def common_run(self):
        """abc/qsdabc.py:87-115."""
        self._S, self._Hbar = self.build_qk_mats()
        self._Scond = np.linalg.cond(self._S)
        self._eigenvalues, self._eigenvectors = canonical_geig_solve(
            self._S, self._Hbar, sort_ret_vals=True)
        self._Egs = np.real(self._eigenvalues[0])
        self._Ets = np.real(self._eigenvalues[self._target_root])


class NTSRQK(SRQK):
    """Non-Trotterized SRQK (qkd/nt_srqk.py:22-209): the basis states are exact
    time evolutions of the reference at the points the reference samples,
    expm_multiply(-i H, phi, start=0, stop=dt, num=s+1), i.e. t_m = m dt / s
    (nt_srqk.py:135-137, utils/exp_ops.py:30-33).  Each state is the previous
    one evolved by dt / s on the device (``evolve_exact``); H on it and the
    matrix elements are as in SRQK."""

    def build_qk_mats(self):
        self._omega_lst, homega = [], []
        self._step_energies = []
        n = self._nstates
        S = np.zeros((n, n), dtype=complex)
        H = np.zeros((n, n), dtype=complex)
        ts = np.linspace(0.0, self._dt, n)
        qc = Computer(self._nqb)
        qc.apply_circuit(self._Uprep)
        for m in range(n):
            if m > 0:
                qc = evolve_exact(qc, self._qb_ham, ts[m] - ts[m - 1])
            self._omega_lst.append(qc)
            hq = Computer(qc)
            hq.apply_operator(self._qb_ham)
            homega.append(hq)
            fill_krylov_row(S, H, self._omega_lst, homega, m)
            if self._diagonalize_each_step:
                k = m + 1
                evals, _ = canonical_geig_solve(S[:k, :k], H[:k, :k], sort_ret_vals=True)
                self._step_energies.append(np.real(evals[min(self._target_root, k - 1)]))
        self._n_classical_params = n
        self._n_cnot = 0
        self._n_pauli_trm_measures = n * self._Nl
        self._n_pauli_trm_measures += n * (n - 1) * self._Nl
        self._n_pauli_trm_measures += n * (n - 1)
        return S, H
