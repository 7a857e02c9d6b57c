"""dUCC energies and gradients on the device.

``DUCC`` compiles one problem -- Hamiltonian, operator pool, selected
operators, reference determinant -- into two device programs and a grouped
Hamiltonian, then evaluates, for one parameter vector or a batch of them:

* ``energy``       <Phi|U(t)^dagger H U(t)|Phi>
                   (AnsatzAlgorithm.energy_feval, abc/algorithm.py:458-474)
* ``energy_grad``  the energy and the adjoint gradient
                   (UCCVQE.measure_gradient, abc/uccvqeabc.py:122-251)
* ``pool_gradients``  2 Re <H psi|K_k psi> for every pool operator
                   (UCCVQE.measure_gradient3, abc/uccvqeabc.py:253-283)
* ``residuals``    the energy and the PQE residuals <I_mu|U^dagger H U|ref>
                   (UCCNPQE.get_residual_vector, ucc/uccnpqe.py:249-292)

The forward program holds, per selected operator mu, the JW strings of
t_mu * tau_mu in the order ``get_qubit_operator('commuting_grp_lex')``
gives them (abc/ansatz.py:25-82, sq_op_pool.cc:97-104); the gradient program
holds K_mu = c_mu * JW(tau_mu) in ``jw_transform`` order.  The strings of one
excitation share their x-mask, so each excitation is one fused pass.

``UCCNVQE``, ``ADAPTVQE`` and ``UCCNPQE`` are thin drivers with the
reference's energy/gradient/residual entry points.  ``engine='percall'`` runs the same numbers
through the public ``Computer`` API call for call as the reference's
drivers do (state copies, apply_operator, vdot per parameter) -- the plain
per-call path the fused engine is compared against.
"""

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check, lib, ptr
from .circuit import Circuit
from .computer import Computer, _new_state, inner_product
from .device import prog_from_strings, sum_from_terms
from .gate import gate
from .sq_op_pool import SQOpPool, find_irrep
from .sq_operator import SQOperator
from .utils import build_refprep, compact_excitation_circuit, ref_to_basis_idx, trotterize

__all__ = ["DUCC", "Evaluator", "Pack", "evaluator_config", "UCCNVQE", "ADAPTVQE", "UCCNPQE",
           "SPQE", "ansatz_strings", "gradient_strings"]


def evaluator_config(compact=True):
    """Process-wide: let evaluators created from now on use the compact
    sector paths (True, the default; real states where every coefficient is
    real, two parameter sets per CTA in the forward program), the same with
    one set per CTA ("one-set"), with complex state storage ("complex"), only the
    global-memory one ("global"; "global-complex" with complex storage), or
    keep full-space states (False)."""
    mode = {"global": 2, "global-no-rows": 3, "complex": 4, "global-complex": 5,
            "one-set": 6}.get(compact, 1 if compact else 0)
    check(lib().qfb_ucc_config(mode), "qfb_ucc_config")


class Evaluator:
    """A qfb_ucc evaluator: ``nbatch`` parameter rows per run, its own psi and
    sigma states, device parameter/output blocks and reduction scratch; one
    run is captured into a CUDA graph and replayed."""

    def __init__(self, ducc, nbatch, capture=True):
        self._ducc = ducc  # keeps the programs and the Hamiltonian alive
        self.nbatch = int(nbatch)
        self.nparam = ducc.nparam
        h = ctypes.c_void_p()
        check(lib().qfb_ucc_create(ducc.fwd.h, ducc.grad_prog.h, ducc.unrot_prog.h, ducc.H.h,
                                   ducc.nqubit, ducc.ref_index, self.nbatch, ctypes.byref(h)),
              "qfb_ucc_create")
        self.h = h
        dp, de, dg = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().qfb_ucc_buffers(h, ctypes.byref(dp), ctypes.byref(de), ctypes.byref(dg)))
        self.d_params, self.d_energy, self.d_grad = dp.value, de.value, dg.value
        self.capture = capture
        self._captured = set()
        self.generation = 0  # bumped whenever a run overwrites psi and sigma

    @property
    def device_bytes(self):
        """Device memory this evaluator holds."""
        n = ctypes.c_uint64()
        check(lib().qfb_ucc_memory(self.h, ctypes.byref(n)), "qfb_ucc_memory")
        return n.value

    @property
    def path(self):
        """0: full space; 1: sigma on the sector; 2: compact sector states in
        shared memory; 3: compact sector states in global memory."""
        n = ctypes.c_int32()
        check(lib().qfb_ucc_path(self.h, ctypes.byref(n)), "qfb_ucc_path")
        return n.value

    @property
    def real_states(self):
        """True when the compact states are kept as real doubles."""
        n = ctypes.c_int32()
        check(lib().qfb_ucc_real_states(self.h, ctypes.byref(n)), "qfb_ucc_real_states")
        return bool(n.value)

    @property
    def sets_per_cta(self):
        """Parameter sets a CTA of the compact forward program holds (2: two
        real sets per 16-byte slot; 0: not the compact shared path)."""
        n = ctypes.c_int32()
        check(lib().qfb_ucc_sets_per_cta(self.h, ctypes.byref(n)), "qfb_ucc_sets_per_cta")
        return n.value

    @property
    def h_rows(self):
        """Entries of H on the compact sector (0 unless path == 2)."""
        n = ctypes.c_int64()
        check(lib().qfb_ucc_rows(self.h, ctypes.byref(n)), "qfb_ucc_rows")
        return n.value

    @property
    def sector_size(self):
        """Indices of the particle-number sector H psi is formed on (0: all)."""
        n = ctypes.c_int64()
        check(lib().qfb_ucc_sector(self.h, ctypes.byref(n)), "qfb_ucc_sector")
        return n.value

    def _ensure_graph(self, with_grad):
        if self.capture and with_grad not in self._captured:
            check(lib().qfb_ucc_capture(self.h, int(with_grad)), "qfb_ucc_capture")
            self._captured.add(with_grad)

    def eval(self, P, with_grad=True):
        P = np.ascontiguousarray(P, dtype=np.float64)
        if P.shape != (self.nbatch, self.nparam):
            raise ValueError(f"parameters of shape {P.shape}, expected "
                             f"{(self.nbatch, self.nparam)}")
        self._ensure_graph(with_grad)
        e = np.empty(self.nbatch)
        g = np.empty((self.nbatch, self.nparam)) if with_grad else None
        check(lib().qfb_ucc_eval(self.h, ptr(P), ptr(e), None if g is None else ptr(g)),
              "qfb_ucc_eval")
        self.generation += 1
        return e, g

    def set_pool(self, prog):
        """Give the evaluator an ADAPT pool program (one parameter per operator)."""
        check(lib().qfb_ucc_set_pool(self.h, prog.h), "qfb_ucc_set_pool")
        self._pool_prog = prog  # keeps it alive
        self.npool = prog.nparam
        d = ctypes.c_void_p()
        check(lib().qfb_ucc_pool_buffer(self.h, ctypes.byref(d)), "qfb_ucc_pool_buffer")
        self.d_pool = d.value

    def eval_pool(self, P):
        """Energies and every pool operator's gradient 2 Re <H psi|K_k psi> per row."""
        P = np.ascontiguousarray(P, dtype=np.float64)
        if P.shape != (self.nbatch, self.nparam):
            raise ValueError(f"parameters of shape {P.shape}, expected "
                             f"{(self.nbatch, self.nparam)}")
        self._ensure_graph(3)
        e = np.empty(self.nbatch)
        g = np.empty((self.nbatch, self.npool))
        check(lib().qfb_ucc_eval_pool(self.h, ptr(P), ptr(e), ptr(g)), "qfb_ucc_eval_pool")
        self.generation += 1
        return e, g

    def set_residuals(self, dets, phases):
        """Give the evaluator the PQE excited determinants (basis indices) and
        their phase factors; eval_residuals / run(4) then return the residuals."""
        d = np.ascontiguousarray(dets, dtype=np.uint64)
        ph = np.ascontiguousarray(phases, dtype=np.complex128)
        if d.shape != ph.shape or d.ndim != 1 or len(d) == 0:
            raise ValueError("set_residuals: one phase per determinant, at least one")
        check(lib().qfb_ucc_set_residuals(self.h, ptr(d), ptr(ph), len(d)),
              "qfb_ucc_set_residuals")
        self.nres = len(d)
        r = ctypes.c_void_p()
        check(lib().qfb_ucc_residual_buffer(self.h, ctypes.byref(r)), "qfb_ucc_residual_buffer")
        self.d_res = r.value
        self._captured.discard(4)

    def eval_residuals(self, P):
        """Energies and the PQE residuals Re(<I_k|U^dagger H U|ref> phase_k) per row."""
        P = np.ascontiguousarray(P, dtype=np.float64)
        if P.shape != (self.nbatch, self.nparam):
            raise ValueError(f"parameters of shape {P.shape}, expected "
                             f"{(self.nbatch, self.nparam)}")
        self._ensure_graph(4)
        e = np.empty(self.nbatch)
        r = np.empty((self.nbatch, self.nres))
        check(lib().qfb_ucc_eval_residuals(self.h, ptr(P), ptr(e), ptr(r)),
              "qfb_ucc_eval_residuals")
        self.generation += 1
        return e, r

    def run(self, with_grad=True):
        """Enqueue one evaluation on the library's stream (device buffers in and
        out, no host synchronisation).  ``with_grad`` 0/False: energies; 1/True:
        energies and gradients; 2: the gradient sweep alone on the states the
        last energy-only run left; 3: energies and pool gradients (set_pool);
        4: energies and PQE residuals (set_residuals)."""
        mode = int(with_grad)
        self._ensure_graph(mode)
        check(lib().qfb_ucc_run(self.h, mode), "qfb_ucc_run")
        self.generation += 1

    def tensors(self):
        """(params, energy, grad) as torch float64 CUDA views of the device blocks."""
        import torch

        def view(addr, shape):
            class _I:
                __cuda_array_interface__ = {"shape": shape, "typestr": "<f8",
                                            "data": (int(addr), False), "version": 2}
            return torch.as_tensor(_I(), device="cuda")

        return (view(self.d_params, (self.nbatch, self.nparam)),
                view(self.d_energy, (self.nbatch,)),
                view(self.d_grad, (self.nbatch, self.nparam)))

    def __del__(self):
        try:
            if self.h:
                lib().qfb_ucc_destroy(self.h)
                self.h = None
        except Exception:
            pass


class Pack:
    """Parameter sets of several dUCC problems evaluated in one launch
    (qfb_pack_*): every problem must take the compact shared-memory path
    (``Evaluator.path == 2``: up to ~16 qubits) with the same state storage.
    Item i of a run evaluates ``params[i]`` of problem ``members[i]`` (an index
    into ``duccs``), with its gradient when asked; one CTA per item."""

    def __init__(self, duccs, capacity=256):
        self.duccs = list(duccs)
        self._evs = [d.evaluator(1) for d in self.duccs]  # members: kept alive with the pack
        arr = (ctypes.c_void_p * len(self._evs))(*[ev.h.value for ev in self._evs])
        h = ctypes.c_void_p()
        check(lib().qfb_pack_create(arr, len(self._evs), int(capacity), ctypes.byref(h)),
              "qfb_pack_create")
        self.h = h
        cap, mp, nb = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_uint64()
        check(lib().qfb_pack_info(h, ctypes.byref(cap), ctypes.byref(mp), ctypes.byref(nb)))
        self.capacity, self.maxparam, self.pack_bytes = cap.value, mp.value, nb.value
        pi, pp, pe, pg = (ctypes.c_void_p() for _ in range(4))
        check(lib().qfb_pack_buffers(h, ctypes.byref(pi), ctypes.byref(pp), ctypes.byref(pe),
                                     ctypes.byref(pg)))
        self._addr = (pi.value, pp.value, pe.value, pg.value)

    @property
    def device_bytes(self):
        """Device memory of the pack and of its member evaluators."""
        return self.pack_bytes + sum(ev.device_bytes for ev in self._evs)

    def run(self, members, params, with_grad=True):
        """Energies [n] and gradients (a list of per-item arrays, None where not
        asked) of items (members[i], params[i])."""
        n = len(members)
        m = np.ascontiguousarray(members, dtype=np.int32)
        wg = np.broadcast_to(np.asarray(with_grad, dtype=np.int32), (n,)).copy()
        P = np.zeros((max(n, 1), self.maxparam))
        for i, (k, p) in enumerate(zip(m, params)):
            p = np.asarray(p, dtype=np.float64).reshape(-1)
            if not 0 <= k < len(self.duccs) or p.shape[0] != self.duccs[k].nparam:
                raise ValueError(f"item {i}: member {k} with {p.shape[0]} parameters")
            P[i, :p.shape[0]] = p
        e = np.empty(max(n, 1))
        g = np.empty((max(n, 1), self.maxparam))
        check(lib().qfb_pack_run(self.h, ptr(m), ptr(wg), n, ptr(P), ptr(e), ptr(g)),
              "qfb_pack_run")
        grads = [g[i, :self.duccs[k].nparam].copy() if wg[i] else None for i, k in enumerate(m)]
        return e[:n].copy(), grads

    def tensors(self):
        """(items int32 [capacity, 2], params, energy, grad) as torch CUDA views
        of the device blocks, for callers that stage copies on their own
        streams and enqueue ``launch``."""
        import torch

        def view(addr, shape, typestr):
            class _I:
                __cuda_array_interface__ = {"shape": shape, "typestr": typestr,
                                            "data": (int(addr), False), "version": 2}
            return torch.as_tensor(_I(), device="cuda")

        ai, ap, ae, ag = self._addr
        C, MP = self.capacity, self.maxparam
        return (view(ai, (C, 2), "<i4"), view(ap, (C, MP), "<f8"), view(ae, (C,), "<f8"),
                view(ag, (C, MP), "<f8"))

    def launch(self, nitems):
        """Enqueue the first ``nitems`` items of the device blocks on the
        library's stream."""
        check(lib().qfb_pack_launch(self.h, int(nitems)), "qfb_pack_launch")

    def __del__(self):
        try:
            if self.h:
                lib().qfb_pack_destroy(self.h)
                self.h = None
        except Exception:
            pass


def _sa_components(op):
    """sa_SD operator -> its component anti-Hermitian excitations
    (abc/ansatz.py:38-55)."""
    terms = op.terms()
    half = len(terms) // 2
    out = []
    for coeff, cr, ann in terms[:half]:
        s = SQOperator()
        s.add_term(coeff, cr, ann)
        s.add_term(-coeff, ann, cr)
        out.append(s)
    return out


def _strings_of(qo, who):
    xs, zs, sc = [], [], []
    for c, circ in qo.terms():
        m = circ._pauli_masks()
        if m is None:
            raise ValueError(f"{who}: non-Pauli term")
        x, z, e = m
        if e:
            raise ValueError(f"{who}: non-canonical Pauli term")
        c = complex(c)
        if abs(c.real) > 1.0e-14:
            raise ValueError(f"exponentiate_pauli_string() called with a real coefficient {c}")
        xs.append(x)
        zs.append(z)
        sc.append(c.imag)
    return xs, zs, sc


def ansatz_strings(pool, tops, pool_type=None, qubit_excitations=False):
    """(x, z, scale, param) of U(t) = prod_mu exp(t_mu K_mu) in application order."""
    X, Z, S, P = [], [], [], []
    for mu, top in enumerate(tops):
        op = pool[top][1]
        comps = _sa_components(op) if pool_type == "sa_SD" else [op]
        for comp in comps:
            child = SQOperator()
            child.add_op(comp)
            q = child.jw_transform(qubit_excitations)
            q.simplify()
            q.order_terms()
            xs, zs, sc = _strings_of(q, "ansatz")
            X += xs
            Z += zs
            S += sc
            P += [mu] * len(sc)
    return X, Z, S, P


def gradient_strings(pool, tops, qubit_excitations=False):
    """(x, z, scale, param) of K_mu = c_mu JW(tau_mu) (uccvqeabc.py:154-157, :176-179)."""
    X, Z, S, P = [], [], [], []
    for mu, top in enumerate(tops):
        c, op = pool[top]
        child = SQOperator()
        child.add_op(op)
        q = child.jw_transform(qubit_excitations)
        q.mult_coeffs(c)
        xs, zs, sc = _strings_of(q, "gradient")
        X += xs
        Z += zs
        S += sc
        P += [mu] * len(sc)
    return X, Z, S, P


def _creators_annihilators(sq_op, ref):
    """Creation and annihilation indices of a particle-hole excitation read
    as acting on the reference (uccnpqe.py:197-207, ansatz.py:136-144)."""
    t = sq_op.terms()[0]
    if ref[t[2][-1]]:
        return t[1], t[2]
    return t[2], t[1]


def excited_determinants(pool, tops, ref, qubit_excitations=False):
    """(basis index, phase factor) of each operator's excited determinant
    (UCCNPQE.fill_excited_dets, uccnpqe.py:193-247): the reference with the
    operator's annihilators emptied and creators filled, and the coefficient
    of that determinant in JW(operator)|ref>."""
    ref_idx = ref_to_basis_idx(ref)
    out = []
    for top in tops:
        sq_op = pool[top][1]
        creators, annihilators = _creators_annihilators(sq_op, ref)
        det = list(ref)
        for p in reversed(annihilators):
            if det[p] == 0:
                raise ValueError("no ops should destroy reference, something went wrong!!")
            det[p] = 0
        for p in reversed(creators):
            if det[p] == 1:
                raise ValueError("no ops should destroy reference, something went wrong!!")
            det[p] = 1
        I = ref_to_basis_idx(det)
        q = sq_op.jw_transform(qubit_excitations)
        phase = 0.0 + 0.0j
        for c, x, z in q._pauli_terms(applied=True):
            if ref_idx ^ x == I:
                ny = bin(x & z).count("1")
                sgn = -1.0 if bin(ref_idx & z).count("1") & 1 else 1.0
                phase += complex(c) * (1j ** ny) * sgn
        out.append((I, phase))
    return out


class DUCC:
    """A compiled dUCC problem; evaluations take [nparam] or [batch, nparam]."""

    def __init__(self, hamiltonian, pool, tops, ref, pool_type=None, qubit_excitations=False,
                 nqubit=None):
        self.nqubit = int(nqubit if nqubit is not None else len(ref))
        self.ref = list(ref)
        self.ref_index = ref_to_basis_idx(ref)
        self.tops = list(tops)
        self.nparam = len(self.tops)
        pt = hamiltonian._pauli_terms(applied=True)
        if pt is None:
            raise ValueError("DUCC: the Hamiltonian must be a sum of Pauli strings")
        self.H = sum_from_terms(pt)
        if self.H.maxbit > self.nqubit:
            raise ValueError("Hamiltonian acts beyond the reference's qubits")
        fx, fz, fs, fp = ansatz_strings(pool, self.tops, pool_type, qubit_excitations)
        self.fwd = prog_from_strings(fx, fz, fs, fp, self.nparam)
        gx, gz, gs, gp = gradient_strings(pool, self.tops, qubit_excitations)
        self.grad_prog = prog_from_strings(gx, gz, gs, gp, self.nparam)
        # U_mu is un-applied from K_mu itself for particle-hole pools
        # (uccvqeabc.py:228-230) and from the component excitations of the
        # ansatz for spin-adapted ones (uccvqeabc.py:208-224)
        self.unrot_prog = self.fwd if pool_type == "sa_SD" else self.grad_prog
        self._pool = pool
        self._qe = qubit_excitations
        self._pool_sum = None
        self._evals = {}

    def evaluator(self, nbatch, capture=True):
        """The batched, graph-captured evaluator for ``nbatch`` parameter rows."""
        ev = self._evals.get(nbatch)
        if ev is None:
            ev = Evaluator(self, nbatch, capture)
            if len(self._evals) >= 4:
                self._evals.pop(next(iter(self._evals)))
            self._evals[nbatch] = ev
        return ev

    # ---- states ----------------------------------------------------------
    def _prepare(self, params):
        P = np.ascontiguousarray(np.atleast_2d(np.asarray(params, dtype=np.float64)))
        if P.shape[1] != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters, got {P.shape[1]}")
        B = P.shape[0]
        psi = _new_state(self.nqubit, B)
        try:
            idx = np.array([self.ref_index], dtype=np.uint64)
            one = np.array([1.0 + 0j])
            for b in range(B):
                check(lib().qfb_state_set_basis(psi, b, ptr(idx), ptr(one), 1))
            if self.nparam:
                check(lib().qfb_prog_apply(self.fwd.h, psi, ptr(P), B, 1), "ansatz")
        except Exception:
            lib().qfb_state_destroy(psi)
            raise
        return psi, P, B

    def state(self, params):
        """U(t)|ref> as a Computer (first parameter row)."""
        psi, P, B = self._prepare(np.atleast_2d(params)[:1])
        qc = Computer.__new__(Computer)
        qc._h, qc._n, qc._thr, qc._timings = psi, self.nqubit, 1e-6, []
        return qc

    # ---- evaluations -----------------------------------------------------
    def energy(self, params):
        P = np.ascontiguousarray(np.atleast_2d(np.asarray(params, dtype=np.float64)))
        if P.shape[1] != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters, got {P.shape[1]}")
        e, _ = self.evaluator(P.shape[0]).eval(P, with_grad=False)
        return float(e[0]) if np.ndim(params) == 1 else e

    def energy_grad(self, params):
        P = np.ascontiguousarray(np.atleast_2d(np.asarray(params, dtype=np.float64)))
        if P.shape[1] != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters, got {P.shape[1]}")
        e, g = self.evaluator(P.shape[0]).eval(P, with_grad=True)
        if np.ndim(params) == 1:
            return float(e[0]), g[0]
        return e, g

    def energy_grad_percall(self, params):
        """The same numbers through the per-call C ABI (one call per stage)."""
        psi, P, B = self._prepare(params)
        sig = None
        try:
            sig = _new_state(self.nqubit, B)
            check(lib().qfb_sum_apply(self.H.h, sig, psi), "H psi")
            ev = np.zeros(B, dtype=np.complex128)
            check(lib().qfb_vdot(psi, sig, ptr(ev)), "energy")
            g = np.zeros((B, self.nparam))
            if self.nparam:
                check(lib().qfb_ucc_gradient(self.grad_prog.h, self.unrot_prog.h, psi, sig,
                                             ptr(P), B, ptr(g)), "gradient")
        finally:
            lib().qfb_state_destroy(psi)
            if sig is not None:
                lib().qfb_state_destroy(sig)
        if np.ndim(params) == 1:
            return float(ev.real[0]), g[0]
        return ev.real, g

    def residuals(self, params, dets=None):
        """(energies, PQE residuals) for [nparam] or [batch, nparam] parameters:
        Re(<I_k|U^dagger H U|ref> phase_k) for each excited determinant
        (UCCNPQE.get_residual_vector, uccnpqe.py:249-292), all rows in one
        graph-captured evaluator run (mode 4).  ``dets`` defaults to the
        excited determinants of the ansatz operators."""
        P = np.ascontiguousarray(np.atleast_2d(np.asarray(params, dtype=np.float64)))
        if P.shape[1] != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters, got {P.shape[1]}")
        if dets is None:
            if getattr(self, "_exdets", None) is None:
                self._exdets = excited_determinants(self._pool, self.tops, self.ref, self._qe)
            dets = self._exdets
        ev = self.evaluator(P.shape[0])
        key = tuple(d for d, _ in dets)
        if getattr(ev, "_res_key", None) != key:
            ev.set_residuals([d for d, _ in dets], [ph for _, ph in dets])
            ev._res_key = key
        e, r = ev.eval_residuals(P)
        if np.ndim(params) == 1:
            return float(e[0]), r[0]
        return e, r

    def _pool_sum_handle(self):
        if self._pool_sum is None:
            terms, seg = [], []
            for k, (c, op) in enumerate(self._pool):
                child = SQOperator()
                child.add_op(op)
                q = child.jw_transform(self._qe)
                q.mult_coeffs(c)
                pt = q._pauli_terms(applied=True)
                terms += pt
                seg += [k] * len(pt)
            self._pool_sum = sum_from_terms(terms, seg, len(self._pool))
        return self._pool_sum

    def _pool_program(self):
        if getattr(self, "_pool_prog", None) is None:
            gx, gz, gs, gp = gradient_strings(self._pool, range(len(self._pool)), self._qe)
            self._pool_prog = prog_from_strings(gx, gz, gs, gp, len(self._pool))
        return self._pool_prog

    def pool_gradients(self, params):
        """2 Re <H psi | K_k psi> for every operator of the pool
        (measure_gradient3): the evaluator's graph-captured run of mode 3 (psi,
        sigma, then every operator's inner product in one launch)."""
        P = np.ascontiguousarray(np.atleast_2d(np.asarray(params, dtype=np.float64)))
        ev = self.evaluator(P.shape[0])
        if getattr(ev, "_pool_prog", None) is None:
            try:
                ev.set_pool(self._pool_program())
            except RuntimeError:  # a pool outside the Givens form
                return self.pool_gradients_grouped(params)
        _, g = ev.eval_pool(P)
        return g[0] if np.ndim(params) == 1 else g

    def pool_gradients_grouped(self, params):
        """The same through the grouped Pauli-sum expectation values of the
        pool (one x-group per operator, qfb_sum_expval)."""
        ps = self._pool_sum_handle()
        psi, P, B = self._prepare(params)
        sig = None
        try:
            sig = _new_state(self.nqubit, B)
            check(lib().qfb_sum_apply(self.H.h, sig, psi), "H psi")
            out = np.zeros(B * ps.nsegment, dtype=np.complex128)
            check(lib().qfb_sum_expval(ps.h, sig, psi, ptr(out)), "pool gradients")
        finally:
            lib().qfb_state_destroy(psi)
            if sig is not None:
                lib().qfb_state_destroy(sig)
        g = 2.0 * out.real.reshape(B, ps.nsegment)
        return g[0] if np.ndim(params) == 1 else g


# ---------------------------------------------------------------------------
# drivers
# ---------------------------------------------------------------------------


class _UCCBase:
    def __init__(self, system, reference=None, pool_type="SD", qubit_excitations=False,
                 engine="fused", trotter_number=1, compact_excitations=False):
        self._sys = system
        self._ref = list(system.hf_reference if reference is None else reference)
        self._nqb = len(self._ref)
        self._qb_ham = system.hamiltonian
        self._pool_type = pool_type
        self._qubit_excitations = qubit_excitations
        # compact (FEB / QEB) excitation circuits apply exp(t kappa) exactly, the
        # unitary the fused program applies: only the per-call gate path differs
        self._compact_excitations = compact_excitations
        self._engine = engine
        self._trotter_number = trotter_number
        self._refprep = build_refprep(self._ref)
        self._Uprep = Circuit(self._refprep)
        self._tops = []
        self._tamps = []
        self._pool_obj = SQOpPool()
        self._ducc = None
        self._ducc_key = None
        self._curr_energy = 0.0

    def fill_pool(self):
        if isinstance(self._pool_type, SQOpPool):
            self._pool_obj = self._pool_type
            return
        self._pool_obj = SQOpPool()
        irr = getattr(self._sys, "orb_irreps_to_int", None)
        self._pool_obj.set_orb_spaces(self._ref, irr or [])
        self._pool_obj.fill_pool(self._pool_type)

    def _engine_for_tops(self):
        key = tuple(self._tops)
        if self._ducc is None or self._ducc_key != key:
            pt = self._pool_type if isinstance(self._pool_type, str) else None
            self._ducc = DUCC(self._qb_ham, self._pool_obj, self._tops, self._ref, pt,
                              self._qubit_excitations, self._nqb)
            self._ducc_key = key
        return self._ducc

    # ---- the reference's circuit path (abc/ansatz.py:25-82) ----------------
    def ansatz_circuit(self, amplitudes=None):
        tamps = self._tamps if amplitudes is None else amplitudes
        temp = SQOpPool()
        if self._pool_type == "sa_SD":
            for t, top in zip(tamps, self._tops):
                for comp in _sa_components(self._pool_obj[top][1]):
                    temp.add(t, comp)
        else:
            for t, top in zip(tamps, self._tops):
                temp.add(t, self._pool_obj[top][1])
        if self._compact_excitations:
            U = Circuit()
            for t, sq_op in temp:
                exc = sq_op.terms()[1]
                U.add(compact_excitation_circuit(t * exc[0], exc[1], exc[2],
                                                 self._qubit_excitations))
            return U
        A = temp.get_qubit_operator("commuting_grp_lex", qubit_excitations=self._qubit_excitations)
        U, phase = trotterize(A, trotter_number=self._trotter_number)
        if phase != 1.0 + 0.0j:
            raise ValueError("Encountered phase change, phase not equal to (1.0 + 0.0i)")
        return U

    def build_Uvqc(self, amplitudes=None):
        U = self.ansatz_circuit(amplitudes)
        Uvqc = Circuit()
        Uvqc.add(self._Uprep)
        Uvqc.add(U)
        return Uvqc

    def measure_energy(self, Ucirc, computer=None):
        if computer is None:
            computer = Computer(self._nqb)
        computer.apply_circuit(Ucirc)
        val = computer.direct_op_exp_val(self._qb_ham)
        return float(np.real(val))

    # ---- entry points ------------------------------------------------------
    def energy_feval(self, params):
        if self._engine == "fused":
            e = self._engine_for_tops().energy(np.asarray(params, dtype=np.float64))
        else:
            e = self.measure_energy(self.build_Uvqc(amplitudes=list(params)))
        self._curr_energy = e
        return e

    def measure_gradient(self, params=None):
        p = np.asarray(self._tamps if params is None else params, dtype=np.float64)
        if self._engine == "fused":
            return self._engine_for_tops().energy_grad(p)[1]
        return self._measure_gradient_percall(p)

    def gradient_ary_feval(self, params):
        return np.asarray(self.measure_gradient(params))

    def measure_gradient3(self):
        p = np.asarray(self._tamps, dtype=np.float64)
        if self._engine == "fused":
            return self._engine_for_tops().pool_gradients(p)
        Utot = self.build_Uvqc()
        qc_psi = Computer(self._nqb)
        qc_psi.apply_circuit(Utot)
        qc_sig = Computer(qc_psi)
        qc_sig.apply_operator(self._qb_ham)
        grads = np.zeros(len(self._pool_obj))
        for mu, (coeff, operator) in enumerate(self._pool_obj):
            qc_temp = Computer(qc_psi)
            op = SQOperator()
            op.add_op(operator)
            K = op.jw_transform(self._qubit_excitations)
            K.mult_coeffs(coeff)
            qc_temp.apply_operator(K)
            grads[mu] = 2.0 * np.real(np.vdot(qc_sig.get_coeff_vec(), qc_temp.get_coeff_vec()))
        return grads

    def _measure_gradient_percall(self, params):
        """uccvqeabc.py:122-251 through the Computer API, call for call."""
        M = len(self._tamps)
        grads = np.zeros(M)
        Utot = self.build_Uvqc(list(params))
        qc_psi = Computer(self._nqb)
        qc_psi.apply_circuit(Utot)
        qc_sig = Computer(qc_psi)
        qc_sig.apply_operator(self._qb_ham)
        qc_temp = Computer(qc_psi)
        mu = M - 1

        def K(m):
            c, op = self._pool_obj[self._tops[m]]
            s = SQOperator()
            s.add_op(op)
            q = s.jw_transform(self._qubit_excitations)
            q.mult_coeffs(c)
            return q

        Kmu_prev = K(mu)
        qc_temp.apply_operator(Kmu_prev)
        grads[mu] = 2.0 * np.real(np.vdot(qc_sig.get_coeff_vec(), qc_temp.get_coeff_vec()))
        for mu in reversed(range(M - 1)):
            tamp = params[mu + 1]
            Kmu = K(mu)
            if self._pool_type == "sa_SD":
                Umu = Circuit()
                for comp in _sa_components(self._pool_obj[self._tops[mu + 1]][1]):
                    q = comp.jw_transform(self._qubit_excitations)
                    U, p = trotterize(q, factor=-tamp, trotter_number=self._trotter_number)
                    Umu.add(U)
            else:
                Umu, _ = trotterize(Kmu_prev, factor=-tamp, trotter_number=self._trotter_number)
            qc_sig.apply_circuit(Umu)
            qc_psi.apply_circuit(Umu)
            qc_temp = Computer(qc_psi)
            qc_temp.apply_operator(Kmu)
            grads[mu] = 2.0 * np.real(np.vdot(qc_sig.get_coeff_vec(), qc_temp.get_coeff_vec()))
            Kmu_prev = Kmu
        return grads

    def get_gs_energy(self):
        return self._Egs


class UCCNVQE(_UCCBase):
    """dUCC-VQE with all pool operators (ucc/uccnvqe.py:42-271)."""

    def run(self, opt_thresh=1.0e-5, opt_maxiter=200, pool_type=None, optimizer="BFGS",
            use_analytic_grad=True):
        from scipy.optimize import minimize
        if pool_type is not None:
            self._pool_type = pool_type
        self.fill_pool()
        self._tops = list(range(len(self._pool_obj)))
        self._tamps = [0.0] * len(self._pool_obj)
        x0 = np.array(self._tamps)
        opts = {"maxiter": opt_maxiter}
        if optimizer in ("BFGS", "CG", "L-BFGS-B", "TNC", "trust-constr"):
            opts["gtol"] = opt_thresh
        res = minimize(self.energy_feval, x0, method=optimizer,
                       jac=self.gradient_ary_feval if use_analytic_grad else None, options=opts)
        self._Egs = float(res.fun)
        self._tamps = list(res.x)
        self._final_result = res
        return self._Egs


class UCCNPQE(_UCCBase):
    """dUCC-PQE with all pool operators (ucc/uccnpqe.py:24-300): solve the
    projective equations r_mu(t) = <I_mu|U^dagger H U|ref> = 0 by Jacobi
    iterations with Moller-Plesset denominators and DIIS (maths/optimizer.py:
    6-116), or by a scipy minimiser of the summed squared residuals
    (:119-176).  Residuals come from the evaluator's residual run (psi, H psi,
    U^dagger on sigma and the projections in one launch)."""

    _SCIPY_SOLVERS = ("nelder-mead", "powell", "bfgs", "l-bfgs-b", "cg", "slsqp")

    def __init__(self, system, reference=None, max_moment_rank=0, moment_dt=None, **kwargs):
        super().__init__(system, reference, **kwargs)
        self._max_moment_rank = max_moment_rank
        self._moment_dt = moment_dt

    def run(self, pool_type="SD", opt_thresh=1.0e-5, opt_maxiter=40, noise_factor=0.0,
            optimizer="jacobi", diis_max_dim=8):
        if pool_type == "sa_SD":
            raise ValueError("Must use single term particle-hole nbody operators for residual "
                             "calculation")
        self._check_optimizer(optimizer)
        self._optimizer = optimizer
        self._energies = []
        self._pool_type = pool_type
        self._opt_thresh = opt_thresh
        self._opt_maxiter = opt_maxiter
        self._noise_factor = noise_factor
        self._diis_max_dim = diis_max_dim
        self._res_vec_evals = 0
        self._res_m_evals = 0
        self.fill_pool()
        self.initialize_ansatz()
        self.fill_excited_dets()
        self.build_orb_energies()
        self.solve()
        if self._max_moment_rank:
            self.construct_moment_space()
            self.compute_moment_energies()
        return self._Egs

    # ---- moment energy corrections (utils/moment_energy_corrections.py) -------
    def construct_moment_space(self):
        """utils/moment_energy_corrections.py:19-98: the determinants of the
        reference's sector (irrep 0) up to max_moment_rank-fold excitations,
        with their Moller-Plesset denominators and Epstein-Nesbet diagonal
        energies <det|H|det>.  The latter are the sums of H's diagonal terms
        c (-1)^{|det & z|} (only x = 0 strings have diagonal elements), formed
        from the term table rather than by a state-vector pass per
        determinant as in the reference."""
        self._E_mmcc_mp, self._E_mmcc_en = [], []
        if not hasattr(self, "_orb_e"):
            self.build_orb_energies()
        nel = sum(self._ref)
        if not isinstance(self._max_moment_rank, int) or self._max_moment_rank < 0:
            raise TypeError("The maximum moment rank must be a non-negative integer!")
        if self._max_moment_rank > nel:
            self._max_moment_rank = nel
        ex = _sector_excitations(self, self._max_moment_rank, 0)
        self._mmcc_pool = SQOpPool()
        for _, _, _, sq_op in ex:
            self._mmcc_pool.add_term(0.0, sq_op)
        self._mmcc_excitation_indices = [I for I, _, _, _ in ex]
        self._mpdenom = [sum(self._orb_e[x] for x in occ) - sum(self._orb_e[x] for x in unocc)
                         for _, occ, unocc, _ in ex]
        diag = [(complex(c), z) for c, x, z in self._qb_ham._pauli_terms(applied=True) if x == 0]
        self._epstein_nesbet = [
            sum(c * (-1.0 if bin(I & z).count("1") & 1 else 1.0) for c, z in diag)
            for I in self._mmcc_excitation_indices]

    def compute_moment_energies(self):
        """utils/moment_energy_corrections.py:101-150: residuals of the moment
        space from U^dagger exp(i dt H) U |ref> / dt, and the MP- and EN-
        denominator corrected energies."""
        if self._moment_dt is None:
            self._moment_dt = 0.001
        eiH, _ = trotterize(self._qb_ham, factor=self._moment_dt * (0.0 + 1.0j),
                            trotter_number=self._trotter_number)
        U = self.ansatz_circuit()
        qc = Computer(self._nqb)
        qc.apply_circuit(self._Uprep)
        qc.apply_circuit(U)
        qc.apply_circuit(eiH)
        qc.apply_circuit(U.adjoint())
        coeffs = qc.get_coeff_array()
        res = [coeffs[I] / self._moment_dt for I in self._mmcc_excitation_indices]
        E = self._curr_energy
        self._E_mmcc_mp.append(E + sum(np.real(np.conj(r) * r / d)
                                       for r, d in zip(res, self._mpdenom)))
        self._E_mmcc_en.append(E + sum(np.real(np.conj(r) * r / (E - en))
                                       for r, en in zip(res, self._epstein_nesbet)))

    def _check_optimizer(self, optimizer):
        if optimizer.lower() != "jacobi" and optimizer.lower() not in self._SCIPY_SOLVERS:
            raise NotImplementedError("Currently only Jacobi, Nelder-Mead, Powell, BFGS, "
                                      "L-BFGS-B, CG, and SLSQP solvers are implemented")

    def solve(self):
        """abc/uccpqeabc.py:108-123."""
        if self._optimizer.lower() == "jacobi":
            self.jacobi_solver()
        else:
            self.scipy_solver(self.get_sum_residual_square)

    def get_sum_residual_square(self, tamps):
        """abc/uccpqeabc.py:101-106: the function the scipy solvers minimise."""
        r = self.get_residual_vector(tamps)
        return float(np.sum(np.square(np.abs(r))))

    def scipy_solver(self, function_to_minimize):
        """maths/optimizer.py:119-176: scipy.optimize.minimize of the summed
        squared residuals, with the reference's tolerance options."""
        from scipy.optimize import minimize
        opts = {"maxiter": self._opt_maxiter}
        method = self._optimizer.lower()
        if method in ("bfgs", "cg", "l-bfgs-b"):
            opts["gtol"] = self._opt_thresh
        if method == "nelder-mead":
            opts["fatol"] = self._opt_thresh
            opts["adaptive"] = True
        if method in ("powell", "l-bfgs-b", "slsqp"):
            opts["ftol"] = self._opt_thresh
        res = minimize(function_to_minimize, list(self._tamps), method=self._optimizer,
                       options=opts)
        self._tamps = list(res.x)
        self._Egs = self.energy_feval(self._tamps)
        self._energies.append(self._Egs)

    def initialize_ansatz(self):
        self._tops = list(range(len(self._pool_obj)))
        self._tamps = [0.0] * len(self._pool_obj)

    def fill_excited_dets(self):
        self._excited_dets = excited_determinants(self._pool_obj, self._tops, self._ref,
                                                  self._qubit_excitations)

    def build_orb_energies(self):
        """Spin-orbital energies (abc/ansatz.py:84-119): the system's RHF
        orbital energies when it has them, else from the reference energy
        and its single flips."""
        self._orb_e = []
        if hasattr(self._sys, "hf_orbital_energies"):
            for e in self._sys.hf_orbital_energies:
                self._orb_e += [e] * 2
            return
        qc = Computer(self._nqb)
        qc.apply_circuit(self._refprep)
        E0 = float(np.real(qc.direct_op_exp_val(self._qb_ham)))
        nocc = sum(self._ref)
        for i in range(self._nqb):
            qc = Computer(self._nqb)
            qc.apply_circuit(self._refprep)
            qc.apply_gate(gate("X", i, i))
            Ei = float(np.real(qc.direct_op_exp_val(self._qb_ham)))
            self._orb_e.append(E0 - Ei if i < nocc else Ei - E0)

    def get_res_over_mpdenom(self, residuals):
        out = []
        for mu, m in enumerate(self._tops):
            creators, annihilators = _creators_annihilators(self._pool_obj[m][1], self._ref)
            denom = sum(self._orb_e[x] for x in annihilators) - sum(self._orb_e[x] for x in creators)
            out.append(residuals[mu] / denom)
        return out

    def get_residual_vector(self, trial_amps):
        p = np.asarray(trial_amps, dtype=np.float64)
        if self._engine == "fused":
            eng = self._engine_for_tops()
            E, r = eng.residuals(p, self._excited_dets)
            self._curr_energy = E
        else:
            r = self._residuals_percall(p)
        r = np.asarray(r, dtype=np.float64)
        if self._noise_factor > 1e-12:
            r = np.random.normal(r, self._noise_factor)
        self._res_vec_norm = float(np.linalg.norm(r))
        self._res_vec_evals += 1
        self._res_m_evals += len(self._tamps)
        return list(r)

    def _residuals_percall(self, params):
        """uccnpqe.py:249-292 through the Computer API, call for call."""
        U = self.ansatz_circuit(list(params))
        qc = Computer(self._nqb)
        qc.apply_circuit(self._Uprep)
        qc.apply_circuit(U)
        qc.apply_operator(self._qb_ham)
        qc.apply_circuit(U.adjoint())
        coeffs = qc.get_coeff_vec()
        out = []
        for I, ph in self._excited_dets:
            r = coeffs[I] * ph
            if abs(np.imag(r)) > 1.0e-12:
                raise ValueError("residual has imaginary component, something went wrong!!")
            out.append(float(np.real(r)))
        return out

    def jacobi_solver(self):
        import copy
        t_diis = [copy.deepcopy(self._tamps)]
        e_diis = []
        Ek = self.energy_feval(self._tamps)
        self._energies = []
        for _ in range(1, self._opt_maxiter + 1):
            t_old = copy.deepcopy(self._tamps)
            r_k = self.get_res_over_mpdenom(self.get_residual_vector(self._tamps))
            self._tamps = list(np.add(self._tamps, r_k))
            t_diis.append(copy.deepcopy(self._tamps))
            e_diis.append(np.subtract(copy.deepcopy(self._tamps), t_old))
            if self._diis_max_dim >= 2:
                self._tamps = _diis(self._diis_max_dim, t_diis, e_diis)
            Ek = self.energy_feval(self._tamps)
            self._energies.append(Ek)
            if self._res_vec_norm < self._opt_thresh:
                break
        self._Egs = Ek


def _sector_excitations(alg, max_rank, irrep):
    """(basis index, occupied, unoccupied, tau - tau^dagger) for every
    determinant of the reference's (N_alpha, N_beta) sector and irrep, other
    than the reference, of excitation rank <= max_rank, in basis-index order
    (spqe.py:186-240, utils/moment_energy_corrections.py:42-90)."""
    ref = alg._ref
    nq = alg._nqb
    ref_idx = ref_to_basis_idx(ref)
    nalpha = sum(ref[0::2])
    nbeta = sum(ref[1::2])
    irreps = getattr(alg._sys, "orb_irreps_to_int", None) or [0] * (nq // 2 + 1)
    # the sector's determinants (alpha strings x beta strings) in basis-index
    # order: the reference scans all 2^n indices for them
    from itertools import combinations
    alpha_strings = [sum(1 << q for q in c) for c in combinations(range(0, nq, 2), nalpha)]
    beta_strings = [sum(1 << q for q in c) for c in combinations(range(1, nq, 2), nbeta)]
    out = []
    for I in sorted(a | b for a in alpha_strings for b in beta_strings):
        occ = [q for q in range(nq) if I >> q & 1]
        if find_irrep(irreps, occ) != irrep:
            continue
        excit = ref_idx ^ I
        if excit == 0 or bin(excit).count("1") // 2 > max_rank:
            continue
        occ_idx = [q for q in range(nq) if excit >> q & 1 and ref[q] == 1]
        unocc_idx = [q for q in range(nq) if excit >> q & 1 and ref[q] == 0]
        sq_op = SQOperator()
        sq_op.add(+1.0, unocc_idx, occ_idx)
        sq_op.add(-1.0, occ_idx[::-1], unocc_idx[::-1])
        sq_op.simplify()
        out.append((I, occ_idx, unocc_idx, sq_op))
    return out


class SPQE(UCCNPQE):
    """Selected PQE (ucc/spqe.py:24-605): grow the ansatz from the residuals of
    every determinant of the reference's particle-number sector, then solve the
    projective equations of the chosen operators with UCCNPQE's Jacobi / DIIS
    iterations.

    The selection step applies U, exp(i dt H) (trotterized) and U^dagger to the
    reference as the reference does (spqe.py:427-442); |r_I|^2 is read from the
    resulting amplitudes of the pool's determinants.  The micro-iterations take
    their residuals from the evaluator's residual run (engine "fused") or from
    the reference's Computer calls (engine "percall"), solved by Jacobi / DIIS
    or a scipy minimiser of the summed squared residuals.  A finite M_omega
    estimates the selection residuals from seeded device draws.
    """

    def __init__(self, system, reference=None, diis_max_dim=8, irrep=0, **kwargs):
        super().__init__(system, reference, **kwargs)
        self._diis_max_dim = diis_max_dim
        self._irrep = irrep

    def run(self, spqe_thresh=1.0e-2, spqe_maxiter=20, dt=0.001, M_omega="inf",
            opt_thresh=1.0e-5, opt_maxiter=30, use_cumulative_thresh=True,
            max_excit_rank=None, optimizer="Jacobi", seed=None):
        """``seed`` (not in the reference, whose draws are unseeded) fixes the
        device sampler's draws of a finite ``M_omega``: macro-iteration k
        draws with seed + k."""
        self._check_optimizer(optimizer)
        self._spqe_thresh = spqe_thresh
        self._spqe_maxiter = spqe_maxiter
        self._dt = dt
        self._M_omega = M_omega if M_omega == "inf" else int(M_omega)
        self._seed = seed
        self._use_cumulative_thresh = use_cumulative_thresh
        self._optimizer = optimizer
        self._opt_thresh = opt_thresh
        self._opt_maxiter = opt_maxiter
        self._noise_factor = 0.0
        self._nbody_counts = []
        self._n_classical_params_lst = []
        self._energies = []
        self._tops = []
        self._tamps = []
        self._stop_macro = False
        self._converged = False
        self._res_vec_evals = 0
        self._res_m_evals = 0
        self._curr_energy = 0.0
        self._eiH, _ = trotterize(self._qb_ham, factor=self._dt * (0.0 + 1.0j),
                                  trotter_number=self._trotter_number)
        for occupation in self._ref:
            if occupation:
                self._nbody_counts.append(0)
        self._build_determinant_pool(max_excit_rank)
        self.build_orb_energies()
        if self._max_moment_rank:
            self.construct_moment_space()
        self._spqe_iter = 1
        while not self._stop_macro:
            self.update_ansatz()
            if self._converged:
                break
            self.fill_excited_dets()
            self.solve()
            if self._max_moment_rank:
                self.compute_moment_energies()
            self._spqe_iter += 1
        self._Egs = self._energies[-1]
        return self._Egs

    def _build_determinant_pool(self, max_excit_rank):
        """One operator per determinant of the reference's (N_alpha, N_beta)
        sector and irrep, up to max_excit_rank-fold excitations, in basis-index
        order (spqe.py:159-240): tau - tau^dagger with the determinant's
        creators and annihilators in ascending order."""
        nalpha = sum(self._ref[0::2])
        nbeta = sum(self._ref[1::2])
        if max_excit_rank is None:
            max_excit_rank = nalpha + nbeta
        elif not isinstance(max_excit_rank, int) or max_excit_rank <= 0:
            raise TypeError("The maximum excitation rank max_excit_rank must be a positive integer!")
        elif max_excit_rank > nalpha + nbeta:
            max_excit_rank = nalpha + nbeta
        self._pool_type = max_excit_rank
        self._pool_obj = SQOpPool()
        self._coeff_idx_to_pool_idx = {}
        self._indices_of_zeroable_residuals_for_pool = set()
        for I, _, _, sq_op in _sector_excitations(self, max_excit_rank, self._irrep):
            self._coeff_idx_to_pool_idx[I] = len(self._pool_obj)
            self._indices_of_zeroable_residuals_for_pool.add(I)
            self._pool_obj.add_term(0.0, sq_op)
        self._pool_idx_to_coeff_idx = {v: k for k, v in self._coeff_idx_to_pool_idx.items()}

    def update_ansatz(self):
        """spqe.py:427-590 (M_omega = 'inf'): residuals of every pool
        determinant not yet in the ansatz from U^dagger exp(i dt H) U |ref>.
        The reference's energy evaluation at the start of this step only
        feeds a printout and is not repeated here."""
        U = self.ansatz_circuit()
        qc = Computer(self._nqb)
        qc.apply_circuit(self._Uprep)
        qc.apply_circuit(U)
        qc.apply_circuit(self._eiH)
        qc.apply_circuit(U.adjoint())
        if self._M_omega != "inf":
            self._update_ansatz_sampled(qc)
            return
        coeffs = qc.get_coeff_array()
        in_ansatz = {self._pool_idx_to_coeff_idx[i] for i in self._tops}
        res_sq = [(float(np.real(np.conj(coeffs[I]) * coeffs[I])), I)
                  for I in self._indices_of_zeroable_residuals_for_pool - in_ansatz]
        res_sq.sort()
        self._curr_res_sq_norm = sum(r for r, _ in res_sq) / (self._dt * self._dt)
        self.conv_status()
        if self._converged:
            return
        if self._use_cumulative_thresh:
            res_sq_sum = 0.0
            temp_ops = []
            for rmu_sq, I in res_sq:
                res_sq_sum += rmu_sq / (self._dt * self._dt)
                if res_sq_sum > self._spqe_thresh * self._spqe_thresh:
                    pool_idx = self._coeff_idx_to_pool_idx[I]
                    if pool_idx not in self._tops:
                        temp_ops.append(pool_idx)
                        rank = len(self._pool_obj[pool_idx][1].terms()[0][1])
                        self._nbody_counts[rank - 1] += 1
            for op in temp_ops[::-1]:
                self._tops.insert(0, op)
                self._tamps.insert(0, 0.0)
        else:
            for rmu_sq, I in reversed(res_sq):
                pool_idx = self._coeff_idx_to_pool_idx[I]
                if pool_idx not in self._tops:
                    self._tops.insert(0, pool_idx)
                    self._tamps.insert(0, 0.0)
                    rank = len(self._pool_obj[pool_idx][1].terms()[0][1])
                    self._nbody_counts[rank - 1] += 1
                    break
        self._n_classical_params_lst.append(len(self._tops))

    def _update_ansatz_sampled(self, qc):
        """spqe.py:444-503: M_omega draws of basis states from |r_I|^2 estimate
        the residuals.  The draws come from the device sampler (no read-back of
        the state); the estimated norm sums every sampled fraction but the
        largest, and the step converges when one determinant takes every
        draw.  Otherwise every sampled determinant but the most frequent one
        enters the ansatz front first, in increasing count order.  Two
        departures from the reference: a determinant enters only if its
        operator is not already in the ansatz (the reference compares the
        determinant's index with the operator indices, so it can add an
        operator twice), and spqe_maxiter bounds the macro-iterations here as
        it does with exact residuals (the reference's sampled loop has no
        bound).  Determinants outside the pool are skipped."""
        seed = None if self._seed is None else int(self._seed) + self._spqe_iter
        draws = np.asarray(qc.sample(self._M_omega, seed), dtype=np.int64)
        mus, counts = np.unique(draws, return_counts=True)
        nmu = sorted(zip(counts.tolist(), mus.tolist()))
        frac = [(c / self._M_omega, mu) for c, mu in nmu]
        self._curr_res_sq_norm = sum(f for f, _ in sorted(frac)[:-1]) / (self._dt * self._dt)
        if len(nmu) == 1:
            self._converged = True
            self._stop_macro = True
            return
        if self._spqe_iter > self._spqe_maxiter:
            self._stop_macro = True
            return
        for _, mu in nmu[:-1]:
            pool_idx = self._coeff_idx_to_pool_idx.get(mu)
            if pool_idx is None or pool_idx in self._tops:
                continue
            self._tops.insert(0, pool_idx)
            self._tamps.insert(0, 0.0)
            rank = len(self._pool_obj[pool_idx][1].terms()[0][1])
            self._nbody_counts[rank - 1] += 1
        self._n_classical_params_lst.append(len(self._tops))

    def conv_status(self):
        """spqe.py:593-603."""
        if abs(self._curr_res_sq_norm) < abs(self._spqe_thresh * self._spqe_thresh):
            self._converged = True
            self._stop_macro = True
        elif self._spqe_iter > self._spqe_maxiter:
            self._converged = False
            self._stop_macro = True
        elif len(self._tops) == len(self._pool_obj):
            self._converged = True
            self._stop_macro = True

    def jacobi_solver(self):
        """maths/optimizer.py:40-116 as SPQE runs it: the energies list gets
        one entry per macro-iteration, the final one."""
        import copy
        t_diis = [copy.deepcopy(self._tamps)]
        e_diis = []
        Ek = self.energy_feval(self._tamps)
        for _ in range(1, self._opt_maxiter + 1):
            t_old = copy.deepcopy(self._tamps)
            r_k = self.get_res_over_mpdenom(self.get_residual_vector(self._tamps))
            self._tamps = list(np.add(self._tamps, r_k))
            t_diis.append(copy.deepcopy(self._tamps))
            e_diis.append(np.subtract(copy.deepcopy(self._tamps), t_old))
            if self._diis_max_dim >= 2:
                self._tamps = _diis(self._diis_max_dim, t_diis, e_diis)
            Ek = self.energy_feval(self._tamps)
            if self._res_vec_norm < self._opt_thresh:
                break
        self._Egs = Ek
        self._energies.append(Ek)


def _diis(diis_max_dim, t_diis, e_diis):
    """DIIS extrapolation of the amplitudes (maths/optimizer.py:6-37)."""
    import copy
    if len(t_diis) > diis_max_dim:
        del t_diis[0]
        del e_diis[0]
    dim = len(t_diis) - 1
    B = np.ones((dim + 1, dim + 1)) * -1
    bsol = np.zeros(dim + 1)
    B[-1, -1] = 0.0
    bsol[-1] = -1.0
    for i, ei in enumerate(e_diis):
        for j, ej in enumerate(e_diis):
            B[i, j] = np.dot(np.real(ei), np.real(ej))
    B[:-1, :-1] /= np.abs(B[:-1, :-1]).max()
    x = np.linalg.lstsq(B, bsol, rcond=None)[0][:-1]
    t_new = np.zeros(len(t_diis[0]))
    for l in range(dim):
        t_new = np.add(t_new, x[l] * np.asarray(t_diis[l + 1]))
    return copy.deepcopy(list(np.real(t_new)))


class ADAPTVQE(_UCCBase):
    """ADAPT-VQE (ucc/adaptvqe.py:81-458): grow the ansatz by the largest
    pool gradient, re-optimise, repeat."""

    def run(self, avqe_thresh=1.0e-2, pool_type=None, opt_thresh=1.0e-5, opt_maxiter=200,
            adapt_maxiter=20, optimizer="BFGS"):
        from scipy.optimize import minimize
        if pool_type is not None:
            self._pool_type = pool_type
        self.fill_pool()
        self._tops, self._tamps = [], []
        self._energies, self._grad_norms = [], []
        for _ in range(adapt_maxiter):
            grads = self.measure_gradient3()
            norm = float(np.sqrt(np.sum(grads ** 2)))
            self._grad_norms.append(norm)
            if norm < abs(avqe_thresh):
                break
            k = int(np.argmax(np.abs(grads)))
            self._tops.append(k)
            self._tamps.append(0.0)
            res = minimize(self.energy_feval, np.array(self._tamps), method=optimizer,
                           jac=self.gradient_ary_feval,
                           options={"gtol": opt_thresh, "maxiter": opt_maxiter})
            self._tamps = list(res.x)
            self._energies.append(float(res.fun))
        self._Egs = self._energies[-1] if self._energies else self.energy_feval([])
        return self._Egs
