"""Compile helpers of the reference: Pauli exponentials, Trotter products,
reference-state preparation and string builders.

* ``exponentiate_pauli_string``  utils/exponentiate.py:9-87
* ``trotterize`` / ``trotterize_w_cRz``  utils/trotterization.py:10-215
* ``build_refprep`` / ``ref_string`` / ``integer_to_ref``  utils/state_prep.py
* ``build_circuit`` / ``build_operator`` / ``smart_print``  helper/io_helper.py

The circuits returned are the reference's gate for gate (basis change, CNOT
ladder, Rz(-2 Im c), uncompute), so their size, CNOT count and printout
match.  Each also records the exponential it implements, which lets
``Computer.apply_circuit`` run it as one fused pass.
"""

import cmath
import math

import numpy as np

from .circuit import Circuit
from .gate import gate as _gate
from .qubit_basis import QubitBasis
from .qubit_operator import QubitOperator

__all__ = ["exponentiate_pauli_string", "trotterize", "trotterize_w_cRz", "build_refprep",
           "ref_string", "integer_to_ref", "build_circuit", "build_operator", "smart_print",
           "open_shell", "correct_spin", "flip_spin", "build_eq_dets"]


def exponentiate_pauli_string(coefficient, term, Use_cRz=False, ancilla_idx=None,
                              Use_open_cRz=False):
    """exp(coefficient * term) for an imaginary coefficient -> (Circuit, phase)."""
    coefficient = complex(coefficient)
    if abs(coefficient.real) > 1.0e-14:
        raise ValueError(
            f"exponentiate_pauli_string() called with a real coefficient {coefficient}")
    if term.size() == 0:
        return (Circuit(), cmath.exp(coefficient))
    exponential = Circuit()
    to_z = Circuit()
    cx_circ = Circuit()
    prev_target = None
    max_target = None
    letters = []
    for g in term.gates():
        gid = g.gate_id()
        target = g.target()
        control = g.control()
        if gid == "X":
            to_z.add(_gate("H", target, control))
        elif gid == "Y":
            to_z.add(_gate("Rx", target, control, np.pi / 2))
        elif gid == "I":
            continue
        letters.append((gid, target))
        if prev_target is not None:
            cx_circ.add(_gate("cX", target, prev_target))
        prev_target = target
        max_target = target
    if Use_cRz:
        z_rot = _gate("cRz", max_target, ancilla_idx, -2.0 * coefficient.imag)
    else:
        z_rot = _gate("Rz", max_target, max_target, -2.0 * coefficient.imag)
    exponential.add(to_z)
    exponential.add(cx_circ)
    if Use_open_cRz:
        exponential.add(_gate("X", ancilla_idx, ancilla_idx))
    exponential.add(z_rot)
    if Use_open_cRz:
        exponential.add(_gate("X", ancilla_idx, ancilla_idx))
    exponential.add(cx_circ.adjoint())
    exponential.add(to_z.adjoint())
    if not Use_cRz and letters:
        # record exp(i theta P): the whole circuit is this one exponential
        x = z = 0
        distinct = True
        for l, q in letters:
            b = 1 << q
            if (x | z) & b:
                distinct = False
                break
            if l in ("X", "Y"):
                x |= b
            if l in ("Y", "Z"):
                z |= b
        if distinct:
            exponential._pexp = [(0, exponential.size(), x, z, coefficient.imag)]
    return (exponential, 1.0)


def trotterize(operator, factor=1.0, trotter_number=1, trotter_order=1):
    """Circuit for exp(factor * operator) as a first-order Trotter product."""
    total_phase = 1.0
    circ = Circuit()
    if trotter_number == 1 and trotter_order == 1:
        for coeff, term in operator.terms():
            gen, phase = exponentiate_pauli_string(factor * coeff, term)
            circ.add_circuit(gen)
            total_phase *= phase
    else:
        if trotter_order > 1:
            raise NotImplementedError("Higher order trotterization is not yet implemented.")
        ho = QubitOperator()
        for _ in range(1, trotter_number + 1):
            for coeff, term in operator.terms():
                ho.add(factor * coeff / float(trotter_number), term)
        for coeff, term in ho.terms():
            gen, phase = exponentiate_pauli_string(coeff, term)
            circ.add_circuit(gen)
            total_phase *= phase
    return (circ, total_phase)


def trotterize_w_cRz(operator, ancilla_qubit_idx, factor=1.0, Use_open_cRz=False,
                     trotter_number=1, trotter_order=1):
    """Controlled Trotter product (utils/trotterization.py:147-215)."""
    total_phase = 1.0
    circ = Circuit()
    if trotter_number == 1 and trotter_order == 1:
        terms = [(factor * c, t) for c, t in operator.terms()]
    else:
        if trotter_order > 1:
            raise NotImplementedError("Higher order trotterization is not yet implemented.")
        terms = []
        for _ in range(1, trotter_number + 1):
            for c, t in operator.terms():
                terms.append((factor * c / float(trotter_number), t))
    for c, t in terms:
        gen, phase = exponentiate_pauli_string(c, t, Use_cRz=True, ancilla_idx=ancilla_qubit_idx,
                                               Use_open_cRz=Use_open_cRz)
        circ.add_circuit(gen)
        total_phase *= phase
    return (circ, total_phase)


def build_refprep(ref):
    refprep = Circuit()
    for j, occupied in enumerate(ref):
        if occupied:
            refprep.add(_gate("X", j, j))
    return refprep


def ref_string(ref, nqb):
    temp = list(ref)
    temp.reverse()
    idx = int("".join(str(x) for x in temp), 2)
    return QubitBasis(idx).str(nqb)


def integer_to_ref(n, nqubits):
    """Occupation list of basis index n (bit k -> qubit k)."""
    return [(n >> k) & 1 for k in range(nqubits)]


def ref_to_basis_idx(ref):
    return sum(int(b) << k for k, b in enumerate(ref))


def build_circuit(Inputstr):
    """'X_0 cX_1_0 Rx_2_0.5' -> Circuit (helper/io_helper.py:52-75)."""
    circ = Circuit()
    for tok in Inputstr.split():
        parts = tok.split("_")
        if len(parts) == 2:
            circ.add(_gate(parts[0], int(parts[1]), int(parts[1])))
        elif "R" in parts[0]:
            circ.add(_gate(parts[0], int(parts[1]), int(parts[1]), float(parts[2])))
        else:
            circ.add(_gate(parts[0], int(parts[1]), int(parts[2])))
    return circ


def build_operator(Inputstr):
    """'c1, circ1; c2, circ2' -> QubitOperator (helper/io_helper.py:87-94)."""
    ops = QubitOperator()
    for term in Inputstr.split(";"):
        c, circ = term.split(",")
        ops.add(complex(c), build_circuit(circ))
    return ops


def smart_print(obj):
    from .computer import Computer
    if isinstance(obj, QubitOperator):
        print("\n Quantum operator:")
        first = True
        for c, circ in obj.terms():
            if not first:
                print("+", end=" ")
            first = False
            print(c, end=" ")
            print("(" + " ".join(circ.str()[1:-1].split(" ")) + ")", "|Ψ>")
    if isinstance(obj, Circuit):
        print("\n Quantum circuit:")
        print("(" + " ".join(obj.str()[1:-1].split(" ")) + ")", "|Ψ>")
    if isinstance(obj, Computer):
        print("\n Quantum Computer:")
        print(obj.str())


# ---------------------------------------------------------------------------
# compact excitation circuits (utils/compact_excitation_circuits.py:9-291)
# ---------------------------------------------------------------------------

def compact_excitation_circuit(theta, creation, annihilation, qubit_excitations):
    """Circuit of exp(theta * kappa) for a particle-number-conserving
    fermionic (kappa = t - t^dagger) or qubit (Q - Q^dagger) excitation with
    few CNOTs (utils/compact_excitation_circuits.py:9-91): a CNOT staircase
    carrying the fermionic sign, a multi-qubit-controlled Ry between CNOT
    ladders, the staircase undone.  The gate list equals the reference's gate
    for gate, so results and CNOT counts match."""
    creation, annihilation = list(creation), list(annihilation)
    if len(creation) != len(annihilation):
        raise ValueError("Compact fermionic/qubit excitations are implemented for "
                         "particle-number-conserving operators only.")
    shared = sorted(set(creation) & set(annihilation))
    if len(shared) > 1:
        raise ValueError("A GSD excitation of the form p^ q^ p q was encountered!")
    cre_u = [p for p in creation if p not in annihilation]
    ann_u = [p for p in annihilation if p not in creation]
    gsd_sign, unique_stair = 1, False
    if shared:
        gsd_sign = -1
        # the repeated index sits at the same position in both lists
        pos = [i for i in range(2) for lst in (creation, annihilation) if lst[i] == shared[0]]
        unique_stair = pos in ([0, 0], [1, 1])
    circ = Circuit()
    stair = None
    if not qubit_excitations:
        stair = (_fermion_sign_circuit(cre_u, ann_u) if unique_stair
                 else _fermion_sign_circuit(creation, annihilation))
        circ.add(stair)
    circ.add(_qubit_excitation(theta, cre_u, ann_u, shared, gsd_sign, qubit_excitations))
    if stair is not None:
        circ.add(stair.adjoint())
    return circ


def _fermion_sign_circuit(creation, annihilation):
    """CNOT staircase and one CZ that give the excitation's fermionic sign
    (compact_excitation_circuits.py:94-149): the qubits below the operator
    indices whose Jordan-Wigner Z strings survive the product, less the
    operator indices themselves."""
    ops = list(creation) + list(annihilation)
    parity = {}
    for p in ops:
        for q in range(p):
            parity[q] = parity.get(q, 0) ^ 1
    keep = [q for q in range(max(ops) + 1) if parity.get(q, 0) and q not in ops]
    keep.reverse()
    circ = Circuit()
    if not keep:
        return circ
    for a, b in zip(keep[1:], keep[:-1]):
        circ.add(_gate("CNOT", a, b))
    circ.add(_gate("cZ", creation[0], keep[-1]))
    return circ


def _qubit_excitation(theta, creation, annihilation, shared, gsd_sign, qubit_excitations):
    """CNOT ladders around the multi-qubit-controlled Ry
    (compact_excitation_circuits.py:152-207)."""
    ladder = Circuit()
    for t in creation[1:]:
        ladder.add(_gate("CNOT", t, creation[0]))
    for t in annihilation[1:]:
        ladder.add(_gate("CNOT", t, annihilation[0]))
    ladder.add(_gate("CNOT", annihilation[0], creation[0]))
    circ = Circuit()
    circ.add(ladder)
    circ.add(_controlled_ry(theta, creation[0], creation[1:], annihilation, shared, gsd_sign,
                            qubit_excitations))
    circ.add(ladder.adjoint())
    return circ


def _controlled_ry(theta, target, ctrl_cre, ctrl_ann, shared, gsd_sign, qubit_excitations):
    """Multi-qubit-controlled Ry(2 theta) as 2^c single-qubit Ry rotations of
    +-theta / 2^(c-1) interleaved with CNOT / anti-controlled CNOT gates in
    Gray-code order (compact_excitation_circuits.py:210-291)."""
    controls = list(ctrl_ann) + list(reversed(ctrl_cre)) + list(shared)
    c = len(controls)
    n_ry = 1 << c
    step = theta / (1 << (c - 1))
    sign_f = 1
    if not qubit_excitations:
        # fermionic sign of the rotation angle by many-body rank
        rank = len(ctrl_ann)
        sign_f = -1
        if rank == 1 or rank % 4 == 0 or (rank - 1) % 4 == 0:
            sign_f = 1
        sign_f *= gsd_sign
    circ = Circuit()
    for i in range(n_ry):
        circ.add(_gate("Ry", target, target, (1 - 2 * (i % 2)) * sign_f * step))
        for j, ctl in enumerate(controls):
            if (i + 1) % (n_ry // (1 << (j + 1))) == 0:
                last = (i + 1) % (n_ry // 2) == 0 or i == n_ry - 1
                circ.add(_gate("CNOT" if (last or shared) else "aCNOT", target, ctl))
                break
    return circ


# ---- open-shell helpers (utils/state_prep.py:53-141) -----------------------
def open_shell(ref):
    """True when some spatial orbital of the determinant is singly occupied."""
    return any(ref[2 * i] + ref[2 * i + 1] == 1 for i in range(len(ref) // 2))


def _spin(ref):
    return sum(0.5 * ref[2 * i] - 0.5 * ref[2 * i + 1] for i in range(len(ref) // 2))


def correct_spin(ref, abs_spin):
    """True when |S_z| of the determinant equals abs_spin."""
    return abs(_spin(ref)) == abs_spin


def flip_spin(ref, orb_idx):
    """The determinant with the alpha and beta occupations of spatial orbital
    orb_idx exchanged."""
    temp = list(ref)
    temp[2 * orb_idx], temp[2 * orb_idx + 1] = ref[2 * orb_idx + 1], ref[2 * orb_idx]
    return temp


def build_eq_dets(open_shell_ref):
    """Every determinant reachable from open_shell_ref by spin flips of its
    singly occupied orbitals with the same |S_z|, the input first, in the order
    the flips discover them (utils/state_prep.py:143-187)."""
    one_e_orbs = [i for i in range(len(open_shell_ref) // 2)
                  if open_shell_ref[2 * i] + open_shell_ref[2 * i + 1] == 1]
    abs_spin = abs(_spin(open_shell_ref))
    found = [list(open_shell_ref)]
    for ref in found:
        for orb in one_e_orbs:
            temp = flip_spin(ref, orb)
            if temp not in found:
                found.append(temp)
    return [r for r in found if correct_spin(r, abs_spin)]


class local_timer:
    """Wall-clock seconds since construction or the last reset (timer.h:6-19,
    bound as qforte.local_timer)."""

    def __init__(self):
        import time
        self._now = time.perf_counter
        self._t0 = self._now()

    def reset(self):
        self._t0 = self._now()

    def get(self):
        return self._now() - self._t0
