"""``Circuit``: an ordered gate list, as QForte's ``Circuit`` (circuit.h:13-102).

Two additions serve the device engine without changing what a circuit means:

* a canonical Pauli circuit may be held in mask form (``_pauli = (x, z)``)
  and its ``Gate`` objects built only when someone asks for them, so operator
  algebra on large Hamiltonians does not create hundreds of thousands of
  gate objects;
* a circuit made by ``exponentiate_pauli_string`` carries the exponential it
  implements (``_pexp`` segments: gate range, x, z, angle).  Concatenation and
  ``adjoint`` keep the segments; any other edit drops them.  ``Computer``
  applies an annotated range as one fused pass instead of its 2w+1 gates; the
  two are the same unitary.
"""

from .gate import Gate, make_gate
from .pauli import letters, masks_of_letters, pauli_mul

__all__ = ["Circuit"]

_PAULI_GATES = {}


def _pauli_gate(letter, q):
    g = _PAULI_GATES.get((letter, q))
    if g is None:
        g = make_gate(letter, q, q)
        _PAULI_GATES[(letter, q)] = g
    return g


class Circuit:
    __slots__ = ("_g", "_pauli", "_pexp", "_plan")

    def __init__(self, other=None):
        if other is None:
            self._g = []
            self._pauli = None
            self._pexp = None
            self._plan = None
        else:
            if not isinstance(other, Circuit):
                raise TypeError("Circuit(other) expects a Circuit")
            self._g = None if other._g is None else list(other._g)
            self._pauli = other._pauli
            self._pexp = None if other._pexp is None else list(other._pexp)
            self._plan = other._plan

    @classmethod
    def _from_masks(cls, x, z):
        c = cls.__new__(cls)
        c._g = None
        c._pauli = (x, z)
        c._pexp = None
        c._plan = None
        return c

    # -- internal ---------------------------------------------------------
    def _gates(self):
        if self._g is None:
            x, z = self._pauli
            self._g = [_pauli_gate(l, q) for l, q in letters(x, z)]
        return self._g

    def _edit(self):
        g = self._gates()
        self._pauli = None
        self._pexp = None
        self._plan = None
        return g

    def _pauli_masks(self):
        """(x, z, e) of the left-to-right product of the gates, or None when a
        gate is not X, Y or Z."""
        if self._pauli is not None:
            return self._pauli[0], self._pauli[1], 0
        seq = []
        for g in self._g:
            lab = g.gate_id()
            if lab not in ("X", "Y", "Z") or g.target() != g.control():
                return None
            seq.append((lab, g.target()))
        return masks_of_letters(seq)

    def _applied_pauli_masks(self):
        """(x, z, e) of the operator the gates apply in list order (the last
        gate leftmost), or None when a gate is not X, Y or Z."""
        if self._pauli is not None:
            return self._pauli[0], self._pauli[1], 0
        seq = []
        for g in reversed(self._g):
            lab = g.gate_id()
            if lab not in ("X", "Y", "Z") or g.target() != g.control():
                return None
            seq.append((lab, g.target()))
        return masks_of_letters(seq)

    # -- building (bindings.cc:24-56) -------------------------------------
    def add(self, item):
        if isinstance(item, Gate):
            self.add_gate(item)
        elif isinstance(item, Circuit):
            self.add_circuit(item)
        else:
            raise TypeError("Circuit.add expects a Gate or a Circuit")

    def add_gate(self, gate):
        g = self._gates()
        self._pauli = None
        self._plan = None
        g.append(gate)

    def add_circuit(self, circ):
        g = self._gates()
        n0 = len(g)
        if circ._pexp:
            segs = [] if self._pexp is None else self._pexp
            segs = segs + [(s + n0, e + n0, x, z, th) for (s, e, x, z, th) in circ._pexp]
            self._pexp = segs
        g.extend(circ._gates())
        self._pauli = None
        self._plan = None

    def insert_gate(self, pos, gate):
        if pos > self.size():
            raise RuntimeError("Circuit::insert_gate: position out of range")
        self._edit().insert(pos, gate)

    def remove_gate(self, pos):
        if pos >= self.size():
            raise RuntimeError("Circuit::remove_gate: position out of range")
        del self._edit()[pos]

    def swap_gates(self, pos1, pos2):
        n = self.size()
        if pos1 >= n or pos2 >= n:
            raise RuntimeError("Circuit::swap_gates: position out of range")
        g = self._edit()
        g[pos1], g[pos2] = g[pos2], g[pos1]

    def insert_circuit(self, pos, circ):
        if pos > self.size():
            raise RuntimeError("Circuit::insert_circuit: position out of range")
        g = self._edit()
        g[pos:pos] = list(circ._gates())

    def remove_gates(self, pos1, pos2):
        n = self.size()
        if pos1 >= n or pos2 >= n:
            raise RuntimeError("Circuit::remove_gates: position out of range")
        del self._edit()[pos1:pos2]

    def replace_gate(self, pos, gate):
        if pos >= self.size():
            raise RuntimeError("Circuit::replace_gate: position out of range")
        self._edit()[pos] = gate

    # -- queries ----------------------------------------------------------
    def gates(self):
        return list(self._gates())

    def gate(self, n):
        return self._gates()[n]

    def size(self):
        if self._g is None:
            x, z = self._pauli
            return bin(x | z).count("1")
        return len(self._g)

    def is_pauli(self):
        if self._pauli is not None:
            return True
        return all(g.gate_id() in ("X", "Y", "Z") for g in self._g)

    def num_qubits(self):
        if self._g is None:
            m = self._pauli[0] | self._pauli[1]
            return m.bit_length()
        mx = 0
        for g in self._g:
            mx = max(mx, g.target() + 1, g.control() + 1)
        return mx

    def get_num_cnots(self):
        n = 0
        for g in self._gates():
            lab = g.gate_id()
            if lab in ("CNOT", "cX", "aCNOT", "acX"):
                n += 1
            elif lab in ("A", "SWAP"):
                n += 3
        return n

    def get_parameters(self):
        return [g.parameter() for g in self._gates() if g.has_parameter()]

    def set_parameters(self, params):
        """circuit.cc:10-27."""
        g = self._gates()
        idx = 0
        n = len(params)
        out = list(g)
        for k, gt in enumerate(g):
            if gt.has_parameter():
                if idx < n and abs(gt.parameter() - params[idx]) > 1e-12:
                    out[k] = make_gate(gt.gate_id(), gt.target(), gt.control(), params[idx])
                idx += 1
        if idx != n:
            raise RuntimeError("Circuit::set_parameters: number of parameters does not match "
                               "number of gates with parameters")
        self._g = out
        self._pauli = None
        self._pexp = None
        self._plan = None

    def set_parameter(self, pos, param):
        if pos >= self.size():
            raise RuntimeError("Circuit::set_parameter: position out of range")
        gt = self._gates()[pos]
        if not gt.has_parameter():
            raise RuntimeError("Circuit::set_parameter: gate does not have a parameter")
        self._edit()[pos] = make_gate(gt.gate_id(), gt.target(), gt.control(), param)

    def adjoint(self):
        """Adjoint gates in reverse order (circuit.cc:98-105)."""
        out = Circuit()
        g = self._gates()
        out._g = [gt.adjoint() for gt in reversed(g)]
        if self._pexp:
            n = len(g)
            out._pexp = [(n - e, n - s, x, z, -th) for (s, e, x, z, th) in reversed(self._pexp)]
        return out

    def canonicalize_pauli_circuit(self):
        """Order by qubit and multiply same-qubit Paulis (circuit.cc:107-169).

        The gate list is read as the operator product left to right; returns
        the phase (1, -1, 1j or -1j) that the merge produced."""
        if self._pauli is not None:
            return 1.0 + 0j
        if not self._g:
            return 1.0 + 0j
        if not self.is_pauli():
            raise RuntimeError(
                "Circuit::canonicalize_pauli_circuit is undefined for circuits with gates other "
                "than X, Y, or Z")
        x, z, e = self._pauli_masks()
        self._g = None
        self._pauli = (x, z)
        self._pexp = None
        self._plan = None
        return (1.0 + 0j, 1j, -1.0 + 0j, -1j)[e]

    def simplify(self):
        raise NotImplementedError(
            "Circuit.simplify (gate-commutation peephole, circuit.cc:246-340) is outside the "
            "state-vector path this library provides")

    # -- printing / comparison --------------------------------------------
    def str(self):
        return "[" + " ".join(g.str() for g in reversed(self._gates())) + "]"

    __str__ = str
    __repr__ = str

    def _cmp_key(self):
        return [(g.gate_id(), g.target(), g.control()) for g in self._gates()]

    def __eq__(self, other):
        if not isinstance(other, Circuit):
            return NotImplemented
        if self._pauli is not None and other._pauli is not None:
            return self._pauli == other._pauli
        a, b = self._gates(), other._gates()
        return len(a) == len(b) and all(x == y for x, y in zip(a, b))

    def __lt__(self, other):
        a, b = self._gates(), other._gates()
        for x, y in zip(a, b):
            if x < y:
                return True
            if y < x:
                return False
        return len(a) < len(b)

    __hash__ = None

    def __len__(self):
        return self.size()


def _product_masks(c1, c2):
    """Masks and phase of the operator product c1 . c2 (both Pauli circuits)."""
    m1 = c1._pauli_masks()
    m2 = c2._pauli_masks()
    if m1 is None or m2 is None:
        return None
    x, z, e = pauli_mul(m1[0], m1[1], m2[0], m2[1])
    return x, z, (e + m1[2] + m2[2]) & 3
