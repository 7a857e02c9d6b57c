"""``QubitOperator``: a list of (coefficient, Circuit), as qubit_operator.h:12-72.

Term order and coefficients follow the reference step for step:

* ``canonical_order`` canonicalises every circuit and multiplies in its phase
  (qubit_operator.cc:148-152);
* ``simplify`` combines like terms in first-appearance order, sorts them by
  the reference's Circuit ordering (the ``std::map`` of qubit_operator.cc:
  154-177) and drops |c| <= 1e-12;
* ``operator_product`` forms every (left, right) product with the left
  operator simplified first (qubit_operator.cc:179-201);
* ``order_terms`` sorts by target sequence, then gate-id sequence
  (qubit_operator.cc:125-146).  The reference's comparator ends in
  ``a.size() < a.size()`` (always false) and uses the unstable ``std::sort``,
  so terms that agree on their common prefix have no defined order there;
  here they keep their input order.

Circuits that are canonical Pauli strings are held in mask form throughout.
"""

import functools

from .circuit import Circuit, _product_masks
from .pauli import canonical_key, ipow_mul

__all__ = ["QubitOperator", "to_string"]


def to_string(c):
    """helpers.cc to_string(std::complex<double>)."""
    c = complex(c)
    re, im = c.real, c.imag
    if im == 0.0:
        return f"{re:+.6f}"
    if re == 0.0:
        return f"{im:+.6f}j"
    return f"{re:+.6f} {im:+.6f}i"


class QubitOperator:
    __slots__ = ("_t",)

    def __init__(self):
        self._t = []  # [coeff, Circuit]

    # -- building (bindings.cc:95-116) ----------------------------------------
    def add(self, *args):
        if len(args) == 1:
            self.add_op(args[0])
        else:
            self.add_term(args[0], args[1])

    def add_term(self, coeff, circuit):
        if not isinstance(circuit, Circuit):
            raise TypeError("QubitOperator.add_term expects (complex, Circuit)")
        self._t.append([complex(coeff), circuit])

    def add_op(self, qo):
        for c, circ in qo._t:
            self._t.append([c, circ])

    def set_coeffs(self, new_coeffs):
        if len(new_coeffs) != len(self._t):
            raise ValueError("number of new coefficients for quantum operator must equal ")
        for t, c in zip(self._t, new_coeffs):
            t[0] = complex(c)

    def mult_coeffs(self, multiplier):
        m = complex(multiplier)
        for t in self._t:
            t[0] = t[0] * m

    def terms(self):
        return [(c, circ) for c, circ in self._t]

    def __iter__(self):
        return iter(self.terms())

    def __len__(self):
        return len(self._t)

    # -- algebra -----------------------------------------------------------------
    def canonical_order(self):
        for t in self._t:
            t[0] = t[0] * t[1].canonicalize_pauli_circuit()

    def simplify(self, combine_like_terms=True):
        self.canonical_order()
        acc = {}
        for c, circ in self._t:
            key = circ._pauli if circ._pauli is not None else (0, 0)
            if key in acc:
                acc[key][0] += c
            else:
                acc[key] = [c, circ]
        items = sorted(acc.items(), key=lambda kv: canonical_key(*kv[0]))
        if combine_like_terms:
            self._t = [[v[0], v[1]] for _, v in items if abs(v[0]) > 1.0e-12]
        else:
            self._t = [[v[0], v[1]] for _, v in items]

    def operator_product(self, rqo, pre_simplify=True, post_simplify=True):
        if pre_simplify:
            self.simplify()
        out = []
        for cl, circl in self._t:
            for cr, circr in rqo._t:
                m = _product_masks(circl, circr)
                if m is None:
                    c = Circuit(circl)
                    c.add_circuit(circr)
                    out.append([cl * cr, c])
                else:
                    x, z, e = m
                    # the reference multiplies the canonicalisation phase in
                    # afterwards (canonical_order); i^e products are exact
                    out.append([ipow_mul(cl * cr, e), Circuit._from_masks(x, z)])
        self._t = out
        if post_simplify:
            self.simplify()
        else:
            self.canonical_order()

    def order_terms(self):
        self.simplify()

        def cmp(a, b):
            ga, gb = a[1]._gates(), b[1]._gates()
            n = min(len(ga), len(gb))
            for k in range(n):
                if ga[k].target() != gb[k].target():
                    return -1 if ga[k].target() < gb[k].target() else 1
            for k in range(n):
                if ga[k].gate_id() != gb[k].gate_id():
                    return -1 if ga[k].gate_id() < gb[k].gate_id() else 1
            return 0

        self._t.sort(key=functools.cmp_to_key(cmp))

    def check_op_equivalence(self, qo, reorder):
        other = QubitOperator()
        other._t = [[c, Circuit(circ)] for c, circ in qo._t]
        if reorder:
            self.order_terms()
            other.order_terms()
        if len(self._t) != len(other._t):
            return False
        for (c1, k1), (c2, k2) in zip(self._t, other._t):
            if abs(c1 - c2) > 1.0e-10:
                return False
            if not (k1 == k2):
                return False
        return True

    def num_qubits(self):
        return max((circ.num_qubits() for _, circ in self._t), default=0)

    def str(self):
        return "\n".join(to_string(c) + circ.str() for c, circ in self._t)

    __str__ = str
    __repr__ = str

    # -- mask view used by the device compiler -----------------------------------
    def _pauli_terms(self, applied=True):
        """[(coeff * phase, x, z)] for every term, or None if a term holds a
        non-Pauli gate.  ``applied``: the operator each circuit applies when
        its gates run in list order (Computer::apply_operator semantics);
        otherwise the left-to-right product (operator-algebra semantics)."""
        out = []
        for c, circ in self._t:
            m = circ._applied_pauli_masks() if applied else circ._pauli_masks()
            if m is None:
                return None
            x, z, e = m
            out.append((ipow_mul(c, e), x, z))
        return out
