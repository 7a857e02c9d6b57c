"""``SQOperator``: second-quantised operators and the Jordan-Wigner map.

Restates sq_operator.h:14-85 / sq_operator.cc:1-186.  A term is
``(coeff, cre, ann)`` meaning coeff * cre[0]^ cre[1]^ ... ann[0] ann[1] ...

``jw_transform`` follows the reference's sequence of operations exactly --
simplify, then per term the running product of
a_p^dagger -> (X_p - i Y_p)/2 Z_{<p} and a_p -> (X_p + i Y_p)/2 Z_{<p}
factors (each product simplified), times the term coefficient, and a final
simplify -- so the resulting term list, its order and its coefficients are
the reference's.  The image of each (cre, ann) index pattern is cached: it
does not depend on the coefficient, so Hamiltonians that share a pattern
set (every random-integral Hamiltonian of a given orbital count) transform
in one pass over their terms.
"""

import functools

from .circuit import Circuit
from .qubit_operator import QubitOperator, to_string
from .pauli import canonical_key, ipow_mul, pauli_mul

__all__ = ["SQOperator"]


def _perm_parity(order):
    """Parity of the permutation ``order`` (sq_operator.cc:175-191)."""
    inv = 0
    n = len(order)
    for i in range(n):
        oi = order[i]
        for j in range(i + 1, n):
            if order[j] < oi:
                inv += 1
    return inv & 1


def _canon(ops):
    """Indices sorted descending and the sign of that permutation
    (canonicalize_helper, sq_operator.cc:127-140)."""
    order = sorted(range(len(ops)), key=lambda i: -ops[i])
    return [ops[i] for i in order], (-1 if _perm_parity(order) else 1)


def _simplify_masks(terms):
    """QubitOperator::simplify on [(c, x, z)] already canonical."""
    acc = {}
    for c, x, z in terms:
        k = (x, z)
        if k in acc:
            acc[k] += c
        else:
            acc[k] = c
    items = sorted(acc.items(), key=lambda kv: canonical_key(*kv[0]))
    return [(c, k[0], k[1]) for k, c in items if abs(c) > 1.0e-12]


def _product_masks(left, right):
    out = []
    for cl, xl, zl in left:
        for cr, xr, zr in right:
            x, z, e = pauli_mul(xl, zl, xr, zr)
            out.append((ipow_mul(cl * cr, e), x, z))
    return out


@functools.lru_cache(maxsize=None)
def _jw_image(cre, ann, qubit_excitation):
    """jw_helper (sq_operator.cc:193-223) for the creators then the
    annihilators: [(c, x, z)] before the term coefficient is applied."""
    holder = []
    for ops, creator in ((cre, True), (ann, False)):
        halfi = complex(-0.0, -0.5) if creator else complex(0.0, 0.5)
        for p in ops:
            zs = 0 if qubit_excitation else (1 << p) - 1
            b = 1 << p
            temp = [(complex(0.5, 0.0), b, zs), (halfi, b, zs | b)]
            if not holder:
                holder = temp
            else:
                holder = _simplify_masks(_product_masks(_simplify_masks(holder), temp))
    return tuple(holder)


class SQOperator:
    __slots__ = ("_t",)

    def __init__(self):
        self._t = []  # [coeff, [cre], [ann]]

    def add(self, *args):
        if len(args) == 1:
            self.add_op(args[0])
        else:
            self.add_term(*args)

    def add_term(self, coeff, cre_ops, ann_ops):
        self._t.append([complex(coeff), [int(i) for i in cre_ops], [int(i) for i in ann_ops]])

    def add_op(self, sqo):
        for c, cr, an in sqo._t:
            self._t.append([c, list(cr), list(an)])

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
        return [(c, list(cr), list(an)) for c, cr, an in self._t]

    def canonical_order(self):
        for t in self._t:
            t[1], s1 = _canon(t[1])
            t[2], s2 = _canon(t[2])
            if s1 < 0:
                t[0] = complex(-t[0].real, -t[0].imag)
            if s2 < 0:
                t[0] = complex(-t[0].real, -t[0].imag)

    def simplify(self):
        """sq_operator.cc:154-173: canonical order, combine, sort, drop |c| <= 1e-12."""
        self.canonical_order()
        acc = {}
        for c, cr, an in self._t:
            k = (tuple(cr), tuple(an))
            if k in acc:
                acc[k] += c
            else:
                acc[k] = c
        self._t = [[c, list(k[0]), list(k[1])] for k, c in sorted(acc.items())
                   if abs(c) > 1.0e-12]

    def _jw_masks(self, qubit_excitation=False):
        """[(c, x, z)] of the transformed operator (after the final simplify)."""
        self.simplify()
        out = []
        for c, cr, an in self._t:
            if not cr and not an:
                out.append((c, 0, 0))
                continue
            for hc, x, z in _jw_image(tuple(cr), tuple(an), bool(qubit_excitation)):
                out.append((hc * c, x, z))
        return _simplify_masks(out)

    def jw_transform(self, qubit_excitation=False):
        qo = QubitOperator()
        qo._t = [[c, Circuit._from_masks(x, z)] for c, x, z in self._jw_masks(qubit_excitation)]
        return qo

    def str(self):
        parts = [""]
        for c, cr, an in self._t:
            parts.append(to_string(c))
            parts.append("(")
            parts.extend(f"{k}^" for k in cr)
            parts.extend(str(k) for k in an)
            parts.append(")\n")
        return " ".join(parts)

    __str__ = str
    __repr__ = str
