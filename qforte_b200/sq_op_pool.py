"""``SQOpPool``: UCC excitation pools (sq_op_pool.h:16-73, sq_op_pool.cc:1-595).

The pools are built in the reference's order, which matters: a disentangled
UCC ansatz is a Trotter product, and its factors do not commute across
excitations.

* ``GSD``: generalised spin-conserving singles and doubles, de-duplicated
  against earlier terms and their adjoints (sq_op_pool.cc:112-323).
* ``S`` ... ``SDTQPH``: particle-hole excitations of the reference
  determinant up to rank 1..6, enumerated from the N- and Sz-preserving
  determinants in ascending integer order (sq_op_pool.cc:324-432; the
  alpha/beta strings are generated with next_permutation from the reference
  occupation, as there).
* ``sa_SD``: spin-adapted singles and doubles (sq_op_pool.cc:433-575).
"""

import math

from .qubit_operator import QubitOperator, to_string
from .sq_operator import SQOperator

__all__ = ["SQOpPool", "QubitOpPool", "find_irrep"]


def find_irrep(orb_irreps_to_int, spinorb_indices):
    """find_irrep.cc:3-12: XOR of the spatial-orbital irreps."""
    irrep = 0
    for idx in spinorb_indices:
        irrep ^= int(orb_irreps_to_int[idx // 2])
    return irrep


def _next_permutation(a):
    """std::next_permutation on a list in place; False when it wrapped."""
    i = len(a) - 2
    while i >= 0 and not (a[i] < a[i + 1]):
        i -= 1
    if i < 0:
        a.reverse()
        return False
    j = len(a) - 1
    while not (a[i] < a[j]):
        j -= 1
    a[i], a[j] = a[j], a[i]
    a[i + 1:] = reversed(a[i + 1:])
    return True


class SQOpPool:
    def __init__(self):
        self._t = []  # [coeff, SQOperator]
        self._ref_int = 0
        self._nso = 0
        self._nocc_a = self._nocc_b = self._nvir_a = self._nvir_b = 0
        self._irreps = []

    def add(self, coeff, sq_op):
        self.add_term(coeff, sq_op)

    def add_term(self, coeff, sq_op):
        self._t.append([complex(coeff), sq_op])

    def set_coeffs(self, new_coeffs):
        if len(new_coeffs) != len(self._t):
            raise ValueError("Number of new coefficients for quantum operator must equal.")
        for t, c in zip(self._t, new_coeffs):
            t[0] = complex(c)

    def terms(self):
        return [(c, op) for c, op in self._t]

    def __getitem__(self, i):
        c, op = self._t[i]
        return (c, op)

    def __iter__(self):
        return iter(self.terms())

    def __len__(self):
        return len(self._t)

    def set_orb_spaces(self, ref, orb_irreps_to_int=None):
        """sq_op_pool.cc:32-71."""
        self._ref_int = 0
        mult = 1
        for occ in ref:
            self._ref_int += int(occ) * mult
            mult <<= 1
        self._nso = len(ref)
        if self._nso % 2 != 0:
            raise ValueError("The total number of spinorbitals must be even!")
        self._nocc_a = self._nocc_b = self._nvir_a = self._nvir_b = 0
        alpha = True
        for occ in ref:
            occ = int(occ)
            if alpha:
                self._nocc_a += occ
                self._nvir_a += occ ^ 1
            else:
                self._nocc_b += occ
                self._nvir_b += occ ^ 1
            alpha = not alpha
        if not orb_irreps_to_int:
            self._irreps = [0] * (self._nso // 2)
        else:
            self._irreps = [int(v) for v in orb_irreps_to_int]

    def get_qubit_op_pool(self):
        A = QubitOpPool()
        for c, op in self._t:
            A.add_term(c, op.jw_transform())
        return A

    def get_qubit_operator(self, order_type, combine_like_terms=True, qubit_excitations=False):
        """sq_op_pool.cc:83-109."""
        parent = QubitOperator()
        if order_type == "unique_lex":
            for c, op in self._t:
                child = op.jw_transform(qubit_excitations)
                child.mult_coeffs(c)
                parent.add_op(child)
            parent.simplify()
            parent.order_terms()
        elif order_type == "commuting_grp_lex":
            for c, op in self._t:
                child = op.jw_transform(qubit_excitations)
                child.mult_coeffs(c)
                child.simplify(combine_like_terms)
                child.order_terms()
                parent.add_op(child)
        else:
            raise ValueError("Invalid order_type specified.")
        return parent

    # ------------------------------------------------------------------
    def fill_pool(self, pool_type):
        if pool_type == "GSD":
            self._fill_gsd()
        elif pool_type in ("S", "SD", "SDT", "SDTQ", "SDTQP", "SDTQPH"):
            self._fill_particle_hole(len(pool_type) if pool_type != "S" else 1)
        elif pool_type == "sa_SD":
            self._fill_sa_sd()
        else:
            raise ValueError("Invalid pool_type specified.")

    def _fill_gsd(self):
        norb = self._nso // 2
        irr = self._irreps
        for i in range(norb):
            ia, ib = 2 * i, 2 * i + 1
            for a in range(i, norb):
                aa, ab = 2 * a, 2 * a + 1
                if not find_irrep(irr, [ia, aa]):
                    if aa != ia:
                        t = SQOperator()
                        t.add_term(+1.0, [aa], [ia])
                        t.add_term(-1.0, [ia], [aa])
                        t.simplify()
                        if t._t:
                            self.add_term(1.0, t)
                    if ab != ib:
                        t = SQOperator()
                        t.add_term(+1.0, [ab], [ib])
                        t.add_term(-1.0, [ib], [ab])
                        t.simplify()
                        if t._t:
                            self.add_term(1.0, t)
        uniqe, adjnt = [], []
        seen_u, seen_a = set(), set()
        for i in range(norb):
            ia, ib = 2 * i, 2 * i + 1
            for j in range(i, norb):
                ja, jb = 2 * j, 2 * j + 1
                for a in range(norb):
                    aa, ab = 2 * a, 2 * a + 1
                    for b in range(a, norb):
                        ba, bb = 2 * b, 2 * b + 1
                        if find_irrep(irr, [ia, ja, aa, ba]):
                            continue
                        # (cre, ann) of the six spin blocks, in the reference's order
                        blocks = (
                            ((aa, ba), (ia, ja), aa != ba and ia != ja),
                            ((ab, bb), (ib, jb), ab != bb and ib != jb),
                            ((aa, bb), (ia, jb), aa != bb and ia != jb),
                            ((ab, ba), (ib, ja), ab != ba and ib != ja),
                            ((aa, bb), (ib, ja), aa != bb and ib != ja),
                            ((ab, ba), (ia, jb), ab != ba and ia != jb),
                        )
                        for (c0, c1), (a0, a1), ok in blocks:
                            if not ok:
                                continue
                            t = SQOperator()
                            t.add_term(+1.0, [c0, c1], [a0, a1])
                            t.add_term(-1.0, [a1, a0], [c1, c0])
                            t.simplify()
                            if not t._t:
                                continue
                            t0, t1 = t._t[0], t._t[1]
                            vtemp = (t0[1][0], t0[1][1], t0[2][0], t0[2][1])
                            vadjt = (t1[1][0], t1[1][1], t1[2][0], t1[2][1])
                            if vtemp not in seen_u and vtemp not in seen_a:
                                uniqe.append(vtemp)
                                adjnt.append(vadjt)
                                seen_u.add(vtemp)
                                seen_a.add(vadjt)
                                self.add_term(1.0, t)

    def _fill_particle_hole(self, max_nbody):
        n = self._nso
        ref_bin = format(self._ref_int, "064b")[64 - n:]
        alpha = [ref_bin[i] for i in range(n) if i % 2 == 1]
        beta = [ref_bin[i] for i in range(n) if i % 2 == 0]
        alpha_perms, beta_perms = [], []
        a = list(alpha)
        while True:
            alpha_perms.append(list(a))
            if not _next_permutation(a):
                break
        b = list(beta)
        while True:
            beta_perms.append(list(b))
            if not _next_permutation(b):
                break
        dets = []
        for sa in alpha_perms:
            for sb in beta_perms:
                s = "".join(sb[i] + sa[i] for i in range(len(sa)))
                dets.append(int(s, 2) if s else 0)
        dets.sort()
        for det in dets:
            excit = format(self._ref_int ^ det, "064b")[64 - n:]
            nex = excit.count("1")
            if nex % 2 != 0:
                raise ValueError("The number of excitation indices must be an even number!")
            rank = nex // 2
            if rank == 0 or rank > max_nbody:
                continue
            occ_idx, unocc_idx = [], []
            for i, ch in enumerate(excit):
                if ch != "1":
                    continue
                if ref_bin[i] == "1":
                    occ_idx.append(n - i - 1)
                else:
                    unocc_idx.append(n - i - 1)
            if find_irrep(self._irreps, occ_idx + unocc_idx):
                continue
            t = SQOperator()
            t.add_term(+1.0, unocc_idx, occ_idx)
            t.add_term(-1.0, occ_idx[::-1], unocc_idx[::-1])
            t.simplify()
            self.add_term(1.0, t)

    def _fill_sa_sd(self):
        if self._nocc_a != self._nocc_b:
            raise ValueError("sa_SD operator pool requires a closed-shell reference determinant!")
        nocc, nvir = self._nocc_a, self._nvir_a
        irr = self._irreps
        r2 = 1.0 / math.sqrt(2)
        for i in range(nocc):
            ia, ib = 2 * i, 2 * i + 1
            for a in range(nvir):
                aa, ab = 2 * nocc + 2 * a, 2 * nocc + 2 * a + 1
                if not find_irrep(irr, [ia, aa]):
                    t = SQOperator()
                    t.add_term(+r2, [aa], [ia])
                    t.add_term(+r2, [ab], [ib])
                    t.add_term(-r2, [ia], [aa])
                    t.add_term(-r2, [ib], [ab])
                    t.simplify()
                    self.add_term(1.0, t)
        s12 = math.sqrt(12)
        for i in range(nocc):
            ia, ib = 2 * i, 2 * i + 1
            for j in range(i, nocc):
                ja, jb = 2 * j, 2 * j + 1
                for a in range(nvir):
                    aa, ab = 2 * nocc + 2 * a, 2 * nocc + 2 * a + 1
                    for b in range(a, nvir):
                        ba, bb = 2 * nocc + 2 * b, 2 * nocc + 2 * b + 1
                        if find_irrep(irr, [ia, ja, aa, ba]):
                            continue
                        t2a = SQOperator()
                        if aa != ba and ia != ja:
                            t2a.add_term(2.0 / s12, [aa, ba], [ia, ja])
                        if ab != bb and ib != jb:
                            t2a.add_term(2.0 / s12, [ab, bb], [ib, jb])
                        if aa != bb and ia != jb:
                            t2a.add_term(1.0 / s12, [aa, bb], [ia, jb])
                        if ab != ba and ib != ja:
                            t2a.add_term(1.0 / s12, [ab, ba], [ib, ja])
                        if aa != bb and ib != ja:
                            t2a.add_term(1.0 / s12, [aa, bb], [ib, ja])
                        if ab != ba and ia != jb:
                            t2a.add_term(1.0 / s12, [ab, ba], [ia, jb])
                        if ja != ia and ba != aa:
                            t2a.add_term(-2.0 / s12, [ja, ia], [ba, aa])
                        if jb != ib and bb != ab:
                            t2a.add_term(-2.0 / s12, [jb, ib], [bb, ab])
                        if jb != ia and bb != aa:
                            t2a.add_term(-1.0 / s12, [jb, ia], [bb, aa])
                        if ja != ib and ba != ab:
                            t2a.add_term(-1.0 / s12, [ja, ib], [ba, ab])
                        if ja != ib and bb != aa:
                            t2a.add_term(-1.0 / s12, [ja, ib], [bb, aa])
                        if jb != ia and ba != ab:
                            t2a.add_term(-1.0 / s12, [jb, ia], [ba, ab])
                        t2b = SQOperator()
                        if aa != bb and ia != jb:
                            t2b.add_term(0.5, [aa, bb], [ia, jb])
                        if ab != ba and ib != ja:
                            t2b.add_term(0.5, [ab, ba], [ib, ja])
                        if aa != bb and ib != ja:
                            t2b.add_term(-0.5, [aa, bb], [ib, ja])
                        if ab != ba and ia != jb:
                            t2b.add_term(-0.5, [ab, ba], [ia, jb])
                        if jb != ia and bb != aa:
                            t2b.add_term(-0.5, [jb, ia], [bb, aa])
                        if ja != ib and ba != ab:
                            t2b.add_term(-0.5, [ja, ib], [ba, ab])
                        if ja != ib and bb != aa:
                            t2b.add_term(0.5, [ja, ib], [bb, aa])
                        if jb != ia and ba != ab:
                            t2b.add_term(0.5, [jb, ia], [ba, ab])
                        t2a.simplify()
                        t2b.simplify()
                        na = complex(0.0)
                        nb = complex(0.0)
                        for c, _, _ in t2a._t:
                            na += abs(c) ** 2
                        for c, _, _ in t2b._t:
                            nb += abs(c) ** 2
                        if t2a._t:
                            t2a.mult_coeffs(_csqrt(2.0 / na))
                        if t2b._t:
                            t2b.mult_coeffs(_csqrt(2.0 / nb))
                        if t2a._t:
                            self.add_term(1.0, t2a)
                        if t2b._t:
                            self.add_term(1.0, t2b)

    def str(self):
        s = [""]
        for k, (c, op) in enumerate(self._t):
            s += ["----->", str(k), "<-----\n", to_string(c), "[\n", op.str(), "]\n\n"]
        return " ".join(s)

    __str__ = str
    __repr__ = str


def _csqrt(v):
    import cmath
    return cmath.sqrt(complex(v))


class QubitOpPool:
    """A list of (coefficient, QubitOperator) (qubit_op_pool.h:12-69)."""

    def __init__(self):
        self._t = []

    def add(self, coeff, op):
        self.add_term(coeff, op)

    def add_term(self, coeff, op):
        self._t.append([complex(coeff), op])

    def set_coeffs(self, new_coeffs):
        if len(new_coeffs) != len(self._t):
            raise ValueError(
                "Number of new coefficients for quantum op pool must equal number of terms in "
                "pool.")
        for t, c in zip(self._t, new_coeffs):
            t[0] = complex(c)

    def set_op_coeffs(self, new_coeffs):
        for _, op in self._t:
            if len(new_coeffs) != len(op._t):
                raise ValueError("Number of new coeficients for quantum operator must equal "
                                 "number of terim in operator.")
            op.set_coeffs(new_coeffs)

    def set_terms(self, new_terms):
        for c, op in new_terms:
            self._t.append([complex(c), op])

    def terms(self):
        return [(c, op) for c, op in self._t]

    def __iter__(self):
        return iter(self.terms())

    def __len__(self):
        return len(self._t)

    def __getitem__(self, i):
        c, op = self._t[i]
        return (c, op)

    def join_op_from_right_lazy(self, q_op):
        for _, op in self._t:
            op.operator_product(q_op, False, False)

    def join_op_from_right(self, q_op):
        for _, op in self._t:
            op.operator_product(q_op, False)
            op.simplify()

    def join_op_from_left(self, q_op):
        out = []
        for c, op in self._t:
            t = QubitOperator()
            t.add_op(q_op)
            t.operator_product(op, False)
            t.simplify()
            out.append([c, t])
        self._t = out

    def join_as_commutator(self, q_op):
        """term -> [q_op, term] (qubit_op_pool.cc:174-193)."""
        out = []
        for c, op in self._t:
            ham = QubitOperator()
            ham.add_op(q_op)
            ham.operator_product(op, False)
            amh = QubitOperator()
            amh.add_op(op)
            amh.operator_product(q_op, False)
            amh.mult_coeffs(-1.0)
            ham.add_op(amh)
            ham.simplify()
            out.append([c, ham])
        self._t = out

    def square(self, upper_triangle_only):
        out = []
        n = len(self._t)
        for I in range(n):
            for J in (range(I, n) if upper_triangle_only else range(n)):
                t = QubitOperator()
                t.add_op(self._t[I][1])
                t.operator_product(self._t[J][1], False)
                t.simplify()
                out.append([self._t[I][0].conjugate() * self._t[J][0], t])
        self._t = out

    def fill_pool(self, pool_type, nqb):
        """complete_qubit / cqoy (qubit_op_pool.cc:195-246)."""
        from .circuit import Circuit
        from .gate import make_gate
        if pool_type not in ("complete_qubit", "cqoy"):
            raise ValueError("Invalid pool_type specified.")
        names = {1: "X", 2: "Y", 3: "Z"}
        for I in range(4 ** nqb):
            digits = []
            v = I
            for _ in range(nqb):
                digits.append(v % 4)
                v //= 4
            digits.reverse()  # most significant first, as pauli_idx_str pads
            circ = Circuit()
            ny = 0
            for k, d in enumerate(digits):
                if d == 2:
                    ny += 1
                if d != 0:
                    circ.add_gate(make_gate(names[d], k, k))
            if pool_type == "cqoy" and ny % 2 == 0:
                continue
            op = QubitOperator()
            op.add_term(1.0, circ)
            self.add_term(1.0, op)

    def str(self):
        s = [""]
        for k, (c, op) in enumerate(self._t):
            s += ["----->", str(k), "<-----\n", to_string(c), "[\n", op.str(), "\n", "]\n\n"]
        return " ".join(s)

    __str__ = str
    __repr__ = str
