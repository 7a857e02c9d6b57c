"""Pauli strings in mask form and their exact products.

A canonical Pauli circuit (one X, Y or Z per qubit, sorted by qubit -- what
``Circuit::canonicalize_pauli_circuit`` produces, circuit.cc:107-169) is held
as two integers: ``x`` (qubits carrying X or Y) and ``z`` (qubits carrying Z
or Y).  Products are computed symplectically; the phase is a power of i, so
multiplying a coefficient by it is exact, as the reference's table lookups
(circuit.cc:120-132) are.
"""

__all__ = ["pauli_mul", "ipow_mul", "canonical_key", "letters", "masks_of_letters"]


def _pc(v):
    return bin(v).count("1")


def pauli_mul(x1, z1, x2, z2):
    """(x1,z1) . (x2,z2) = i^e (x1^x2, z1^z2); returns (x, z, e mod 4).

    With P(x,z) = i^{x.z} X^x Z^z per qubit, the product picks up
    i^{x1 z1 + x2 z2 - x3 z3} (-1)^{z1 x2}.
    """
    x3, z3 = x1 ^ x2, z1 ^ z2
    e = _pc(x1 & z1) + _pc(x2 & z2) - _pc(x3 & z3) + 2 * _pc(z1 & x2)
    return x3, z3, e & 3


def ipow_mul(c, e):
    """c * i^e, exactly (component swaps and sign flips only)."""
    e &= 3
    if e == 0:
        return c
    if e == 1:
        return complex(-c.imag, c.real)
    if e == 2:
        return complex(-c.real, -c.imag)
    return complex(c.imag, -c.real)


_LETTER = {1: "X", 3: "Y", 2: "Z"}  # (x bit) | (z bit << 1)


def letters(x, z):
    """[(letter, qubit), ...] in ascending qubit order."""
    out = []
    m = x | z
    q = 0
    while m:
        if m & 1:
            out.append((_LETTER[((x >> q) & 1) | (((z >> q) & 1) << 1)], q))
        m >>= 1
        q += 1
    return out


def canonical_key(x, z):
    """Sort key equal to the reference's Circuit ordering (circuit.cc:346,
    gate.cc:203-219) on canonical Pauli circuits: lexicographic over gates,
    each gate compared by (gate_id, target, control)."""
    return tuple((l, q, q) for l, q in letters(x, z))


def masks_of_letters(seq):
    """Left-to-right product of [(letter, qubit), ...]: returns (x, z, e)."""
    x = z = e = 0
    for l, q in seq:
        b = 1 << q
        if l == "X":
            x2, z2 = b, 0
        elif l == "Y":
            x2, z2 = b, b
        elif l == "Z":
            x2, z2 = 0, b
        else:
            raise ValueError(f"not a Pauli letter: {l}")
        x, z, de = pauli_mul(x, z, x2, z2)
        e += de
    return x, z, e & 3
