"""Seeded synthetic workloads with the shapes of the reference's measured
cases.

``layered_random_circuit`` is the gate-application sweep: every layer applies
a uniformly random gate from {H, X, Y, Z, S, T, Rx, Ry, Rz} (angles U(0, 2 pi))
to every qubit, then a uniformly random gate from {cX, cZ, SWAP, cR} (angle
U(0, 2 pi)) to each pair of a random perfect matching of the qubits (one
qubit idles when n is odd), starting from |0...0>.
"""

import math

import numpy as np

from .circuit import Circuit
from .gate import gate

ONE_QUBIT = ("H", "X", "Y", "Z", "S", "T", "Rx", "Ry", "Rz")
TWO_QUBIT = ("cX", "cZ", "SWAP", "cR")

__all__ = ["layered_random_circuit", "ONE_QUBIT", "TWO_QUBIT"]


def layered_random_circuit(nqubit, layers, seed):
    """(Circuit, [(kind, target, control, parameter), ...]) of the sweep."""
    rng = np.random.default_rng(seed)
    spec = []
    for _ in range(layers):
        for q in range(nqubit):
            k = ONE_QUBIT[rng.integers(len(ONE_QUBIT))]
            spec.append((k, q, q, float(rng.uniform(0.0, 2.0 * math.pi))))
        perm = rng.permutation(nqubit)
        for i in range(0, nqubit - 1, 2):
            k = TWO_QUBIT[rng.integers(len(TWO_QUBIT))]
            spec.append((k, int(perm[i]), int(perm[i + 1]), float(rng.uniform(0.0, 2.0 * math.pi))))
    circ = Circuit()
    for k, t, c, p in spec:
        circ.add(gate(k, t, c, p))
    return circ, spec
