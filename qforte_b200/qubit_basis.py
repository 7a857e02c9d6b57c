"""``QubitBasis``: a computational basis state as a 64-bit integer.

qubit_basis.h:15-58 / qubit_basis.cc:3-15: qubit k is bit k of the index
(LSB = qubit 0); ``str(n)`` prints qubit 0 first.
"""

__all__ = ["QubitBasis"]

_MASK64 = (1 << 64) - 1


class QubitBasis:
    __slots__ = ("_s",)
    max_qubits = 64

    def __init__(self, n=0):
        self._s = int(n) & _MASK64

    @staticmethod
    def maskbit(pos):
        return (1 << pos) & _MASK64

    def get_bit(self, pos):
        return bool(self._s & (1 << pos))

    def set_bit(self, pos, val):
        if val:
            self._s |= 1 << pos
        else:
            self._s &= ~(1 << pos) & _MASK64

    def flip_bit(self, pos):
        self._s ^= 1 << pos

    def set(self, state):
        self._s = int(state) & _MASK64

    def zero(self):
        self._s = 0

    def index(self):
        return self._s

    def get_state(self):
        return self._s

    def str(self, nqubit):
        return "|" + "".join("1" if (self._s >> i) & 1 else "0" for i in range(nqubit)) + ">"

    def default_str(self):
        return self.str(64)

    __str__ = default_str
    __repr__ = default_str

    def __eq__(self, other):
        return isinstance(other, QubitBasis) and self._s == other._s

    def __hash__(self):
        return hash(self._s)
