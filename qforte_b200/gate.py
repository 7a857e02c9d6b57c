"""Gates: the 4x4 complex matrix model of QForte's ``Gate`` and ``make_gate``.

Restates ``src/qforte/gate.h:19-154``, ``gate.cc:12-236`` and
``make_gate.cc:7-256``: the same gate set, the same matrices, the same angle
normalisation and the same adjoint rules, so circuits built here act on a
state exactly as the reference's do.  1-qubit gates use the top-left 2x2
block; 2-qubit matrix indices are ``(control_bit << 1) | target_bit``.
"""

import cmath
import math

import numpy as np

__all__ = ["Gate", "make_gate", "gate", "control_gate", "normalize_angle", "ONE_QUBIT_GATES",
           "TWO_QUBIT_GATES"]

ONE_QUBIT_GATES = ("X", "Y", "Z", "H", "R", "Rx", "Ry", "Rz", "V", "S", "T", "I")
TWO_QUBIT_GATES = ("A", "cX", "CNOT", "acX", "aCNOT", "cY", "cZ", "cR", "cV", "cRz", "SWAP")

# GateType names by label (gate.cc:221-236); unknown labels map to "Undefined".
_LABEL_TO_TYPE = {
    "X": "X", "Y": "Y", "Z": "Z", "H": "H", "R": "R", "Rx": "Rx", "Ry": "Ry", "Rz": "Rz",
    "V": "V", "S": "S", "T": "T", "I": "I", "A": "A", "CNOT": "cX", "cX": "cX",
    "aCNOT": "acX", "acX": "acX", "cY": "cY", "cZ": "cZ", "cR": "cR", "cV": "cV",
    "cRz": "cRz", "SWAP": "SWAP", "adj(V)": "adjV", "adj(cV)": "adjcV",
}


def normalize_angle(angle, period):
    """Fold ``angle`` into [-period/2, period/2] as make_gate.cc:7-16 does."""
    angle = math.fmod(angle, period)
    if angle < -period / 2:
        angle += period
    elif angle > period / 2:
        angle -= period
    return angle


class Gate:
    """A 1- or 2-qubit gate: label, target, control, 4x4 matrix, optional parameter.

    ``parameter`` is ``None`` or ``(value, minus_on_adjoint)`` (gate.h:126-128).
    """

    __slots__ = ("_label", "_target", "_control", "_mat", "_param")

    def __init__(self, label, target, control, matrix, parameter=None):
        self._label = str(label)
        self._target = int(target)
        self._control = int(control)
        self._mat = matrix
        self._param = parameter

    # -- accessors (bindings.cc:193-218) --
    def gate_id(self):
        return self._label

    def gate_type(self):
        return _LABEL_TO_TYPE.get(self._label, "Undefined")

    def target(self):
        return self._target

    def control(self):
        return self._control

    def matrix(self):
        return self._mat

    def nqubits(self):
        return 1 if self._target == self._control else 2

    def has_parameter(self):
        return self._param is not None

    def parameter(self):
        return None if self._param is None else self._param[0]

    def minus_parameter_on_adjoint(self):
        return False if self._param is None else bool(self._param[1])

    def update_parameter(self, parameter):
        if not self.has_parameter():
            raise ValueError("Gate does not have a parameter.")
        return make_gate(self._label, self._target, self._control, parameter)

    def adjoint(self):
        """gate.cc:135-179."""
        adj = self._mat.conj().T.copy()
        self_adjoint = bool(np.all(np.abs(adj - self._mat) ** 2 <= 1.0e-12))
        if self._param is not None:
            v, minus = self._param
            return Gate(self._label, self._target, self._control, adj,
                        (v * (1.0 - 2.0 * float(bool(minus))), minus))
        if self_adjoint:
            return self
        t = self.gate_type()
        if t == "T":
            return Gate("R", self._target, self._control, adj, (-math.pi / 4, True))
        if t == "S":
            return Gate("R", self._target, self._control, adj, (-math.pi / 2, True))
        lab = self._label
        if len(lab) > 4 and lab.startswith("adj(") and lab.endswith(")"):
            return Gate(lab[4:-1], self._target, self._control, adj, self._param)
        return Gate("adj(" + lab + ")", self._target, self._control, adj, self._param)

    # -- printing --
    def str(self):
        if self._target == self._control:
            return f"{self._label}{self._target}"
        return f"{self._label}{self._target}_{self._control}"

    __str__ = str

    def __repr__(self):
        s = f"{self._label} gate, target qubit:{self._target}, contol qubit:{self._control}\n"
        idx = range(2) if self.nqubits() == 1 else range(4)
        for i in idx:
            for j in idx:
                v = self._mat[i, j]
                s += f"  {v.real:+f} {v.imag:+f} i"
            s += "\n"
        return s

    # -- comparisons (gate.cc:183-219) --
    def _key(self):
        return (self._label, self._target, self._control)

    def __eq__(self, other):
        if not isinstance(other, Gate):
            return NotImplemented
        if self._key() != other._key():
            return False
        if self._param is not None and other._param is not None:
            return abs(self._param[0] - other._param[0]) < 1.0e-12
        return True

    def __ne__(self, other):
        r = self.__eq__(other)
        return r if r is NotImplemented else not r

    __neq__ = __ne__

    def __lt__(self, other):
        a, b = self._key(), other._key()
        if a != b:
            return a < b
        if self._param is not None and other._param is not None:
            return self._param[0] < other._param[0]
        return False

    __hash__ = None


def make_gate(kind, target, control, parameter=0.0):
    """make_gate.cc:18-235."""
    target = int(target)
    control = int(control)
    p = float(parameter)
    j = 1j
    m = np.zeros((4, 4), dtype=np.complex128)
    if target == control:
        par = None
        if kind == "X":
            m[0, 1] = m[1, 0] = 1.0
        elif kind == "Y":
            m[0, 1], m[1, 0] = -j, j
        elif kind == "Z":
            m[0, 0], m[1, 1] = 1.0, -1.0
        elif kind == "H":
            c = 1.0 / math.sqrt(2.0)
            m[0, 0] = m[0, 1] = m[1, 0] = c
            m[1, 1] = -c
        elif kind == "R":
            p = normalize_angle(p, 2 * math.pi)
            m[0, 0], m[1, 1] = 1.0, cmath.exp(j * p)
            par = (p, True)
        elif kind == "Rx":
            p = normalize_angle(p, 4 * math.pi)
            a, b = math.cos(0.5 * p), j * math.sin(0.5 * p)
            m[0, 0], m[0, 1], m[1, 0], m[1, 1] = a, -b, -b, a
            par = (p, True)
        elif kind == "Ry":
            p = normalize_angle(p, 4 * math.pi)
            a, b = math.cos(0.5 * p), math.sin(0.5 * p)
            m[0, 0], m[0, 1], m[1, 0], m[1, 1] = a, -b, b, a
            par = (p, True)
        elif kind == "Rz":
            p = normalize_angle(p, 4 * math.pi)
            m[0, 0], m[1, 1] = cmath.exp(-j * 0.5 * p), cmath.exp(j * 0.5 * p)
            par = (p, True)
        elif kind == "V":
            a, b = 0.5 + 0.5j, 0.5 - 0.5j
            m[0, 0], m[0, 1], m[1, 0], m[1, 1] = a, b, b, a
        elif kind == "S":
            m[0, 0], m[1, 1] = 1.0, j
        elif kind == "T":
            m[0, 0], m[1, 1] = 1.0, (1.0 + j) / math.sqrt(2.0)
        elif kind == "I":
            m[0, 0] = m[1, 1] = 1.0
        else:
            raise ValueError(f"make_gate()\ntype = {kind} is not a valid quantum gate type")
        return Gate(kind, target, control, m, par)
    m[0, 0] = m[1, 1] = m[2, 2] = m[3, 3] = 1.0
    par = None
    if kind == "A":
        p = normalize_angle(p, 2 * math.pi)
        c, s = math.cos(p), math.sin(p)
        m[1, 1], m[1, 2], m[2, 1], m[2, 2] = c, s, s, -c
        par = (p, False)
    elif kind in ("cX", "CNOT"):
        m[2, 2] = m[3, 3] = 0.0
        m[2, 3] = m[3, 2] = 1.0
    elif kind in ("acX", "aCNOT"):
        m[0, 0] = m[1, 1] = 0.0
        m[0, 1] = m[1, 0] = 1.0
    elif kind == "cY":
        m[2, 2] = m[3, 3] = 0.0
        m[2, 3], m[3, 2] = -j, j
    elif kind == "cZ":
        m[3, 3] = -1.0
    elif kind == "cR":
        p = normalize_angle(p, 2 * math.pi)
        m[3, 3] = cmath.exp(j * p)
        par = (p, True)
    elif kind == "cV":
        a, b = 0.5 + 0.5j, 0.5 - 0.5j
        m[2, 2], m[2, 3], m[3, 2], m[3, 3] = a, b, b, a
    elif kind == "cRz":
        p = normalize_angle(p, 4 * math.pi)
        m[2, 2], m[3, 3] = cmath.exp(-j * 0.5 * p), cmath.exp(j * 0.5 * p)
        par = (p, True)
    elif kind == "SWAP":
        m[1, 1] = m[2, 2] = 0.0
        m[1, 2] = m[2, 1] = 1.0
    else:
        raise ValueError(f"make_gate()\ntype = {kind} is not a valid quantum gate type")
    return Gate(kind, target, control, m, par)


def _real_param(parameter):
    c = complex(parameter)
    if c.imag != 0.0:
        raise ValueError("Gate parameter must be real.")
    return c.real


_ONE_Q_PARAM_OK = ("X", "Y", "Z", "H", "R", "Rx", "Ry", "Rz", "V", "S", "T", "I")
_TWO_Q_NOPARAM = ("SWAP", "cV", "CNOT", "cX", "aCNOT", "acX", "cY", "cZ")
_ONE_Q_NOPARAM = ("X", "Y", "Z", "H", "V", "S", "T", "I")


def _is_index(v):
    return not isinstance(v, (float, complex)) and hasattr(type(v), "__index__")


def gate(type, target, *args, **kwargs):
    """The module-level ``gate`` factory with the three pybind overloads
    (bindings.cc:238-290), resolved the way pybind11 resolves them (an
    integer third argument selects the ``control`` overloads):

    * ``gate(type, target, parameter=0.0)``          1-qubit gates
    * ``gate(type, target, control)``                parameter-free gates only
    * ``gate(type, target, control, parameter=0.0)`` any gate
    """
    nargs = len(args)
    if nargs > 2:
        raise TypeError("gate() takes at most 4 positional arguments")
    if "control" in kwargs or nargs == 2 or (nargs == 1 and _is_index(args[0])
                                             and "parameter" not in kwargs):
        control = args[0] if nargs >= 1 else kwargs.pop("control")
        if nargs == 2 or "parameter" in kwargs:
            parameter = args[1] if nargs == 2 else kwargs.pop("parameter")
            return make_gate(type, target, control, _real_param(parameter))
        if type in _TWO_Q_NOPARAM:
            return make_gate(type, target, control, 0.0)
        if int(target) == int(control) and type in _ONE_Q_NOPARAM:
            return make_gate(type, target, control, 0.0)
        raise ValueError(
            f"make_gate()\ttarget = {target}, control = {control}, is not a valid quantum gate "
            f"input for type = {type}")
    parameter = args[0] if nargs == 1 else kwargs.pop("parameter", 0.0)
    p = _real_param(parameter)
    if type in _ONE_Q_PARAM_OK:
        return make_gate(type, target, target, p)
    raise ValueError(
        f"make_gate()\ttarget = {target}, parameter = {p} is not a valid quantum gate input "
        f"for type = {type}")


def control_gate(control, U):
    """make_control_gate (make_gate.cc:237-256)."""
    if U.target() == control:
        raise ValueError("Cannot create Control-U where targer == control !")
    m = np.zeros((4, 4), dtype=np.complex128)
    m[0, 0] = m[1, 1] = 1.0
    u = U.matrix()
    m[2, 2], m[2, 3], m[3, 2], m[3, 3] = u[0, 0], u[0, 1], u[1, 0], u[1, 1]
    par = (U.parameter(), U.minus_parameter_on_adjoint()) if U.has_parameter() else None
    return Gate("cU", U.target(), control, m, par)
