"""qforte_b200: QForte's state-vector hot path, B200-native.

A drop-in for the ``qforte`` objects that drive the state-vector engine --
``Computer``, ``Gate``/``gate``, ``Circuit``, ``QubitOperator``,
``SQOperator``, ``SQOpPool``, ``QubitOpPool``, ``QubitBasis`` and the compile
helpers -- with the amplitudes held in HBM and every operation a
hand-written sm_100a kernel in libqfb.so (C ABI: include/qfb.h).  The
algorithm drivers that run on it keep the reference's names: ``UCCNVQE``,
``ADAPTVQE``, ``UCCNPQE``, ``SPQE``, ``QITE``, ``SRQK``, ``NTSRQK``, ``MRSQK``.
"""

from .gate import Gate, control_gate, gate, make_gate, normalize_angle
from .circuit import Circuit
from .qubit_operator import QubitOperator
from .sq_operator import SQOperator
from .sq_op_pool import QubitOpPool, SQOpPool, find_irrep
from .qubit_basis import QubitBasis
from .computer import (Computer, ComputerC64, add_gate_to_computer, inner_product,
                       prepare_computer_from_circuit, prepare_computer_from_gates)
from .utils import (build_circuit, build_operator, build_refprep, compact_excitation_circuit,
                    exponentiate_pauli_string, integer_to_ref, local_timer, ref_string, smart_print,
                    trotterize, trotterize_w_cRz)
from .systems import Molecule, create_external_mol, random_molecule, system_factory
from .ucc import ADAPTVQE, SPQE, UCCNPQE, UCCNVQE
from .qite import QITE
from .krylov import MRSQK, NTSRQK, SRQK

__version__ = "0.1.0"
