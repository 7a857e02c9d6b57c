"""The reference's own drivers' engine calls, replayed on the oracle.

tests/golden/dropin_trace_*.npz record every Computer call the reference's
UCCNVQE (He/cc-pVDZ, its tests/test_uccsd.py:13-29) and ADAPTVQE (H4/STO-6G,
SDTQ pool, its tests/test_adapt_vqe.py:12-40) made on the reference's compiled
Computer, with its results.  Replayed call for call on the oracle's host state
with this package's Gate, Circuit and QubitOperator, every result must equal
the reference's (energies and expectation values 1e-12, state projections
1e-12), and the last energy the reference's FCI value within the tolerance its
test states.  The same traces run on the device Computer in
test_gpu_dropin_replay.py.
"""

import collections

import numpy as np
import pytest

from dropin_trace import replay
from test_dropin_reference_drivers import DropinComputer
from tests.conftest import golden

TOL = 1e-12


@pytest.mark.parametrize("name", ["uccnvqe_he", "adaptvqe_h4"])
def test_reference_driver_trace_on_the_oracle(name):
    z = golden(f"dropin_trace_{name}.npz")
    err = collections.defaultdict(float)
    energies = []

    def check(i, call, rec, got):
        assert rec.shape == got.shape, (i, call)
        err[call] = max(err[call], float(np.max(np.abs(rec - got))) if rec.size else 0.0)
        if call == "direct_op_exp_val":
            energies.append(got[0])

    n = replay(z, lambda a: DropinComputer(a), check, inner=lambda a, b: a.s.dot(b.s))
    assert n == len(z["calls"]) and energies
    for call, e in err.items():
        assert e < TOL, (call, e)
    assert abs(energies[-1].real - float(z["e_fci"])) < float(z["tol"])
    assert abs(energies[-1].real - float(z["energy"])) < TOL
