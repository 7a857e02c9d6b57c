"""The reference's own drivers' engine calls, replayed on the device Computer.

tests/golden/dropin_trace_*.npz record every Computer call the reference's
UCCNVQE (He/cc-pVDZ, its tests/test_uccsd.py:13-29) and ADAPTVQE (H4/STO-6G,
SDTQ pool, its tests/test_adapt_vqe.py:12-40) made on the reference's compiled
Computer -- constructors and copies, apply_circuit, apply_operator,
direct_op_exp_val, get_coeff_vec, ... -- with the reference's results
(tests/golden/make_dropin_trace.py).  Replayed call for call through
qforte_b200.Computer (the C ABI, the CUDA kernels), every result must equal
the reference's (1e-12) and the last energy is the reference's FCI value
within the tolerance its test states: the drop-in engine answers the
reference's drivers as the reference's engine did.
"""

import collections

import numpy as np
import pytest

import qforte_b200 as qb
from dropin_trace import replay
from tests.conftest import golden

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("name", ["uccnvqe_he", "adaptvqe_h4"])
def test_reference_driver_trace_on_the_device(cuda, name):
    z = golden(f"dropin_trace_{name}.npz")
    err = collections.defaultdict(float)
    count = collections.Counter()
    energies = []

    def check(i, call, rec, got):
        assert rec.shape == got.shape, (i, call)
        err[call] = max(err[call], float(np.max(np.abs(rec - got))) if rec.size else 0.0)
        count[call] += 1
        if call == "direct_op_exp_val":
            energies.append(got[0])

    n = replay(z, lambda a: qb.Computer(a), check, inner=qb.inner_product)
    assert n == len(z["calls"]) and count["direct_op_exp_val"] > 10 and count["get_coeff_vec"] > 10
    for call, e in err.items():
        assert e < TOL, (call, e)
    assert abs(energies[-1].real - float(z["e_fci"])) < float(z["tol"])
    assert abs(energies[-1].real - float(z["energy"])) < TOL
