"""The reference's own drivers' engine calls, replayed on the device Computer,
and the reference's own objects handed to it.

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


def test_reference_objects_on_the_device(cuda):
    """The reference's compiled Gate / Circuit / QubitOperator / QubitOpPool
    passed straight to the device Computer (rebuilt by duck typing at each
    entry point): states, expectation values and pool expectation values equal
    the reference Computer's on the same objects (1e-12)."""
    from test_foreign_objects import reference_circuit, reference_engine, reference_operator
    qf = reference_engine()
    n = 9
    for seed in range(3):
        rc = reference_circuit(qf, n, 200, 10 + seed)
        ref = qf.Computer(n)
        ref.apply_circuit(rc)
        qc = qb.Computer(n)
        qc.apply_circuit(rc)
        assert np.max(np.abs(qc.get_coeff_array() - np.array(ref.get_coeff_vec()))) < TOL
        g = qf.gate("cRz", 3, 1, 0.7)
        ref.apply_gate(g)
        qc.apply_gate(g)
        assert np.max(np.abs(qc.get_coeff_array() - np.array(ref.get_coeff_vec()))) < TOL
        qo = reference_operator(qf, n, 40, seed)
        assert abs(qc.direct_op_exp_val(qo) - ref.direct_op_exp_val(qo)) < TOL
        pool = qf.QubitOpPool()
        for k in range(4):
            pool.add(complex(0.5 + k, -0.25 * k), reference_operator(qf, n, 10, 100 * seed + k))
        assert np.max(np.abs(np.array(qc.direct_oppl_exp_val(pool)) -
                             np.array(ref.direct_oppl_exp_val(pool)))) < TOL
        ref.apply_operator(qo)
        qc.apply_operator(qo)
        assert np.max(np.abs(qc.get_coeff_array() - np.array(ref.get_coeff_vec()))) < 1e-11
