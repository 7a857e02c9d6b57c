"""The drop-in boundary seen from the reference's side.

The reference's own Python package -- its drivers (UCCNVQE, ADAPTVQE, ...),
system factory and adapters, utilities -- is imported from its sources with
its compiled module ``qforte.qforte`` replaced by this package: the one-line
patch of src/qforte/__init__.py:5 (``from .qforte import *`` ->
``from qforte_b200 import *``).  Every object those drivers build (Gate,
Circuit, QubitOperator, SQOperator, SQOpPool, QubitOpPool, QubitBasis, ...) is
then this package's.

These tests need the reference's sources, which exist only in the build
container ($QFORTE_REF_SRC, default /root/reference/src/qforte), and run
without a GPU: the state the drivers evolve is the oracle's host state (a
stand-in with the Computer methods they call).  The engine behind
qforte_b200.Computer is covered by the GPU tests, including the same two
end-to-end runs through this package's drivers (test_gpu_drivers.py).

Pins: the reference's tests/test_uccsd.py:13-29 (He/cc-pVDZ UCCSD-VQE at FCI
within 1e-10) and tests/test_adapt_vqe.py:12-40 (H4/STO-6G ADAPT-VQE, SDTQ
pool, at FCI within 5e-11).
"""

import importlib.util
import os
import sys
import types
import warnings

import numpy as np
import pytest

from test_qite_host import HostComputer

REF_SRC = os.environ.get("QFORTE_REF_SRC", "/root/reference/src/qforte")


class DropinComputer(HostComputer):
    """The oracle's host state with the rest of the Computer surface the
    reference's drivers call (computer.h:22-185)."""

    def get_nqubit(self):
        return self.n

    def set_coeff_vec(self, c):
        self.s.psi[:] = np.asarray(c, dtype=np.complex128)

    def direct_oppl_exp_val(self, pool):
        return [c * self.direct_op_exp_val(op) for c, op in pool.terms()]

    def direct_idxd_oppl_exp_val(self, pool, idxs):
        t = pool.terms()
        return [t[i][0] * self.direct_op_exp_val(t[i][1]) for i in idxs]


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(os.path.join(REF_SRC, "__init__.py")):
        pytest.skip("the reference's Python sources are not present here")
    import qforte_b200
    saved = {k: v for k, v in sys.modules.items() if k == "qforte" or k.startswith("qforte.")}
    for k in saved:
        del sys.modules[k]
    shim = types.ModuleType("qforte.qforte")
    shim.__dict__.update({k: getattr(qforte_b200, k) for k in dir(qforte_b200)
                          if not k.startswith("_")})
    shim.Computer = DropinComputer
    shim.inner_product = lambda a, b: a.s.dot(b.s)

    def prepare(n, circ):
        qc = DropinComputer(n)
        qc.apply_circuit(circ)
        return qc

    shim.prepare_computer_from_circuit = prepare
    sys.modules["qforte.qforte"] = shim
    spec = importlib.util.spec_from_file_location(
        "qforte", os.path.join(REF_SRC, "__init__.py"), submodule_search_locations=[REF_SRC])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qforte"] = mod
    try:
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")  # the reference's own docstring escapes
            spec.loader.exec_module(mod)
        yield mod
    finally:
        for k in [k for k in sys.modules if k == "qforte" or k.startswith("qforte.")]:
            del sys.modules[k]
        sys.modules.update(saved)


def _data(name):
    return os.path.join(os.path.dirname(os.path.dirname(REF_SRC.rstrip("/"))), "tests", name)


def test_reference_objects_are_this_packages(ref):
    import qforte_b200
    for name in ("Gate", "Circuit", "QubitOperator", "SQOperator", "SQOpPool", "QubitOpPool",
                 "QubitBasis", "gate"):
        assert getattr(ref, name) is getattr(qforte_b200, name), name
    # the reference's own drivers, not this package's
    assert ref.UCCNVQE.__module__.startswith("qforte.ucc")
    assert ref.ADAPTVQE.__module__.startswith("qforte.ucc")


def test_reference_uccsd_vqe_runs_on_this_package(ref):
    """tests/test_uccsd.py:13-29 of the reference, as written there."""
    mol = ref.system_factory(system_type="molecule", build_type="external", basis="cc-pvdz",
                             filename=_data("He-ccpvdz.json"))
    assert isinstance(mol.hamiltonian, ref.QubitOperator)
    alg = ref.UCCNVQE(mol)
    alg.run(pool_type="SD", use_analytic_grad=True)
    assert abs(alg.get_gs_energy() - (-2.887594831090938)) < 1.0e-10


def test_reference_adapt_vqe_runs_on_this_package(ref):
    """tests/test_adapt_vqe.py:12-40 of the reference, as written there."""
    mol = ref.system_factory(stytem_type="molecule", build_type="external", basis="sto-6g",
                             filename=_data("H4-sto6g-075a.json"))
    alg = ref.ADAPTVQE(mol, print_summary_file=False)
    alg.run(adapt_maxiter=20, avqe_thresh=1.0e-4, opt_thresh=1.0e-5, use_analytic_grad=True,
            pool_type="SDTQ")
    assert abs(alg.get_gs_energy() - (-2.1628978832666865)) < 5.0e-11
