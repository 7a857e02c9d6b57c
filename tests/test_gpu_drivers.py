"""End-to-end pins from the reference's own test-suite: the optimised energies
of its UCCSD-VQE and ADAPT-VQE tests, reached through the device engine."""

import numpy as np
import pytest

import qforte_b200 as qb
from qforte_b200.ucc import ADAPTVQE, UCCNVQE
from tests.conftest import golden
from tests.helpers import random_problem, sq_from_integrals

pytestmark = pytest.mark.gpu


def _mol(name):
    H, ref = sq_from_integrals(golden(name))
    mol = qb.Molecule()
    mol.sq_hamiltonian = H
    mol.hamiltonian = H.jw_transform()
    mol.hf_reference = ref
    return mol


def test_he_uccsd_vqe_reaches_fci(cuda):
    """tests/test_uccsd.py:13-29: He/cc-pVDZ dUCCSD-VQE (BFGS, analytic
    gradient) reaches the FCI energy -2.887594831090938 within 1e-10."""
    alg = UCCNVQE(_mol("he_ccpvdz_integrals.npz"))
    E = alg.run(pool_type="SD", optimizer="BFGS")
    assert abs(E - -2.887594831090938) < 1e-10


def test_h4_adapt_vqe_reaches_fci(cuda):
    """tests/test_adapt_vqe.py:12-40: H4/STO-6G ADAPT-VQE with the SDTQ pool
    reaches the FCI energy -2.1628978832666865 within 5e-11."""
    alg = ADAPTVQE(_mol("h4_sto6g_integrals.npz"))
    E = alg.run(adapt_maxiter=20, avqe_thresh=1.0e-4, opt_thresh=1.0e-5, pool_type="SDTQ")
    assert abs(E - -2.1628978832666865) < 5e-11


def test_percall_path_matches_fused_engine(cuda):
    """The plain per-call path (the reference driver's Computer calls) and the
    fused engine give the same energies and gradients."""
    mol, pool = random_problem(4, 11)
    z = golden("ucc_norb4_seed11.npz")
    fused = UCCNVQE(mol, engine="fused")
    plain = UCCNVQE(mol, engine="percall")
    for alg in (fused, plain):
        alg._pool_type = "SD"
        alg.fill_pool()
        alg._tops = list(range(len(alg._pool_obj)))
        alg._tamps = list(z["amps"])
    assert abs(fused.energy_feval(z["amps"]) - float(z["energy"])) < 1e-10
    assert abs(plain.energy_feval(z["amps"]) - float(z["energy"])) < 1e-10
    gf = fused.measure_gradient(z["amps"])
    gp = plain.measure_gradient(z["amps"])
    assert np.max(np.abs(gf - z["grad"])) < 1e-8
    assert np.max(np.abs(gp - z["grad"])) < 1e-8
