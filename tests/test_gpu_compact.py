"""Compact (FEB / QEB) excitation circuits (utils/compact_excitation_circuits.py)
through the device gate kernels: the reference's states, and the same energies
as the fused Pauli-exponential program (the circuits apply exp(t kappa)
exactly, as tests/test_feb_qeb_circuits.py of the reference checks)."""

import numpy as np
import pytest

import qforte_b200 as qb
from qforte_b200.ucc import DUCC, UCCNVQE
from tests.conftest import golden
from tests.helpers import random_problem
from tests.test_host_algebra import _compact_ops

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pool_type", ["SD", "GSD", "sa_SD"])
@pytest.mark.parametrize("qe", [False, True])
def test_compact_ansatz_state_matches_reference(cuda, pool_type, qe):
    z = golden("compact_norb4.npz")
    key = f"{pool_type}_{'qe' if qe else 'fe'}"
    U = qb.Circuit()
    for j in range(4):
        U.add(qb.gate("X", j, j))
    for t, op in zip(z[f"{pool_type}_amps"], _compact_ops(pool_type)):
        e = op.terms()[1]
        U.add(qb.compact_excitation_circuit(t * e[0], e[1], e[2], qe))
    qc = qb.Computer(8)
    qc.apply_circuit(U)
    assert np.max(np.abs(qc.get_coeff_array() - z[f"{key}_psi"])) < 1e-12


@pytest.mark.parametrize("pool_type", ["SD", "GSD", "sa_SD"])
@pytest.mark.parametrize("qe", [False, True])
def test_compact_circuits_give_the_fused_energies(cuda, pool_type, qe):
    """Energy of the compact-circuit ansatz on the per-call path (gates
    through Computer) equals the fused engine's (1e-10, as the reference's
    test_feb_qeb_circuits), which needs no change of program."""
    mol, pool = random_problem(4, 11, pool_type)
    percall = UCCNVQE(mol, pool_type=pool_type, qubit_excitations=qe, engine="percall",
                      compact_excitations=True)
    fused = UCCNVQE(mol, pool_type=pool_type, qubit_excitations=qe, engine="fused",
                    compact_excitations=True)
    amps = np.random.default_rng(3).uniform(-0.3, 0.3, len(pool))
    for alg in (percall, fused):
        alg.fill_pool()
        alg._tops = list(range(len(alg._pool_obj)))
        alg._tamps = list(amps)
    assert abs(percall.energy_feval(amps) - fused.energy_feval(amps)) < 1e-10
    standard = UCCNVQE(mol, pool_type=pool_type, qubit_excitations=qe, engine="percall")
    standard.fill_pool()
    standard._tops = list(range(len(standard._pool_obj)))
    assert abs(standard.energy_feval(amps) - fused.energy_feval(amps)) < 1e-10
    assert (percall.build_Uvqc(list(amps)).get_num_cnots()
            < standard.build_Uvqc(list(amps)).get_num_cnots())
