"""PQE residuals on the device (UCCNPQE.get_residual_vector,
ucc/uccnpqe.py:249-292): the evaluator's residual run on every evaluator path
against the reference's residual vectors and the oracle, batches of
parameter rows, the per-call Computer path, and the reference test's
He/cc-pVDZ UCCSD-PQE energy (tests/test_uccsd.py:68-84)."""

import numpy as np
import pytest

from oracle import oracle as O
from qforte_b200.ucc import DUCC, UCCNPQE, evaluator_config, excited_determinants
from tests.conftest import golden
from tests.helpers import kops_forward, oracle_terms, random_problem
from tests.test_gpu_drivers import _mol

pytestmark = pytest.mark.gpu

R_TOL = 1e-10  # residuals are energies: the energy tolerance


@pytest.mark.parametrize("mode", [True, "global", False])
@pytest.mark.parametrize("name", ["pqe_norb4_seed11.npz", "pqe_norb6_seed11.npz"])
def test_residuals_match_reference_on_every_path(cuda, name, mode):
    """Compact shared-memory, compact global-memory and full-space evaluators
    give the reference's residual vector at its amplitudes."""
    z = golden(name)
    mol, pool = random_problem(int(z["norb"]), int(z["seed"]))
    tops = list(range(len(pool)))
    evaluator_config(mode)
    try:
        eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
        E, r = eng.residuals(z["amps"])
        path = eng.evaluator(1).path
    finally:
        evaluator_config(True)
    assert path in {True: (2,), "global": (3,), False: (0, 1)}[mode]
    assert np.max(np.abs(r - z["residuals"])) < R_TOL
    Ev = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference).energy(z["amps"])
    assert abs(E - Ev) < 1e-12


@pytest.mark.parametrize("B", [3, 17])
def test_residual_batches_match_the_oracle(cuda, B):
    mol, pool = random_problem(5, 4)
    tops = list(range(len(pool)))
    rng = np.random.default_rng(B)
    P = rng.uniform(-0.2, 0.2, (B, len(tops)))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    E, R = eng.residuals(P)
    dets = excited_determinants(pool, tops, mol.hf_reference)
    hterms = oracle_terms(mol.hamiltonian)
    kf = kops_forward(pool, tops)
    for b in (0, B - 1):
        r_o = O.pqe_residuals(10, mol.hf_reference, kf, P[b], hterms, dets)
        assert np.max(np.abs(R[b] - r_o)) < R_TOL
    # the residual run leaves energies and gradients of other modes intact
    E2, G2 = eng.energy_grad(P)
    assert np.max(np.abs(E2 - E)) < 1e-12
    E3, R3 = eng.residuals(P)
    assert np.max(np.abs(R3 - R)) == 0.0


def test_residuals_16_qubits_compact_vs_full_space(cuda):
    """16 qubits (a 4,900-amplitude sector: states beyond 48 KB of shared
    memory per CTA): the compact residual kernel against the full-space path."""
    mol, pool = random_problem(8, 11)
    tops = list(range(len(pool)))
    P = np.random.default_rng(5).uniform(-0.1, 0.1, (2, len(tops)))
    out = {}
    for mode in (True, False):
        evaluator_config(mode)
        try:
            eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
            out[mode] = eng.residuals(P) + (eng.evaluator(2).path,)
        finally:
            evaluator_config(True)
    assert out[True][2] == 2 and out[False][2] in (0, 1)
    assert np.max(np.abs(out[True][0] - out[False][0])) < 1e-12
    assert np.max(np.abs(out[True][1] - out[False][1])) < R_TOL


def test_percall_residuals_match_fused(cuda):
    """The reference's residual recipe through the Computer API (U, H, U
    adjoint, get_coeff_vec) gives the evaluator's residuals."""
    z = golden("pqe_norb4_seed11.npz")
    mol, _ = random_problem(4, 11)
    out = {}
    for engine in ("fused", "percall"):
        alg = UCCNPQE(mol, engine=engine)
        alg._pool_type = "SD"
        alg._noise_factor = 0.0
        alg._res_vec_evals = alg._res_m_evals = 0
        alg.fill_pool()
        alg.initialize_ansatz()
        alg.fill_excited_dets()
        out[engine] = np.array(alg.get_residual_vector(z["amps"]))
    assert np.max(np.abs(out["fused"] - z["residuals"])) < R_TOL
    assert np.max(np.abs(out["percall"] - z["residuals"])) < R_TOL


def test_he_uccsd_pqe_reaches_fci(cuda):
    """tests/test_uccsd.py:68-84: He/cc-pVDZ UCCSD-PQE (Jacobi with DIIS)
    reaches the FCI energy -2.887594831090938 within 1e-11."""
    alg = UCCNPQE(_mol("he_ccpvdz_integrals.npz"))
    E = alg.run(pool_type="SD", opt_thresh=1.0e-7)
    assert abs(E - -2.887594831090938) < 1e-11
