"""GPU parity: the libqfb.so kernels against the oracle and the reference's
golden vectors.  Tolerances: amplitudes 1e-12
max-abs, energies 1e-10, gradients 1e-8; basis-index work bit-exact."""

import math

import numpy as np
import pytest

import qforte_b200 as qb
from oracle import oracle as O
from qforte_b200.ucc import DUCC
from tests.conftest import golden
from tests.helpers import (kops_forward, kops_gradient, oracle_terms, oracle_terms_from_arrays,
                           qo_from_arrays, random_problem)

pytestmark = pytest.mark.gpu

AMP_TOL = 1e-12
E_TOL = 1e-10
G_TOL = 1e-8

ONE = ["X", "Y", "Z", "H", "R", "Rx", "Ry", "Rz", "V", "S", "T", "I"]
TWO = ["A", "cX", "acX", "cY", "cZ", "cR", "cV", "cRz", "SWAP", "CNOT", "aCNOT"]


def _rand_circuit(n, ngates, seed):
    rng = np.random.default_rng(seed)
    circ, ora = qb.Circuit(), []
    for _ in range(ngates):
        if rng.random() < 0.5:
            k, t = ONE[rng.integers(len(ONE))], int(rng.integers(n))
            c = t
        else:
            k = TWO[rng.integers(len(TWO))]
            t, c = (int(v) for v in rng.choice(n, 2, replace=False))
        p = float(rng.uniform(0, 4 * math.pi))
        circ.add(qb.gate(k, t, c, p))
        ora.append(O.make_gate(k, t, c, p))
    return circ, ora


def test_gates_match_reference_golden(cuda):
    z = golden("gates_n6.npz")
    qc = qb.Computer(int(z["n"]))
    circ = qb.Circuit()
    for k, t, c, p in zip(z["kinds"], z["target"], z["control"], z["param"]):
        circ.add(qb.gate(str(k), int(t), int(c), float(p)))
    qc.apply_circuit(circ)
    assert np.max(np.abs(qc.get_coeff_array() - z["psi"])) < AMP_TOL


@pytest.mark.parametrize("n,ngates,seed", [(2, 60, 1), (5, 400, 2), (9, 300, 3), (13, 120, 4)])
def test_gates_match_oracle(cuda, n, ngates, seed):
    circ, ora = _rand_circuit(n, ngates, seed)
    qc = qb.Computer(n)
    qc.apply_circuit(circ)
    st = O.State(n)
    st.apply_gates(ora)
    assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < AMP_TOL


def test_every_gate_every_ordering(cuda):
    """tests/test_comprehensive_gate.py:74-91 of the reference: every 2-qubit
    gate on all (target, control) orderings of 5 qubits, from a random state."""
    rng = np.random.default_rng(9)
    psi0 = rng.normal(size=32) + 1j * rng.normal(size=32)
    psi0 /= np.linalg.norm(psi0)
    for k in ("cV", "cX", "acX", "cY", "cZ", "cR", "cRz", "SWAP", "A"):
        for t in range(5):
            for c in range(5):
                if t == c:
                    continue
                qc = qb.Computer(5)
                qc.set_coeff_vec(psi0)
                qc.apply_gate(qb.gate(k, t, c, 0.37))
                st = O.State(5, psi0)
                st.apply_gates([O.make_gate(k, t, c, 0.37)])
                assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < 1e-15, (k, t, c)


def test_operator_application_and_expectations(cuda):
    z = golden("gates_n6.npz")
    qc = qb.Computer(int(z["n"]))
    qc.set_coeff_vec(z["psi"])
    op = qb.build_operator("0.5, X_0 Z_2; 0.3j, Y_1 X_3; -0.7, Z_0 Z_5; 0.2, X_1 X_1; "
                           "0.1, Y_2 Z_2 X_4; -0.25j, Z_3")
    ev = qc.direct_op_exp_val(op)
    assert abs(ev - complex(z["op_expval"])) < E_TOL
    pev = [qc.direct_pauli_circ_exp_val(qb.build_circuit(s))
           for s in ("X_0 Y_1", "Y_2", "Y_1 Y_3 Z_0", "X_5 X_5 Y_4", "Z_1 X_1")]
    assert np.max(np.abs(np.array(pev) - z["pauli_expvals"])) < E_TOL
    pm = qc.perfect_measure_circuit(qb.build_circuit("X_0 Y_2 Z_4"))
    assert abs(pm - float(z["perfect_measure"])) < E_TOL
    qc2 = qb.Computer(qc)
    qc2.apply_operator(op)
    assert np.max(np.abs(qc2.get_coeff_array() - z["op_psi"])) < AMP_TOL
    # a term with a non-Pauli gate takes the general path (copy, circuit, scale, sum)
    opg = qb.build_operator("0.5, X_0 Z_2; 0.3, H_1 cX_3_1")
    qc3 = qb.Computer(qc)
    qc3.apply_operator(opg)
    st = O.State(6, z["psi"])
    st.apply_operator([(0.5, [O.make_gate("X", 0, 0), O.make_gate("Z", 2, 2)]),
                       (0.3, [O.make_gate("H", 1, 1), O.make_gate("cX", 3, 1)])])
    assert np.max(np.abs(qc3.get_coeff_array() - st.psi)) < AMP_TOL


def test_trotterized_exponentials_fused_vs_gates(cuda):
    """exp(c P) circuits run as one fused pass; the gates they stand for give
    the same state (reference: utils/exponentiate.py)."""
    rng = np.random.default_rng(4)
    n = 7
    A = qb.QubitOperator()
    terms = []
    for _ in range(25):
        sup = sorted(rng.choice(n, rng.integers(1, 5), replace=False))
        letters = [("X", "Y", "Z")[rng.integers(3)] for _ in sup]
        circ = qb.Circuit()
        for l, q in zip(letters, sup):
            circ.add(qb.gate(l, int(q)))
        c = 1j * rng.uniform(-1, 1)
        A.add(c, circ)
        terms.append((c, list(zip(letters, [int(q) for q in sup]))))
    U, phase = qb.trotterize(A)
    assert U._pexp is not None and len(U._pexp) == 25
    qc = qb.Computer(n)
    qc.apply_circuit(qb.build_circuit("H_0 H_3 X_5 Ry_2_0.7"))
    qc.apply_circuit(U)
    st = O.State(n)
    st.apply_gates([O.make_gate("H", 0, 0), O.make_gate("H", 3, 3), O.make_gate("X", 5, 5),
                    O.make_gate("Ry", 2, 2, 0.7)])
    g, _ = O.trotterize(terms)
    st.apply_gates(g)
    assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < AMP_TOL
    # the adjoint circuit undoes it
    qc.apply_circuit(U.adjoint())
    st2 = O.State(n)
    st2.apply_gates([O.make_gate("H", 0, 0), O.make_gate("H", 3, 3), O.make_gate("X", 5, 5),
                     O.make_gate("Ry", 2, 2, 0.7)])
    assert np.max(np.abs(qc.get_coeff_array() - st2.psi)) < AMP_TOL


@pytest.mark.parametrize("name", ["ucc_norb4_seed11.npz", "ucc_norb6_seed11.npz"])
def test_ducc_energy_state_gradient_vs_reference(cuda, name):
    z = golden(name)
    mol, pool = random_problem(int(z["norb"]), int(z["seed"]))
    tops = list(range(len(pool)))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    amps = z["amps"]
    E = eng.energy(amps)
    assert abs(E - float(z["energy"])) < E_TOL
    psi = eng.state(amps).get_coeff_array()
    assert np.max(np.abs(psi - z["psi"])) < AMP_TOL
    E2, g = eng.energy_grad(amps)
    assert abs(E2 - float(z["energy"])) < E_TOL
    assert np.max(np.abs(g - z["grad"])) < G_TOL
    # a batch gives each row's single-call result
    rng = np.random.default_rng(5)
    P = np.vstack([amps, rng.uniform(-0.1, 0.1, (3, len(amps)))])
    EB, GB = eng.energy_grad(P)
    for b in range(P.shape[0]):
        e1, g1 = eng.energy_grad(P[b])
        assert abs(EB[b] - e1) < 1e-12 and np.max(np.abs(GB[b] - g1)) < 1e-12
    assert np.max(np.abs(eng.energy(P) - EB)) < 1e-12


def test_ducc_pool_gradients_vs_reference(cuda):
    z = golden("ucc_norb4_seed11.npz")
    mol, gsd = random_problem(4, int(z["seed"]), "GSD")
    tops = [int(t) for t in z["gsd_tops"]]
    eng = DUCC(mol.hamiltonian, gsd, tops, mol.hf_reference)
    g = eng.pool_gradients(z["gsd_amps"])
    assert np.max(np.abs(g - z["pool_grads"])) < G_TOL


def test_ducc_vs_oracle_14_qubits(cuda):
    mol, pool = random_problem(7, 3)
    tops = list(range(len(pool)))
    rng = np.random.default_rng(8)
    amps = rng.uniform(-0.1, 0.1, len(tops))
    hterms = oracle_terms(mol.hamiltonian)
    E_o, st = O.energy(14, mol.hf_reference, kops_forward(pool, tops), amps, hterms)
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    E, g = eng.energy_grad(amps)
    assert abs(E - E_o) < E_TOL
    assert np.max(np.abs(eng.state(amps).get_coeff_array() - st.psi)) < AMP_TOL


def test_ducc_gradient_vs_oracle_14_qubits(cuda):
    """Multi-tile windows (gradient tiles of 2^11 amplitudes on 14 qubits)."""
    mol, pool = random_problem(7, 5)
    tops = list(range(len(pool)))
    rng = np.random.default_rng(12)
    amps = rng.uniform(-0.1, 0.1, len(tops))
    hterms = oracle_terms(mol.hamiltonian)
    g_o = O.measure_gradient(14, mol.hf_reference, kops_forward(pool, tops), amps, hterms,
                             kops_grad=kops_gradient(pool, tops))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    _, g = eng.energy_grad(amps)
    assert np.max(np.abs(g - g_o)) < G_TOL
    # the per-call C ABI path gives the same numbers
    e2, g2 = eng.energy_grad_percall(amps)
    assert np.max(np.abs(g2 - g)) < 1e-12


@pytest.mark.parametrize("norb", [4, 6])
def test_ducc_spin_adapted_pool_vs_oracle(cuda, norb):
    """sa_SD operators span several x-masks: multi-step parameters."""
    mol, pool = random_problem(norb, 17, "sa_SD")
    tops = list(range(len(pool)))
    rng = np.random.default_rng(norb)
    amps = rng.uniform(-0.1, 0.1, len(tops))
    nq = 2 * norb
    hterms = oracle_terms(mol.hamiltonian)
    kf = kops_forward(pool, tops, "sa_SD")
    E_o, st = O.energy(nq, mol.hf_reference, kf, amps, hterms)
    g_o = O.measure_gradient(nq, mol.hf_reference, kf, amps, hterms,
                             kops_grad=kops_gradient(pool, tops), kops_unrot=kf)
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type="sa_SD")
    E, g = eng.energy_grad(amps)
    assert abs(E - E_o) < E_TOL
    assert np.max(np.abs(eng.state(amps).get_coeff_array() - st.psi)) < AMP_TOL
    assert np.max(np.abs(g - g_o)) < G_TOL


def test_gradient_vs_central_differences(cuda):
    mol, pool = random_problem(5, 21)
    tops = list(range(len(pool)))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    rng = np.random.default_rng(2)
    t = rng.uniform(-0.1, 0.1, len(tops))
    _, g = eng.energy_grad(t)
    h = 1e-5
    P = np.repeat(t[None, :], 2 * len(t), axis=0)
    for k in range(len(t)):
        P[2 * k, k] += h
        P[2 * k + 1, k] -= h
    E = eng.energy(P)
    fd = (E[0::2] - E[1::2]) / (2 * h)
    assert np.max(np.abs(fd - g)) < G_TOL


def test_computer_api_and_errors(cuda):
    qc = qb.Computer(3)
    assert qc.get_coeff_vec()[0] == 1.0 and qc.get_nqubit() == 3
    qc.set_state([(qb.QubitBasis(5), 0.6), (qb.QubitBasis(2), 0.8j)])
    a = qc.get_coeff_array()
    assert a[5] == 0.6 and a[2] == 0.8j and np.count_nonzero(a) == 2
    assert qc.coeff(qb.QubitBasis(2)) == 0.8j
    cp = qb.Computer(qc)
    assert cp == qc
    cp.apply_constant(2.0)
    assert abs(qb.inner_product(qc, cp) - 2.0) < 1e-15
    cp.null_state()
    assert not np.any(cp.get_coeff_array())
    cp.reset()
    assert cp.get_coeff_array()[0] == 1.0
    assert qc.direct_gate_exp_val(qb.gate("X", 0)) == 0  # computer.cc:937-954 behaviour
    assert qc.get_coeff_array()[4] == 0.6  # ... with the gate left applied
    with pytest.raises(ValueError):
        qc.apply_gate(qb.gate("X", 3))
    with pytest.raises(ValueError):
        qc.apply_operator(qb.build_operator("1.0, Z_7"))
    with pytest.raises(ValueError):
        qc.set_coeff_vec(np.zeros(4))
    assert "Computer(" in qc.str()
    big = qb.Computer(1)
    big.apply_gate(qb.gate("H", 0))
    assert abs(big.get_coeff_array()[1] - 1 / math.sqrt(2)) < 1e-16


def test_sector_restricted_h_apply(cuda):
    """Programs that keep the reference's numbers of alpha and beta electrons
    form sigma = H psi on that sector only; a program with a spin flip keeps
    the full space.  Both match the oracle."""
    from math import comb
    mol, pool = random_problem(4, 11)
    tops = list(range(len(pool)))
    rng = np.random.default_rng(4)
    amps = rng.uniform(-0.1, 0.1, len(tops))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    assert eng.evaluator(1).sector_size == comb(4, 2) ** 2
    hterms = oracle_terms(mol.hamiltonian)
    E_o, _ = O.energy(8, mol.hf_reference, kops_forward(pool, tops), amps, hterms)
    g_o = O.measure_gradient(8, mol.hf_reference, kops_forward(pool, tops), amps, hterms,
                             kops_grad=kops_gradient(pool, tops))
    E, g = eng.energy_grad(amps)
    assert abs(E - E_o) < E_TOL and np.max(np.abs(g - g_o)) < G_TOL

    # append a spin flip (alpha orbital 1 <- beta orbital 0) to the pool
    flip = qb.SQOperator()
    flip.add(1.0, [2], [1])
    flip.add(-1.0, [1], [2])
    pool.add_term(1.0, flip)
    tops2 = tops + [len(pool) - 1]
    amps2 = np.append(amps, 0.07)
    eng2 = DUCC(mol.hamiltonian, pool, tops2, mol.hf_reference)
    assert eng2.evaluator(1).sector_size == 0
    E_o2, _ = O.energy(8, mol.hf_reference, kops_forward(pool, tops2), amps2, hterms)
    g_o2 = O.measure_gradient(8, mol.hf_reference, kops_forward(pool, tops2), amps2, hterms,
                              kops_grad=kops_gradient(pool, tops2))
    E2, g2 = eng2.energy_grad(amps2)
    assert abs(E2 - E_o2) < E_TOL and np.max(np.abs(g2 - g_o2)) < G_TOL
    assert abs(E2 - E) > 1e-6  # the flip changes the state


@pytest.mark.parametrize("pool_type", ["GSD", "sa_SD"])
def test_sector_for_generalized_and_spin_adapted_pools(cuda, pool_type):
    from math import comb
    mol, pool = random_problem(4, 9, pool_type)
    tops = list(range(0, len(pool), 3))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type=pool_type)
    assert eng.evaluator(2).sector_size == comb(4, 2) ** 2
    rng = np.random.default_rng(1)
    amps = rng.uniform(-0.1, 0.1, len(tops))
    hterms = oracle_terms(mol.hamiltonian)
    kf = kops_forward(pool, tops, pool_type)
    E_o, _ = O.energy(8, mol.hf_reference, kf, amps, hterms)
    g_o = O.measure_gradient(8, mol.hf_reference, kf, amps, hterms,
                             kops_grad=kops_gradient(pool, tops),
                             kops_unrot=kf if pool_type == "sa_SD" else None)
    E, g = eng.energy_grad(np.vstack([amps, amps]))
    assert np.max(np.abs(E - E_o)) < E_TOL and np.max(np.abs(g - g_o[None, :])) < G_TOL


@pytest.fixture
def gate_tiles():
    """Restores the default gate tile shape after a test changes it."""
    from qforte_b200._lib import check, lib
    yield lambda b, L: check(lib().qfb_gates_config(b, L), "qfb_gates_config")
    check(lib().qfb_gates_config(0, 3), "qfb_gates_config")


@pytest.mark.parametrize("tile,low", [(-1, 4), (0, 4), (2, 0), (4, 1), (6, 3), (9, 4), (10, 3),
                                      (11, 3), (12, 3), (12, 6)])
@pytest.mark.parametrize("n,ngates,seed", [(3, 80, 5), (8, 300, 6), (14, 200, 7)])
def test_gate_windows_match_oracle(cuda, gate_tiles, tile, low, n, ngates, seed):
    """Gate runs applied to shared-memory tiles of every shape (and one pass
    per gate, tile -1) against the oracle's gate-by-gate application."""
    gate_tiles(tile, low)
    circ, ora = _rand_circuit(n, ngates, seed)
    qc = qb.Computer(n)
    qc.apply_circuit(circ)
    st = O.State(n)
    st.apply_gates(ora)
    assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < AMP_TOL


def _control_heavy_circuit(n, seed):
    """Gates whose controls and diagonals sit on many qubits at once: runs of
    cX / cRz / cV on one target controlled by every other qubit (more thread
    bits per phase than one segment holds), cZ / cR between two high qubits
    (factors of the thread's bits alone), cR controlled by a low qubit on a
    high target, SWAPs and X (relabelings), between random gates."""
    rng = np.random.default_rng(seed)
    circ, ora = qb.Circuit(), []

    def add(k, t, c, p=0.0):
        circ.add(qb.gate(k, t, c, p))
        ora.append(O.make_gate(k, t, c, p))

    for rep in range(6):
        t = int(rng.integers(3))
        for c in range(n):
            if c != t:
                add(["cX", "cRz", "cV"][c % 3], t, c, float(rng.uniform(0, 6.3)))
        for _ in range(4):
            a, b = (int(v) for v in rng.choice(range(3, n), 2, replace=False))
            add(["cZ", "cR"][rep % 2], a, b, float(rng.uniform(0, 6.3)))
        add("cR", int(rng.integers(3, n)), int(rng.integers(3)), float(rng.uniform(0, 6.3)))
        add("SWAP", 0, 1)
        add("X", 2, 2)
        q = int(rng.integers(n))
        add("T", q, q)
        c2, o2 = _rand_circuit(n, 40, seed + rep)
        for g in c2.gates():
            circ.add(g)
        ora.extend(o2)
    return circ, ora


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("regs", [2, 3])
@pytest.mark.parametrize("n,kind,seed", [(10, "random", 41), (12, "controls", 42),
                                         (13, "random", 43), (14, "controls", 44)])
def test_fused_phases_match_oracle(cuda, fused, regs, n, kind, seed):
    """Tile phases in their fused form (block matrices per variant of the
    thread bits the controls test, per-thread factors) and gate by gate, with
    2 and 3 register bits, from a random state, against the oracle's
    gate-by-gate application."""
    from qforte_b200.device import gates_config
    circ, ora = (_rand_circuit(n, 400, seed) if kind == "random"
                 else _control_heavy_circuit(n, seed))
    psi0 = _random_state(n, seed)
    gates_config(0, 3, regs, 0, fused)
    try:
        qc = qb.Computer(n)
        qc.set_coeff_vec(psi0)
        qc.apply_circuit(circ)
        got = qc.get_coeff_array()
    finally:
        gates_config()
    st = O.State(n, psi0.copy())
    st.apply_gates(ora)
    assert np.max(np.abs(got - st.psi)) < AMP_TOL


@pytest.mark.parametrize("tile,low", [(8, 3), (9, 4), (11, 3), (11, 6)])
@pytest.mark.parametrize("n,kind,seed", [(12, "random", 45), (14, "controls", 46)])
def test_fused_phases_every_tile_shape(cuda, tile, low, n, kind, seed):
    """Fused tile phases in tiles of 8, 9 and 11 qubits (1, 2 and 8 warps of
    amplitude vectors) and with 3 to 6 low qubits kept, from a random state,
    against the oracle's gate-by-gate application."""
    from qforte_b200.device import gates_config
    circ, ora = (_rand_circuit(n, 400, seed) if kind == "random"
                 else _control_heavy_circuit(n, seed))
    psi0 = _random_state(n, seed)
    gates_config(tile, low, 0, 0, True)
    try:
        qc = qb.Computer(n)
        qc.set_coeff_vec(psi0)
        qc.apply_circuit(circ)
        got = qc.get_coeff_array()
    finally:
        gates_config()
    st = O.State(n, psi0.copy())
    st.apply_gates(ora)
    assert np.max(np.abs(got - st.psi)) < AMP_TOL


@pytest.fixture
def dense_blocks():
    """Sets dense K-qubit blocks (FP64 tensor cores) and restores the default."""
    from qforte_b200.device import gates_config
    yield lambda k: gates_config(0, 3, 0, k)
    gates_config(0, 3, 0, 0)


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("k", [5, 6])
@pytest.mark.parametrize("n,ngates,seed", [(10, 300, 31), (13, 250, 32), (16, 200, 33)])
def test_dense_blocks_match_oracle(cuda, dense_blocks, k, n, ngates, seed):
    """Runs of every gate kind fused into dense 2^k x 2^k unitaries and
    applied with FP64 mma.sync, from a random state, against the oracle's
    gate-by-gate application."""
    from qforte_b200.device import gate_plan
    circ, ora = _rand_circuit(n, ngates, seed)
    psi0 = _random_state(n, seed)
    dense_blocks(k)
    runs, singles, _ = gate_plan(circ.gates(), n)
    assert runs > 0
    qc = qb.Computer(n)
    qc.set_coeff_vec(psi0)
    qc.apply_circuit(circ)
    st = O.State(n, psi0.copy())
    st.apply_gates(ora)
    assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < AMP_TOL


@pytest.mark.parametrize("k", [5, 6])
def test_dense_block_of_a_deep_run_on_few_qubits(cuda, dense_blocks, k):
    """400 gates on 5 scattered qubits of 15 become one dense pass."""
    from qforte_b200.device import gate_plan
    n, qs = 15, [1, 4, 7, 11, 14]
    rng = np.random.default_rng(40 + k)
    circ, ora = qb.Circuit(), []
    for _ in range(400):
        if rng.random() < 0.5:
            kk, t = ONE[rng.integers(len(ONE))], int(rng.choice(qs))
            c = t
        else:
            kk = TWO[rng.integers(len(TWO))]
            t, c = (int(v) for v in rng.choice(qs, 2, replace=False))
        p = float(rng.uniform(0, 4 * math.pi))
        circ.add(qb.gate(kk, t, c, p))
        ora.append(O.make_gate(kk, t, c, p))
    psi0 = _random_state(n, 44)
    dense_blocks(k)
    assert gate_plan(circ.gates(), n)[:2] == (1, 0)
    qc = qb.Computer(n)
    qc.set_coeff_vec(psi0)
    qc.apply_circuit(circ)
    st = O.State(n, psi0.copy())
    st.apply_gates(ora)
    assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < AMP_TOL


@pytest.mark.parametrize("form", ["dense5", "fused", "ops"])
def test_gate_runs_on_a_batch_of_states(cuda, form):
    """Every slot of a batched state gets the same passes: dense 5-qubit
    blocks, and tile runs with their phases fused (FP64 tensor cores) or gate
    by gate."""
    import ctypes
    from qforte_b200._lib import check, lib, ptr
    from qforte_b200.device import gates_config, pack_gates
    n = 12
    circ, ora = _rand_circuit(n, 150, 35)
    L = lib()
    h = ctypes.c_void_p()
    check(L.qfb_state_create(n, 3, ctypes.byref(h)))
    try:
        psis = [_random_state(n, 50 + b) for b in range(3)]
        for b, v in enumerate(psis):
            check(L.qfb_state_upload(h, b, ptr(v), 1 << n))
        arr = pack_gates(circ.gates())
        gates_config(0, 3, 0, 5 if form == "dense5" else 0,
                     None if form == "dense5" else form == "fused")
        try:
            check(L.qfb_apply_gates(h, arr.ctypes.data, len(arr)), "qfb_apply_gates")
        finally:
            gates_config()
        for b, v in enumerate(psis):
            out = np.zeros(1 << n, dtype=np.complex128)
            check(L.qfb_state_download(h, b, ptr(out), 1 << n))
            st = O.State(n, v.copy())
            st.apply_gates(ora)
            assert np.max(np.abs(out - st.psi)) < AMP_TOL
    finally:
        L.qfb_state_destroy(h)


def test_gate_tile_wait_that_runs_out_reports_and_leaves_state(cuda, gate_tiles):
    """The tile kernel's bounded wait for its bulk load copies (the gate-by-gate
    phase form, which states smaller than L2 take), made to run out with no
    fault: with the wait limit at 0 every tile gives up at once, flags
    it and leaves its tile unwritten.  The next download reports
    QFB_ETIMEDOUT (RuntimeError), the state is exactly as before, and with the
    limit restored the same circuit gives the oracle's state."""
    from qforte_b200._lib import QFB_ETIMEDOUT, check, lib
    from qforte_b200.device import gate_plan
    gate_tiles(0, 3)
    n = 12
    rng = np.random.default_rng(21)
    circ, ora = qb.Circuit(), []
    for _ in range(60):  # gates on qubits 0-5 only: one tile run, no one-gate pass
        k, t = ONE[rng.integers(len(ONE))], int(rng.integers(6))
        p = float(rng.uniform(0, 4 * math.pi))
        circ.add(qb.gate(k, t, t, p))
        ora.append(O.make_gate(k, t, t, p))
    runs, single, _ = gate_plan(circ.gates(), n)
    assert runs >= 1 and single == 0
    psi0 = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi0 /= np.linalg.norm(psi0)
    qc = qb.Computer(n)
    qc.set_coeff_vec(psi0)
    check(lib().qfb_set_tile_wait_limit(0), "qfb_set_tile_wait_limit")
    try:
        with pytest.raises(RuntimeError, match=f"qfb status {QFB_ETIMEDOUT}"):
            qc.apply_circuit(circ)
            qc.get_coeff_array()
    finally:
        check(lib().qfb_set_tile_wait_limit(2_000_000_000), "qfb_set_tile_wait_limit")
    assert np.array_equal(qc.get_coeff_array(), psi0)
    qc.apply_circuit(circ)
    st = O.State(n, psi0.copy())
    st.apply_gates(ora)
    assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < AMP_TOL
    assert lib().qfb_set_tile_wait_limit(61_000_000_000) != 0


@pytest.mark.parametrize("n", [7, 16])
def test_layered_sweep_circuit_matches_oracle(cuda, gate_tiles, n):
    """The gate-sweep workload (random layers of 1-qubit gates and pairings)."""
    from qforte_b200.workloads import layered_random_circuit
    circ, spec = layered_random_circuit(n, 12, 3)
    st = O.State(n)
    st.apply_gates([O.make_gate(k, t, c, p) for k, t, c, p in spec])
    for tile in (0, -1):
        gate_tiles(tile, 4)
        qc = qb.Computer(n)
        qc.apply_circuit(circ)
        assert np.max(np.abs(qc.get_coeff_array() - st.psi)) < AMP_TOL


@pytest.mark.parametrize("B", [3, 9, 13, 40])
def test_sector_apply_every_batch_width(cuda, B):
    """Small batches take the one-output-per-thread sector kernel, large ones
    the one-output-per-warp kernel; each row equals its single-row result."""
    mol, pool = random_problem(5, 23)
    tops = list(range(len(pool)))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    rng = np.random.default_rng(B)
    P = rng.uniform(-0.1, 0.1, (B, len(tops)))
    EB, GB = eng.energy_grad(P)
    for b in (0, B // 2, B - 1):
        e1, g1 = eng.energy_grad(P[b])
        assert abs(EB[b] - e1) < 1e-12 and np.max(np.abs(GB[b] - g1)) < 1e-12
    hterms = oracle_terms(mol.hamiltonian)
    E_o, _ = O.energy(10, mol.hf_reference, kops_forward(pool, tops), P[B - 1], hterms)
    assert abs(EB[B - 1] - E_o) < E_TOL


@pytest.fixture
def compact_off():
    from qforte_b200.ucc import evaluator_config
    evaluator_config(False)
    yield
    evaluator_config(True)


@pytest.mark.parametrize("norb,seed,pool_type", [(4, 11, "SD"), (6, 3, "SD"), (5, 9, "GSD"),
                                                 (6, 17, "sa_SD"), (7, 5, "SD"), (8, 2, "SD")])
def test_compact_sector_path_matches_full_space(cuda, norb, seed, pool_type):
    """The compact sector evaluator (psi and sigma of one parameter set in a
    CTA's shared memory) against the full-space evaluator and the oracle."""
    from qforte_b200.ucc import evaluator_config
    mol, pool = random_problem(norb, seed, pool_type)
    tops = list(range(0, len(pool), 1 if len(pool) < 400 else 3))
    rng = np.random.default_rng(norb + seed)
    P = rng.uniform(-0.1, 0.1, (5, len(tops)))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type=pool_type)
    ev = eng.evaluator(5)
    E, G = eng.energy_grad(P)
    evaluator_config(False)
    try:
        eng2 = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type=pool_type)
        assert eng2.evaluator(5).path != 2
        E2, G2 = eng2.energy_grad(P)
    finally:
        evaluator_config(True)
    assert np.max(np.abs(E - E2)) < 1e-12 and np.max(np.abs(G - G2)) < 1e-11
    if pool_type in ("SD", "GSD"):
        assert ev.path == 2
    if norb <= 6:
        hterms = oracle_terms(mol.hamiltonian)
        kf = kops_forward(pool, tops, pool_type)
        E_o, _ = O.energy(2 * norb, mol.hf_reference, kf, P[0], hterms)
        g_o = O.measure_gradient(2 * norb, mol.hf_reference, kf, P[0], hterms,
                                 kops_grad=kops_gradient(pool, tops),
                                 kops_unrot=kf if pool_type == "sa_SD" else None)
        assert abs(E[0] - E_o) < E_TOL and np.max(np.abs(G[0] - g_o)) < G_TOL


def test_compact_energy_only_then_gradient_sweep(cuda):
    """Mode 0 (energy) saves the compact states; mode 2 sweeps from them."""
    import torch
    mol, pool = random_problem(6, 4)
    tops = list(range(len(pool)))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    ev = eng.evaluator(3)
    assert ev.path == 2
    rng = np.random.default_rng(6)
    P = rng.uniform(-0.1, 0.1, (3, len(tops)))
    E, G = eng.energy_grad(P)
    d_par, d_en, d_gr = ev.tensors()
    d_par.copy_(torch.from_numpy(P))
    d_gr.zero_()
    ev.run(0)
    ev.run(2)
    torch.cuda.synchronize()
    assert np.max(np.abs(d_en.cpu().numpy() - E)) < 1e-13
    assert np.max(np.abs(d_gr.cpu().numpy() - G)) < 1e-13


@pytest.mark.parametrize("compact", [True, False])
def test_pool_gradients_one_launch_vs_grouped_and_oracle(cuda, compact):
    """Every ADAPT pool gradient from the evaluator's pool stage (mode 3)
    against the grouped Pauli-sum path and the oracle's measure_gradient3."""
    from qforte_b200.ucc import evaluator_config
    mol, gsd = random_problem(5, 31, "GSD")
    rng = np.random.default_rng(3)
    tops = [int(t) for t in rng.choice(len(gsd), 6, replace=False)]
    amps = rng.uniform(-0.1, 0.1, 6)
    evaluator_config(compact)
    try:
        eng = DUCC(mol.hamiltonian, gsd, tops, mol.hf_reference)
        g = eng.pool_gradients(amps)
        ev = eng.evaluator(1)
        assert (ev.path == 2) == compact and getattr(ev, "_pool_prog", None) is not None
        g2 = eng.pool_gradients_grouped(amps)
        P = np.vstack([amps, rng.uniform(-0.1, 0.1, 6)])
        GB = eng.pool_gradients(P)
    finally:
        evaluator_config(True)
    assert np.max(np.abs(g - g2)) < 1e-12
    assert np.max(np.abs(GB[0] - g)) < 1e-12
    hterms = oracle_terms(mol.hamiltonian)
    g_o = O.measure_gradient3(10, mol.hf_reference, kops_forward(gsd, tops), amps, hterms,
                              kops_gradient(gsd, range(len(gsd))))
    assert np.max(np.abs(g - g_o)) < G_TOL
    g_o1 = O.measure_gradient3(10, mol.hf_reference, kops_forward(gsd, tops), P[1], hterms,
                               kops_gradient(gsd, range(len(gsd))))
    assert np.max(np.abs(GB[1] - g_o1)) < G_TOL


@pytest.mark.parametrize("B", [1, 3, 40])
@pytest.mark.parametrize("norb,seed,pool_type", [(4, 11, "SD"), (6, 3, "SD"), (5, 9, "GSD"),
                                                 (6, 17, "sa_SD")])
def test_global_sector_path_matches_shared_and_full(cuda, norb, seed, pool_type, B):
    """Compact sector states in global memory (slot-minor, one launch per
    step record) against the shared-memory path, the full-space path and the
    oracle, for slot groups of 1, 4 and 32 lanes."""
    from qforte_b200.ucc import evaluator_config
    mol, pool = random_problem(norb, seed, pool_type)
    tops = list(range(0, len(pool), 1 if len(pool) < 400 else 3))
    rng = np.random.default_rng(B + norb)
    P = rng.uniform(-0.1, 0.1, (B, len(tops)))
    res = {}
    for mode in (True, "global", "global-no-rows", False):
        evaluator_config(mode)
        try:
            eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type=pool_type)
            res[mode] = eng.energy_grad(P) + (eng.evaluator(B).path,)
        finally:
            evaluator_config(True)
    E3, G3, path3 = res["global"]
    E4, G4, path4 = res["global-no-rows"]
    E1, G1, path1 = res[False]
    E2, G2, path2 = res[True]
    assert path1 in (0, 1) and (pool_type == "sa_SD" or path3 == path4 == 3)
    assert np.max(np.abs(E3 - E1)) < 1e-12 and np.max(np.abs(G3 - G1)) < 1e-11
    assert np.max(np.abs(E3 - E2)) < 1e-12 and np.max(np.abs(G3 - G2)) < 1e-11
    assert np.max(np.abs(E4 - E1)) < 1e-12 and np.max(np.abs(G4 - G1)) < 1e-11
    if B == 3:
        hterms = oracle_terms(mol.hamiltonian)
        kf = kops_forward(pool, tops, pool_type)
        E_o, _ = O.energy(2 * norb, mol.hf_reference, kf, P[2], hterms)
        assert abs(E3[2] - E_o) < E_TOL


def test_global_sector_pool_gradients(cuda):
    from qforte_b200.ucc import evaluator_config
    mol, gsd = random_problem(5, 31, "GSD")
    rng = np.random.default_rng(3)
    tops = [int(t) for t in rng.choice(len(gsd), 6, replace=False)]
    P = rng.uniform(-0.1, 0.1, (2, 6))
    evaluator_config("global")
    try:
        eng = DUCC(mol.hamiltonian, gsd, tops, mol.hf_reference)
        g = eng.pool_gradients(P)
        assert eng.evaluator(2).path == 3 and getattr(eng.evaluator(2), "_pool_prog", None) is not None
    finally:
        evaluator_config(True)
    g2 = np.vstack([eng.pool_gradients_grouped(P[b]) for b in range(2)])
    assert np.max(np.abs(g - g2)) < 1e-12


@pytest.mark.parametrize("norb,seed,pool_type", [(4, 11, "SD"), (6, 3, "SD"), (5, 9, "GSD")])
def test_real_state_storage_matches_complex(cuda, norb, seed, pool_type):
    """The compact paths keep psi and sigma as real doubles when H and every
    step coefficient are real: energies, gradients, pool gradients and PQE
    residuals equal those of complex storage and of the full-space path, in
    shared memory and in global memory (with H rows and without)."""
    from qforte_b200.ucc import evaluator_config
    mol, pool = random_problem(norb, seed, pool_type)
    tops = list(range(0, len(pool), 1 if len(pool) < 400 else 3))
    P = np.random.default_rng(seed).uniform(-0.1, 0.1, (5, len(tops)))
    res = {}
    modes = (True, "complex", "global", "global-complex", "global-no-rows", False)
    for mode in modes:
        evaluator_config(mode)
        try:
            eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
            E, G = eng.energy_grad(P)
            ev = eng.evaluator(5)
            pg = eng.pool_gradients(P)
            out = (E, G, pg, ev.path, ev.real_states)
            if pool_type == "SD":
                out += (eng.residuals(P)[1],)
            res[mode] = out
        finally:
            evaluator_config(True)
    expect = {True: (2, True), "complex": (2, False), "global": (3, True),
              "global-complex": (3, False), "global-no-rows": (3, True)}
    for mode, (path, real) in expect.items():
        assert res[mode][3] == path and res[mode][4] is real, mode
    assert res[False][3] in (0, 1)
    for mode in modes[1:]:
        assert np.max(np.abs(res[True][0] - res[mode][0])) < 1e-12
        assert np.max(np.abs(res[True][1] - res[mode][1])) < 1e-11
        assert np.max(np.abs(res[True][2] - res[mode][2])) < 1e-11
        if pool_type == "SD":
            assert np.max(np.abs(res[True][5] - res[mode][5])) < 1e-11


def _gated_hop(i, a, ks, w, c=1.0):
    """T - T^dagger for T = c a^_a a_i (1 + w prod_k n_k): the strings' z-masks
    differ on the orbitals ks off the hop, so the step has one pattern per
    occupation of ks; with 1 + w = -1 every pattern rotates by the same angle
    (the Givens form).  c = 1j gives commuting XX / YY strings with imaginary
    pattern coefficients."""
    t = qb.SQOperator()
    K = list(ks)
    cw = complex(c) * w
    t.add_term(c, [a], [i])
    t.add_term(-complex(c).conjugate(), [i], [a])
    t.add_term(cw, [a] + K, K[::-1] + [i])
    t.add_term(-cw.conjugate(), [i] + K, K[::-1] + [a])
    return t


def _pattern_problem(custom, seed):
    mol, pool = random_problem(5, seed, "SD")
    pool2 = qb.SQOpPool()
    for c, op in pool.terms():
        pool2.add_term(c, op)
    base = len(pool2.terms())
    for op in custom:
        pool2.add_term(1.0, op)
    tops = [0]
    for k in range(len(custom)):
        tops += [base + k, 3 + 2 * k]
    return mol, pool2, tops


@pytest.mark.parametrize("case", ["real", "complex"])
def test_multi_pattern_steps_on_the_compact_path(cuda, case):
    """Steps whose Givens form has several active patterns (hops gated by
    number operators on other orbitals: 4 and 8 real patterns, or 4 with
    imaginary coefficients, which the compact path keeps as complex states)
    run on the shared-memory compact path with the pattern number in each
    pair word: energies and gradients equal the oracle's and the full-space
    path's."""
    from qforte_b200.ucc import evaluator_config
    if case == "real":
        custom = [_gated_hop(4, 6, [0, 3], -2.0), _gated_hop(2, 8, [0, 4, 3], -2.0)]
    else:
        custom = [_gated_hop(5, 7, [1, 3], -2.0, 1j), _gated_hop(4, 6, [0, 3], -2.0)]
    mol, pool2, tops = _pattern_problem(custom, 7)
    P = np.random.default_rng(12).uniform(-0.3, 0.3, (3, len(tops)))
    eng = DUCC(mol.hamiltonian, pool2, tops, mol.hf_reference)
    ev = eng.evaluator(3)
    assert ev.path == 2 and ev.real_states is (case == "real")
    E, G = eng.energy_grad(P)
    evaluator_config(False)
    try:
        eng2 = DUCC(mol.hamiltonian, pool2, tops, mol.hf_reference)
        assert eng2.evaluator(3).path != 2
        E2, G2 = eng2.energy_grad(P)
    finally:
        evaluator_config(True)
    assert np.max(np.abs(E - E2)) < 1e-12 and np.max(np.abs(G - G2)) < 1e-11
    hterms = oracle_terms(mol.hamiltonian)
    kf = kops_forward(pool2, tops)
    E_o, _ = O.energy(10, mol.hf_reference, kf, P[1], hterms)
    g_o = O.measure_gradient(10, mol.hf_reference, kf, P[1], hterms,
                             kops_grad=kops_gradient(pool2, tops))
    assert abs(E[1] - E_o) < E_TOL and np.max(np.abs(G[1] - g_o)) < G_TOL


@pytest.mark.parametrize("tile,low", [(0, 3), (-1, 4), (12, 3)])
@pytest.mark.parametrize("n,ngates,seed", [(5, 300, 61), (13, 250, 62), (18, 200, 63)])
def test_complex64_gates_track_complex128(cuda, gate_tiles, tile, low, n, ngates, seed):
    """The complex64 throughput variant of the gate path (tile runs and one
    pass per gate, FP32 arithmetic) against the oracle's complex128 state:
    within FP32 rounding (3e-6 max-abs after a few hundred gates), norm 1
    within 1e-5.  Never used for parity with the reference."""
    from qforte_b200.computer import ComputerC64
    gate_tiles(tile, low)
    circ, ora = _rand_circuit(n, ngates, seed)
    psi0 = _random_state(n, seed)
    qc = ComputerC64(n)
    qc.set_coeff_vec(psi0)
    qc.apply_circuit(circ)
    st = O.State(n, psi0.copy())
    st.apply_gates(ora)
    got = qc.get_coeff_array()
    assert got.dtype == np.complex64
    assert np.max(np.abs(got.astype(np.complex128) - st.psi)) < 3e-6
    assert abs(qc.norm2() - 1.0) < 1e-5
    qc.reset()
    assert qc.get_coeff_array()[0] == 1 and abs(qc.norm2() - 1.0) == 0
    with pytest.raises(ValueError):
        qc.apply_circuit(qb.build_circuit(f"X_{n}"))


@pytest.mark.parametrize("n,kind,seed", [(10, "random", 71), (13, "controls", 72), (16, "random", 73)])
def test_complex64_fused_phases_track_complex128(cuda, n, kind, seed):
    """The complex64 variant with its tile phases fused (products in FP64 on
    the tensor cores, amplitudes rounded to FP32 at each phase's store)
    against the oracle's complex128 state: within FP32 rounding (3e-6)."""
    from qforte_b200.computer import ComputerC64
    from qforte_b200.device import gates_config
    circ, ora = (_rand_circuit(n, 300, seed) if kind == "random"
                 else _control_heavy_circuit(n, seed))
    psi0 = _random_state(n, seed)
    gates_config(0, 3, 0, 0, True)
    try:
        qc = ComputerC64(n)
        qc.set_coeff_vec(psi0)
        qc.apply_circuit(circ)
        got = qc.get_coeff_array()
    finally:
        gates_config()
    st = O.State(n, psi0.copy())
    st.apply_gates(ora)
    assert np.max(np.abs(got.astype(np.complex128) - st.psi)) < 3e-6


@pytest.mark.parametrize("norb,seed,pool_type,B", [(4, 11, "SD", 5), (6, 3, "SD", 2),
                                                   (5, 9, "GSD", 7), (8, 2, "SD", 6)])
def test_two_sets_per_cta_match_one_set(cuda, norb, seed, pool_type, B):
    """Real compact states: the forward program with two parameter sets per
    CTA (one 16-byte slot per amplitude, each set with its own angles; an odd
    batch's last CTA holds one set) gives each set's one-set-per-CTA energies
    and gradients, also when the sweep runs alone on the saved states after an
    energy-only run (mode 2)."""
    import torch
    from qforte_b200.ucc import evaluator_config
    mol, pool = random_problem(norb, seed, pool_type)
    tops = list(range(0, len(pool), 1 if len(pool) < 400 else 3))
    P = np.random.default_rng(norb + B).uniform(-0.1, 0.1, (B, len(tops)))
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type=pool_type)
    ev = eng.evaluator(B)
    assert ev.path == 2 and ev.real_states and ev.sets_per_cta == 2
    E, G = ev.eval(P, True)
    evaluator_config("one-set")
    try:
        eng1 = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference, pool_type=pool_type)
        ev1 = eng1.evaluator(B)
        assert ev1.sets_per_cta == 1
        E1, G1 = ev1.eval(P, True)
    finally:
        evaluator_config(True)
    assert np.max(np.abs(E - E1)) < 1e-12 and np.max(np.abs(G - G1)) < 1e-11
    # energy-only run, then the sweep alone on the saved states
    d_par, d_en, d_gr = ev.tensors()
    d_par.copy_(torch.from_numpy(P))
    ev.run(0)
    ev.run(2)
    torch.cuda.synchronize()
    assert np.max(np.abs(d_gr.cpu().numpy() - G1)) < 1e-11
