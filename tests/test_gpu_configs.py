"""GPU parity at the benchmarked configurations themselves, against golden
vectors the compiled reference produced on the same inputs
(tests/golden/make_golden.py, families bench16, grad20, adapt20, sweep20/24/28
and oppl).  Tolerances as everywhere: amplitudes 1e-12 max-abs, energies
1e-10, gradients 1e-8.

* the default benchmark step: 256 parameter sets of the 16-qubit dUCCSD
  problem through the batched evaluator (rows 0 and 255 held to the reference's
  energy_feval and measure_gradient, uccvqeabc.py:122-251);
* the 20-qubit adjoint gradient (875 parameters) through the evaluator and
  through torch.autograd;
* every ADAPT pool gradient of the 20-qubit GSD pool (7,020 operators) in one
  launch, against the reference's measure_gradient3 (uccvqeabc.py:253-283);
* the 100-layer gate sweep at 20, 24 and 28 qubits on the tile path, on one
  pass per gate and in dense 5- and 6-qubit blocks, against the reference's
  apply_circuit (computer.cc:93-114); 32 qubits by norm and inverse;
* direct_oppl_exp_val / direct_idxd_oppl_exp_val (computer.cc:773-806).
"""

import os

import numpy as np
import pytest

import qforte_b200 as qb
from qforte_b200.ucc import DUCC
from tests.conftest import GOLDEN, golden
from tests.helpers import random_problem

pytestmark = pytest.mark.gpu

AMP_TOL = 1e-12
E_TOL = 1e-10
G_TOL = 1e-8


def test_benchmark_batch_rows_match_reference(cuda):
    """The default benchmark step as bench.py runs it: one evaluator of 256
    parameter sets, energies and gradients in one graph replay."""
    z = golden("bench_ucc16_seed11.npz")
    norb, seed, batch = int(z["norb"]), int(z["seed"]), int(z["batch"])
    mol, pool = random_problem(norb, seed)
    assert len(mol.hamiltonian) == int(z["nterms"])
    M = len(pool)
    P = np.random.default_rng(seed + 1).uniform(-0.1, 0.1, (batch, M))
    eng = DUCC(mol.hamiltonian, pool, list(range(M)), mol.hf_reference)
    ev = eng.evaluator(batch)
    E, G = ev.eval(P, True)
    for k, r in enumerate(z["rows"]):
        assert abs(E[r] - z["energies"][k]) < E_TOL, (r, E[r], z["energies"][k])
        assert np.max(np.abs(G[r] - z["grads"][k])) < G_TOL
    # a second replay gives the same numbers (no state carried between steps)
    E2, G2 = ev.eval(P, True)
    assert np.array_equal(E, E2) and np.array_equal(G, G2)


def test_gradient_20_qubits_matches_reference(cuda):
    """Config: adjoint gradient at 20 qubits (10 orbitals, 875 SD parameters),
    through the evaluator and behind torch.autograd."""
    import torch
    from qforte_b200.autograd import ucc_energy
    z = golden("grad_ucc20_seed11.npz")
    norb, seed = int(z["norb"]), int(z["seed"])
    mol, pool = random_problem(norb, seed)
    assert len(mol.hamiltonian) == int(z["nterms"])
    eng = DUCC(mol.hamiltonian, pool, list(range(len(pool))), mol.hf_reference)
    E, G = eng.energy_grad(z["amps"][None, :])
    assert abs(E[0] - float(z["energy"])) < E_TOL
    assert np.max(np.abs(G[0] - z["grad"])) < G_TOL
    t = torch.tensor(z["amps"][None, :], device="cuda", requires_grad=True)
    e = ucc_energy(t, eng)
    e.sum().backward()
    assert abs(float(e.detach()[0]) - float(z["energy"])) < E_TOL
    assert np.max(np.abs(t.grad[0].cpu().numpy() - z["grad"])) < G_TOL


def test_adapt_pool_gradients_20_qubits_match_reference(cuda):
    """Config: all 7,020 GSD pool gradients <psi|[H, A_k]|psi> at 20 qubits in
    one launch, at the 12-operator state of the pool-gradient workload."""
    z = golden("adapt_gsd20_seed11.npz")
    norb, seed = int(z["norb"]), int(z["seed"])
    mol, pool = random_problem(norb, seed, "GSD")
    assert len(pool) == len(z["pool_grads"])
    tops = [int(t) for t in z["tops"]]
    eng = DUCC(mol.hamiltonian, pool, tops, mol.hf_reference)
    g = eng.pool_gradients(z["amps"])
    assert np.max(np.abs(g - z["pool_grads"])) < G_TOL
    # the same selection: the operator ADAPT would add next
    assert int(np.argmax(np.abs(g))) == int(np.argmax(np.abs(z["pool_grads"])))


def _sweep_cases():
    out = []
    for n in (20, 24, 28):
        if os.path.exists(os.path.join(GOLDEN, f"sweep{n}_seed{11 + n}.npz")):
            for tile, dense in ((0, 0), (-1, 0), (0, 5), (0, 6)):
                out.append((n, tile, dense, None))
            out.append((n, 0, 0, False))  # tile phases gate by gate at every size
            out.append((n, 0, 0, True))   # tile phases fused at every size
    return out


@pytest.fixture
def restore_gates_config():
    from qforte_b200.device import gates_config
    yield gates_config
    gates_config(0, 3, 0, 0)


@pytest.mark.parametrize("n,tile,dense,fused", _sweep_cases())
def test_gate_sweep_matches_reference(cuda, restore_gates_config, n, tile, dense, fused):
    """Config: the 100-layer random gate sweep on the register-blocked tile
    path (tile 0; its phases in the default form, gate by gate, and fused into
    8 x 8 matrices on the FP64 tensor cores), on one pass per gate (tile -1)
    and in dense 5- and 6-qubit blocks on the FP64 tensor cores: sampled
    amplitudes at 1e-12, the norm, <Z_k> of every qubit and the mass of each
    value of the top 8 qubits against the reference's state."""
    from qforte_b200.workloads import layered_random_circuit
    z = golden(f"sweep{n}_seed{11 + n}.npz")
    restore_gates_config(tile, 3, 0, dense, fused)
    circ, spec = layered_random_circuit(n, int(z["layers"]), int(z["seed"]))
    assert len(spec) == int(z["ngates"])
    qc = qb.Computer(n)
    qc.apply_circuit(circ)
    psi = qc.get_coeff_array()
    del qc
    assert np.max(np.abs(psi[z["idx"]] - z["amps"])) < AMP_TOL
    prob = psi.real ** 2 + psi.imag ** 2
    assert abs(np.sqrt(prob.sum()) - float(z["norm"])) < AMP_TOL
    zk = np.array([prob.reshape(-1, 2, 1 << k)[:, 0, :].sum() -
                   prob.reshape(-1, 2, 1 << k)[:, 1, :].sum() for k in range(n)])
    assert np.max(np.abs(zk - z["z"])) < AMP_TOL
    assert np.max(np.abs(prob.reshape(256, -1).sum(axis=1) - z["top8"])) < AMP_TOL


def test_operator_pool_expectation_values_match_reference(cuda):
    """direct_oppl_exp_val and direct_idxd_oppl_exp_val (computer.cc:773-806)
    of the commutator pool [H, A_k] (UCCVQE.fill_commutator_pool) at a
    3-operator dUCC state prepared on the device."""
    from qforte_b200.ucc import ADAPTVQE
    z = golden("oppl_norb4_seed11.npz")
    norb, seed = int(z["norb"]), int(z["seed"])
    mol, pool = random_problem(norb, seed, "GSD")
    drv = ADAPTVQE(mol, engine="percall")
    drv._pool_obj = pool
    drv._tops, drv._tamps = [int(t) for t in z["tops"]], list(z["amps"])
    qc = qb.Computer(2 * norb)
    qc.apply_circuit(drv.build_Uvqc())
    assert np.max(np.abs(qc.get_coeff_array() - z["psi"])) < AMP_TOL
    comm = pool.get_qubit_op_pool()
    comm.join_as_commutator(mol.hamiltonian)
    vals = np.array(qc.direct_oppl_exp_val(comm))
    assert vals.shape == z["oppl"].shape
    assert np.max(np.abs(vals - z["oppl"])) < E_TOL
    ivals = np.array(qc.direct_idxd_oppl_exp_val(comm, [int(i) for i in z["idxs"]]))
    assert np.max(np.abs(ivals - z["idxd_oppl"])) < E_TOL
    # the state is left as it was (the reference restores coeff_, computer.cc:796-803)
    assert np.max(np.abs(qc.get_coeff_array() - z["psi"])) < AMP_TOL


def test_gate_sweep_32_qubits_norm_and_inverse(cuda, restore_gates_config):
    """Config: the gate sweep at its largest size, one 32-qubit complex128
    state (64 GiB) worked in place.  Neither the oracle nor the reference can
    hold it (the reference needs 40 bytes an amplitude and overflows 32-bit
    loop counters there, computer.cc:637-643), so the checks are
    size-independent: after 10 layers the norm is 1 within 1e-12, and the
    adjoint circuit returns |0...0> within 1e-12, on the tile runs (phases
    fused and gate by gate) and on dense 5-qubit blocks."""
    import torch
    from qforte_b200.workloads import layered_random_circuit
    free, _ = torch.cuda.mem_get_info()
    if free < 70 * 2 ** 30:
        pytest.skip("needs 64 GiB of free device memory")
    n = 32
    circ, spec = layered_random_circuit(n, 10, 43)
    inv = circ.adjoint()
    qc = qb.Computer(n)
    try:
        for tile, dense, fused in ((0, 0, None), (0, 0, False), (0, 5, None)):
            restore_gates_config(tile, 3, 0, dense, fused)
            qc.reset()
            qc.apply_circuit(circ)
            assert abs(qb.inner_product(qc, qc) - 1.0) < AMP_TOL
            assert abs(qc.coeff(0)) < 1.0
            qc.apply_circuit(inv)
            assert abs(qc.coeff(0) - 1.0) < AMP_TOL
            assert abs(qb.inner_product(qc, qc) - 1.0) < AMP_TOL
    finally:
        del qc
