"""The differentiable dUCC energy (qforte_b200.autograd): the backward pass is
the adjoint reverse sweep; it must equal the reference's own gradient
(golden vectors of the compiled reference), the oracle's, and central finite
differences of the forward pass (h = 1e-5), at the gradient tolerance 1e-8."""

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import golden
from tests.helpers import kops_forward, kops_gradient, oracle_terms, random_problem

pytestmark = pytest.mark.gpu

E_TOL = 1e-10
G_TOL = 1e-8


@pytest.mark.parametrize("name", ["ucc_norb4_seed11.npz", "ucc_norb6_seed11.npz"])
def test_backward_is_the_reference_gradient(cuda, name):
    import torch
    from qforte_b200.autograd import ucc_energy
    from qforte_b200.ucc import DUCC
    z = golden(name)
    mol, pool = random_problem(int(z["norb"]), int(z["seed"]))
    eng = DUCC(mol.hamiltonian, pool, list(range(len(pool))), mol.hf_reference)
    t = torch.tensor(z["amps"], dtype=torch.float64, requires_grad=True)
    E = ucc_energy(t, eng)
    assert E.dim() == 0 and abs(E.item() - float(z["energy"])) < E_TOL
    E.backward()
    assert t.grad.device.type == "cpu"
    assert np.max(np.abs(t.grad.numpy() - z["grad"])) < G_TOL


def test_backward_batched_weights_and_central_differences(cuda):
    import torch
    from qforte_b200.autograd import ucc_energy
    from qforte_b200.ucc import DUCC
    mol, pool = random_problem(5, 21)
    eng = DUCC(mol.hamiltonian, pool, list(range(len(pool))), mol.hf_reference)
    M = len(pool)
    rng = np.random.default_rng(3)
    P = rng.uniform(-0.1, 0.1, (3, M))
    t = torch.tensor(P, device="cuda", requires_grad=True)
    w = torch.tensor([1.0, -2.0, 0.5], device="cuda", dtype=torch.float64)
    E = ucc_energy(t, eng)
    (w * E).sum().backward()
    g = t.grad.cpu().numpy()
    # oracle gradient of each row
    hterms = oracle_terms(mol.hamiltonian)
    tops = list(range(M))
    for b in range(3):
        g_o = O.measure_gradient(10, mol.hf_reference, kops_forward(pool, tops), P[b], hterms,
                                 kops_grad=kops_gradient(pool, tops))
        assert np.max(np.abs(g[b] - w[b].item() * g_o)) < G_TOL
    # central differences of the forward pass, h = 1e-5, row 0
    h = 1e-5
    Q = np.repeat(P[:1], 2 * M, axis=0)
    for k in range(M):
        Q[2 * k, k] += h
        Q[2 * k + 1, k] -= h
    with torch.no_grad():
        EQ = ucc_energy(torch.tensor(Q, device="cuda"), eng).cpu().numpy()
    fd = (EQ[0::2] - EQ[1::2]) / (2 * h)
    assert np.max(np.abs(fd - g[0])) < G_TOL


def test_backward_after_another_forward_on_the_same_evaluator(cuda):
    """Two graphs share one evaluator: the second forward overwrites the
    states the first backward needs, which then re-runs its forward."""
    import torch
    from qforte_b200.autograd import ucc_energy
    from qforte_b200.ucc import DUCC
    mol, pool = random_problem(4, 11)
    eng = DUCC(mol.hamiltonian, pool, list(range(len(pool))), mol.hf_reference)
    rng = np.random.default_rng(5)
    a = torch.tensor(rng.uniform(-0.1, 0.1, len(pool)), requires_grad=True)
    b = torch.tensor(rng.uniform(-0.1, 0.1, len(pool)), requires_grad=True)
    Ea = ucc_energy(a, eng)
    Eb = ucc_energy(b, eng)
    Ea.backward()
    Eb.backward()
    for x in (a, b):
        _, g = eng.energy_grad(x.detach().numpy())
        assert np.max(np.abs(x.grad.numpy() - g)) < 1e-12
