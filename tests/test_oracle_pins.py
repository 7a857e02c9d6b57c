"""The oracle is pinned before it is trusted: its CPU restatement of the
reference's algorithms must reproduce golden vectors that the compiled
reference produced (tests/golden/make_golden.py) and the known answers of the
reference's own tests."""

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import golden
from tests.helpers import kops_forward, kops_gradient, oracle_terms_from_arrays, random_problem


def _ucc_inputs(z, pool_type="SD"):
    norb = int(z["norb"])
    mol, pool = random_problem(norb, int(z["seed"]), pool_type)
    hterms = oracle_terms_from_arrays(z["ham_c"], z["ham_x"], z["ham_z"])
    return mol, pool, hterms


@pytest.mark.parametrize("name", ["ucc_norb4_seed11.npz", "ucc_norb6_seed11.npz"])
def test_oracle_energy_state_gradient(name):
    z = golden(name)
    mol, pool, hterms = _ucc_inputs(z)
    nq = int(z["nqubit"])
    tops = list(range(len(pool)))
    amps = z["amps"]
    E, st = O.energy(nq, list(z["ref"]), kops_forward(pool, tops), amps, hterms)
    assert abs(E - float(z["energy"])) < 1e-12
    assert np.max(np.abs(st.psi - z["psi"])) < 1e-13
    g = O.measure_gradient(nq, list(z["ref"]), kops_forward(pool, tops), amps, hterms,
                           kops_grad=kops_gradient(pool, tops))
    assert np.max(np.abs(g - z["grad"])) < 1e-11


def test_oracle_pool_gradients_norb4():
    z = golden("ucc_norb4_seed11.npz")
    mol, gsd, hterms = _ucc_inputs(z, "GSD")
    nq = int(z["nqubit"])
    tops = [int(t) for t in z["gsd_tops"]]
    g = O.measure_gradient3(nq, list(z["ref"]), kops_forward(gsd, tops), z["gsd_amps"], hterms,
                            kops_gradient(gsd, range(len(gsd))))
    assert np.max(np.abs(g - z["pool_grads"])) < 1e-11


@pytest.mark.parametrize("name", ["ucc_norb4_seed11.npz", "ucc_norb6_seed11.npz"])
def test_oracle_spin_adapted_pool(name):
    z = golden(name)
    mol, pool, hterms = _ucc_inputs(z, "sa_SD")
    nq = int(z["nqubit"])
    tops = list(range(len(pool)))
    amps = z["sa_amps"]
    kf = kops_forward(pool, tops, "sa_SD")
    E, _ = O.energy(nq, list(z["ref"]), kf, amps, hterms)
    assert abs(E - float(z["sa_energy"])) < 1e-12
    g = O.measure_gradient(nq, list(z["ref"]), kf, amps, hterms,
                           kops_grad=kops_gradient(pool, tops), kops_unrot=kf)
    assert np.max(np.abs(g - z["sa_grad"])) < 1e-11


def test_oracle_gates_bitexact():
    z = golden("gates_n6.npz")
    st = O.State(int(z["n"]))
    gates = [O.make_gate(str(k), int(t), int(c), float(p))
             for k, t, c, p in zip(z["kinds"], z["target"], z["control"], z["param"])]
    st.apply_gates(gates)
    # same algorithm, same operation order: bit-identical amplitudes
    assert np.array_equal(st.psi, z["psi"])


def test_oracle_trotter_known_answer():
    """tests/test_trotter.py:15-47 of the reference (tolerance 1e-15)."""
    terms = [(-1.0j * 0.5, []), (-1.0j * -0.04544288414432624, [("Z", 0)])]
    gates, phase = O.trotterize(terms)
    st = O.State(4)
    st.psi[:] = 0
    st.psi[3] = np.sqrt(2 / 3)
    st.psi[12] = -np.sqrt(1 / 3)
    st.apply_gates(gates)
    st.apply_constant(phase)
    c = st.psi
    assert abs(c[3].real - 0.6980209737879599) < 1e-15
    assert abs(c[3].imag - -0.423595782342996) < 1e-15
    assert abs(c[12].real - -0.5187235657531178) < 1e-15
    assert abs(c[12].imag - 0.25349397560041553) < 1e-15


def test_oracle_operator_expval():
    z = golden("gates_n6.npz")
    st = O.State(int(z["n"]), z["psi"])
    op = [(0.5, [("X", 0), ("Z", 2)]), (0.3j, [("Y", 1), ("X", 3)]), (-0.7, [("Z", 0), ("Z", 5)]),
          (0.2, [("X", 1), ("X", 1)]), (0.1, [("Y", 2), ("Z", 2), ("X", 4)]), (-0.25j, [("Z", 3)])]
    s2 = st.copy()
    s2.apply_pauli_operator(op)
    assert np.array_equal(s2.psi, z["op_psi"])
    assert st.direct_op_exp_val(op) == complex(z["op_expval"])


@pytest.mark.parametrize("name", ["pqe_norb4_seed11.npz", "pqe_norb6_seed11.npz"])
def test_oracle_pqe_residuals(name):
    """The oracle's restatement of UCCNPQE.get_residual_vector reproduces the
    reference's residuals at the same amplitudes (uccnpqe.py:249-292)."""
    z = golden(name)
    u = golden(name.replace("pqe_", "ucc_"))
    mol, pool, hterms = _ucc_inputs(u)
    nq = int(u["nqubit"])
    tops = list(range(len(pool)))
    dets = list(zip(z["dets"].tolist(), z["phases"].tolist()))
    r = O.pqe_residuals(nq, list(u["ref"]), kops_forward(pool, tops), z["amps"], hterms, dets)
    assert np.max(np.abs(r - z["residuals"])) < 1e-12


@pytest.mark.parametrize("key", ["SD_fe", "SD_qe", "GSD_fe", "sa_SD_qe"])
def test_oracle_applies_compact_circuits_as_the_reference(key):
    """The oracle's gate kernels give the reference's state for the compact
    ansatz circuits (fixtures from the reference's builder)."""
    z = golden("compact_norb4.npz")
    gates = [O.make_gate("X", j, j) for j in range(4)]
    ids, tg, ct, pr = (z[f"{key}_{f}"] for f in ("ids", "target", "control", "param"))
    gates += [O.make_gate(str(k), int(t), int(c), float(p)) for k, t, c, p in zip(ids, tg, ct, pr)]
    st = O.State(8)
    st.apply_gates(gates)
    assert np.max(np.abs(st.psi - z[f"{key}_psi"])) < 1e-13


def test_oracle_sampler_frequencies():
    """The oracle's seeded sampler draws with the state's probabilities
    (chi-square on a 5-qubit state) and is a function of the seed."""
    rng = np.random.default_rng(3)
    psi = rng.normal(size=32) + 1j * rng.normal(size=32)
    psi /= np.linalg.norm(psi)
    shots = 40000
    idx = O.sample_indices(psi, 11, shots)
    counts = np.bincount(idx.astype(np.int64), minlength=32)
    expect = shots * np.abs(psi) ** 2
    chi2 = float(np.sum((counts - expect) ** 2 / expect))
    assert chi2 < 80.0  # 31 degrees of freedom: p < 1e-5 above 70
    assert np.array_equal(idx, O.sample_indices(psi, 11, shots))
    assert not np.array_equal(idx[:100], O.sample_indices(psi, 12, 100))
