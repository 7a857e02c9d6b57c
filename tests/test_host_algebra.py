"""Host-side object model vs the reference: gate factory, circuits, operator
algebra, Jordan-Wigner, pools.  Term order and coefficients must be the
reference's exactly (they fix the Trotter order of the ansatz)."""

import math

import numpy as np
import pytest

import qforte_b200 as qb
from qforte_b200.pauli import letters
from tests.conftest import golden
from tests.helpers import random_problem


def _arrays(qo):
    c, x, z = [], [], []
    for cc, circ in qo.terms():
        m = circ._pauli_masks()
        assert m is not None and m[2] == 0
        c.append(complex(cc))
        x.append(m[0])
        z.append(m[1])
    return np.array(c), np.array(x, dtype=np.uint64), np.array(z, dtype=np.uint64)


@pytest.mark.parametrize("name", ["ucc_norb4_seed11.npz", "ucc_norb6_seed11.npz"])
def test_jw_hamiltonian_matches_reference(name):
    z = golden(name)
    mol, _ = random_problem(int(z["norb"]), int(z["seed"]))
    c, x, zz = _arrays(mol.hamiltonian)
    assert len(c) == len(z["ham_c"])
    assert np.array_equal(x, z["ham_x"]) and np.array_equal(zz, z["ham_z"])
    assert np.array_equal(c, z["ham_c"])  # bit-identical coefficients


@pytest.mark.parametrize("pt", ["SD", "GSD", "sa_SD", "SDTQ"])
def test_pools_match_reference(pt):
    z = golden("pools_norb4.npz")
    ref = [1] * 4 + [0] * 4
    pool = qb.SQOpPool()
    pool.set_orb_spaces(ref)
    pool.fill_pool(pt)
    owner = z[f"{pt}_owner"]
    assert len(pool) == int(owner.max()) + 1
    k = 0
    for i, (c, op) in enumerate(pool):
        for coeff, cre, ann in op.terms():
            assert owner[k] == i
            assert complex(coeff) == complex(z[f"{pt}_coeff"][k])
            assert cre == [int(v) for v in z[f"{pt}_cre"][k] if v >= 0]
            assert ann == [int(v) for v in z[f"{pt}_ann"][k] if v >= 0]
            k += 1
    assert k == len(owner)
    if pt != "sa_SD":
        amps = z[f"{pt}_amps"]
        tmp = qb.SQOpPool()
        for t, (c, op) in zip(amps, pool):
            tmp.add(t, op)
        A = tmp.get_qubit_operator("commuting_grp_lex")
        c, x, zz = _arrays(A)
        assert np.array_equal(x, z[f"{pt}_A_x"]) and np.array_equal(zz, z[f"{pt}_A_z"])
        assert np.array_equal(c, z[f"{pt}_A_c"])


def test_gate_factory_semantics():
    # parameter normalisation (make_gate.cc:7-16; tests/test_gates.py test_param_gate)
    g = qb.gate("cRz", 0, 1, 9 * math.pi / 2)
    assert abs(g.parameter() - math.pi / 2) < 1e-14
    assert qb.gate("Rx", 0, 7.0).parameter() == pytest.approx(7.0 - 4 * math.pi)
    with pytest.raises(ValueError):
        qb.gate("Rx", 0, 0)  # the (type, target, control) overload refuses parameter gates
    with pytest.raises(ValueError):
        qb.gate("Q", 0)
    with pytest.raises(ValueError):
        qb.gate("X", 0, 1j)
    assert qb.gate("X", 2).str() == "X2" and qb.gate("cX", 1, 0).str() == "cX1_0"
    # adjoint rules (gate.cc:135-179)
    assert qb.gate("T", 0).adjoint().gate_id() == "R"
    assert qb.gate("S", 0).adjoint().parameter() == pytest.approx(-math.pi / 2)
    assert qb.gate("V", 0).adjoint().gate_id() == "adj(V)"
    assert qb.gate("V", 0).adjoint().adjoint().gate_id() == "V"
    assert qb.gate("Rz", 0, 0.3).adjoint().parameter() == pytest.approx(-0.3)
    assert qb.gate("A", 0, 1, 0.3).adjoint().parameter() == pytest.approx(0.3)


def test_circuit_and_operator_basics():
    c = qb.build_circuit("X_0 Y_1 cX_2_0 Rz_1_0.5")
    assert c.size() == 4 and c.get_num_cnots() == 1 and c.num_qubits() == 3
    assert c.str() == "[Rz1 cX2_0 Y1 X0]"
    assert c.get_parameters() == [0.5]
    a = c.adjoint()
    assert [g.gate_id() for g in a.gates()] == ["Rz", "cX", "Y", "X"]
    # canonicalisation: left-to-right product, X.Y = iZ (circuit.cc:120-132)
    p = qb.build_circuit("X_0 Y_0 Z_1")
    assert p.canonicalize_pauli_circuit() == 1j and p.str() == "[Z1 Z0]"
    op = qb.build_operator("0.5, X_0 X_1; 0.25, Z_0; 0.5, X_0 X_1; 1e-13, Y_3")
    op.simplify()
    assert [(c, circ.str()) for c, circ in op.terms()] == [(1.0 + 0j, "[X1 X0]"),
                                                           (0.25 + 0j, "[Z0]")]
    l = qb.build_operator("1.0, X_0")
    r = qb.build_operator("1.0, Y_0")
    l.operator_product(r)
    assert [(c, circ.str()) for c, circ in l.terms()] == [(1j, "[Z0]")]
    assert qb.QubitBasis(5).str(4) == "|1010>"


def test_jw_small_known_answer(ref_qforte):
    """tests/test_jw_transform.py-style check against the live reference."""
    qf = ref_qforte
    for cre, ann in (([2, 3], [4, 6]), ([1], [2]), ([3, 1], [2, 0]), ([5], []), ([], [4])):
        a = qf.SQOperator()
        a.add(1.5 + 0.25j, cre, ann)
        a.add(-0.5, ann[::-1], cre[::-1])
        b = qb.SQOperator()
        b.add(1.5 + 0.25j, cre, ann)
        b.add(-0.5, ann[::-1], cre[::-1])
        qa, qb_ = a.jw_transform(), b.jw_transform()
        ta = [(complex(c), circ.str()) for c, circ in qa.terms()]
        tb = [(complex(c), circ.str()) for c, circ in qb_.terms()]
        assert ta == tb


@pytest.mark.parametrize("name", ["pqe_norb4_seed11.npz", "pqe_norb6_seed11.npz"])
def test_excited_determinants_match_reference(name):
    """UCCNPQE.fill_excited_dets (uccnpqe.py:193-247): the same determinants
    and phase factors as the reference, computed on the host."""
    from qforte_b200.ucc import excited_determinants
    z = golden(name)
    mol, pool = random_problem(int(z["norb"]), int(z["seed"]))
    ex = excited_determinants(pool, range(len(pool)), mol.hf_reference)
    assert [d for d, _ in ex] == z["dets"].tolist()
    assert np.max(np.abs(np.array([p for _, p in ex]) - z["phases"])) == 0.0


def _compact_ops(pool_type, norb=4):
    from qforte_b200.ucc import _sa_components
    ref = [1] * norb + [0] * norb
    pool = qb.SQOpPool()
    pool.set_orb_spaces(ref)
    pool.fill_pool(pool_type)
    if pool_type == "sa_SD":
        return [c for _, op in pool for c in _sa_components(op)]
    return [op for _, op in pool]


@pytest.mark.parametrize("pool_type", ["SD", "GSD", "sa_SD"])
@pytest.mark.parametrize("qe", [False, True])
def test_compact_excitation_circuits_match_reference(pool_type, qe):
    """utils/compact_excitation_circuits.py:9-291: every pool operator's FEB /
    QEB circuit has the reference's gates, targets, controls and angles."""
    z = golden("compact_norb4.npz")
    key = f"{pool_type}_{'qe' if qe else 'fe'}"
    ops = _compact_ops(pool_type)
    amps = z[f"{pool_type}_amps"]
    ids, tg, ct, pr = [], [], [], []
    U = qb.Circuit()
    for t, op in zip(amps, ops):
        e = op.terms()[1]
        circ = qb.compact_excitation_circuit(t * e[0], e[1], e[2], qe)
        U.add(circ)
        for g in circ.gates():
            ids.append(g.gate_id())
            tg.append(g.target())
            ct.append(g.control())
            pr.append(float(g.parameter()) if g.has_parameter() else 0.0)
    assert ids == z[f"{key}_ids"].tolist()
    assert tg == z[f"{key}_target"].tolist() and ct == z[f"{key}_control"].tolist()
    assert pr == z[f"{key}_param"].tolist()
    assert U.get_num_cnots() == int(z[f"{key}_cnots"])


def test_tfim_model_matches_reference(ref_qforte):
    """system_factory(system_type="model", build_type="TFIM") builds the
    reference's transverse-field Ising Hamiltonian (adapters/model_adapters.py:
    5-31): same terms in the same order, same reference determinant."""
    import qforte_b200 as qb
    from qforte.adapters.model_adapters import create_TFIM
    for n, h, J in ((4, 1.0, 0.5), (7, 0.3, -1.2)):
        ours = qb.system_factory(system_type="model", build_type="TFIM", n=n, h=h, J=J)
        ref = create_TFIM(n, h, J)
        assert ours.hf_reference == ref.hf_reference
        a = [(complex(c), [(g.gate_id(), g.target()) for g in circ.gates()])
             for c, circ in ours.hamiltonian.terms()]
        b = [(complex(c), [(g.gate_id(), g.target()) for g in circ.gates()])
             for c, circ in ref.hamiltonian.terms()]
        assert a == b
