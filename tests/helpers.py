"""Shared builders for the tests: golden arrays -> product objects and oracle
term lists."""

import numpy as np

import qforte_b200 as qb
from qforte_b200.circuit import Circuit
from qforte_b200.pauli import letters
from qforte_b200.qubit_operator import QubitOperator


def qo_from_arrays(c, x, z):
    qo = QubitOperator()
    for cc, xx, zz in zip(c, x, z):
        qo._t.append([complex(cc), Circuit._from_masks(int(xx), int(zz))])
    return qo


def oracle_terms(qo):
    """Product QubitOperator -> oracle Pauli term list [(c, [(letter, q)...])]."""
    out = []
    for c, circ in qo.terms():
        m = circ._pauli_masks()
        assert m is not None and m[2] == 0
        out.append((complex(c), letters(m[0], m[1])))
    return out


def oracle_terms_from_arrays(c, x, z):
    return [(complex(cc), letters(int(xx), int(zz))) for cc, xx, zz in zip(c, x, z)]


def kops_forward(pool, tops, pool_type=None):
    """Per-operator ordered JW term lists of the ansatz (oracle input); an
    sa_SD operator contributes its component excitations in turn
    (abc/ansatz.py:38-55)."""
    from qforte_b200.ucc import _sa_components
    out = []
    for top in tops:
        comps = _sa_components(pool[top][1]) if pool_type == "sa_SD" else [pool[top][1]]
        terms = []
        for comp in comps:
            s = qb.SQOperator()
            s.add_op(comp)
            q = s.jw_transform()
            q.simplify()
            q.order_terms()
            terms += oracle_terms(q)
        out.append(terms)
    return out


def kops_gradient(pool, tops):
    out = []
    for top in tops:
        c, op = pool[top]
        s = qb.SQOperator()
        s.add_op(op)
        q = s.jw_transform()
        q.mult_coeffs(c)
        out.append(oracle_terms(q))
    return out


def random_problem(norb, seed, pool_type="SD"):
    mol = qb.random_molecule(norb, norb, seed)
    pool = qb.SQOpPool()
    pool.set_orb_spaces(mol.hf_reference)
    pool.fill_pool(pool_type)
    return mol, pool


def sq_from_integrals(z):
    """The external-integral SQ Hamiltonian (molecule_adapters.py:273-283)."""
    H = qb.SQOperator()
    H.add(float(z["scalar"]), [], [])
    for p, q, v in z["oei"]:
        H.add(v, [int(p)], [int(q)])
    for p, q, r, s, v in z["tei"]:
        H.add(v / 4.0, [int(p), int(q)], [int(s), int(r)])
    nso = int(z["nso"])
    ref = [0] * nso
    for a in range(int(z["na"])):
        ref[2 * a] = 1
    for b in range(int(z["nb"])):
        ref[2 * b + 1] = 1
    return H, ref
