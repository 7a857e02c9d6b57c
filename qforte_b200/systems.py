"""Molecular systems: seeded random-integral Hamiltonians and JSON integrals.

``random_molecule(norb, nel, seed)`` builds the synthetic electronic
Hamiltonian used by every workload here: one-electron integrals h symmetric
with h_pp ~ U(-2, -0.5) and h_pq ~ N(0, 0.1); two-electron integrals
g_pqrs = sum_{l=1..6} L^l_pq L^l_rs with each L^l symmetric N(0, 0.1), which
gives the 8-fold permutational symmetry of real chemist-notation integrals
and a positive semidefinite g; E_nuc = 0.  The second-quantised operator is
assembled by the loop of ``create_psi_mol`` (adapters/molecule_adapters.py:
182-210, no frozen orbitals) and mapped with ``jw_transform``.

``create_external_mol`` reads the reference's JSON integral format
(adapters/molecule_adapters.py:232-297) and ``system_factory`` dispatches to
it (system/system_factory.py:5-57).
"""

import json

import numpy as np

from .sq_operator import SQOperator

__all__ = ["Molecule", "create_TFIM", "random_integrals", "random_molecule", "sq_hamiltonian",
           "create_external_mol", "system_factory", "hf_reference"]


class Molecule:
    """Holder of a system's Hamiltonian and reference (system/molecular_info.py)."""

    def __init__(self, **kw):
        self.multiplicity = kw.get("multiplicity", 1)
        self.charge = kw.get("charge", 0)
        self.filename = kw.get("filename", "")
        self.hamiltonian = None
        self.sq_hamiltonian = None
        self.hf_reference = None
        self.nuclear_repulsion_energy = 0.0
        self.hf_energy = 0.0
        self.point_group = ["C1", ["A"]]
        self.orb_irreps = []
        self.orb_irreps_to_int = []


def random_integrals(norb, seed, nfactor=6):
    rng = np.random.default_rng(seed)
    h = rng.normal(0.0, 0.1, size=(norb, norb))
    h = np.triu(h, 1)
    h = h + h.T
    h[np.diag_indices(norb)] = rng.uniform(-2.0, -0.5, size=norb)
    g = np.zeros((norb,) * 4)
    for _ in range(nfactor):
        L = rng.normal(0.0, 0.1, size=(norb, norb))
        L = np.triu(L) + np.triu(L, 1).T
        g += np.einsum("pq,rs->pqrs", L, L)
    return h, g


def hf_reference(norb, nel):
    return [1] * nel + [0] * (2 * norb - nel)


def sq_hamiltonian(h, g, e_nuc=0.0):
    """The create_psi_mol assembly loop (molecule_adapters.py:182-210)."""
    norb = h.shape[0]
    Hsq = SQOperator()
    Hsq.add(e_nuc, [], [])
    for i in range(norb):
        ia, ib = 2 * i, 2 * i + 1
        for j in range(norb):
            ja, jb = 2 * j, 2 * j + 1
            Hsq.add(h[i, j], [ia], [ja])
            Hsq.add(h[i, j], [ib], [jb])
            for k in range(norb):
                ka, kb = 2 * k, 2 * k + 1
                for l in range(norb):
                    la, lb = 2 * l, 2 * l + 1
                    v = g[i, l, k, j] / 2
                    if ia != jb and kb != la:
                        Hsq.add(v, [ia, jb], [kb, la])
                    if ib != ja and ka != lb:
                        Hsq.add(v, [ib, ja], [ka, lb])
                    if ia != ja and ka != la:
                        Hsq.add(v, [ia, ja], [ka, la])
                    if ib != jb and kb != lb:
                        Hsq.add(v, [ib, jb], [kb, lb])
    return Hsq


def random_molecule(norb, nel=None, seed=0):
    """A Molecule with the seeded random-integral Hamiltonian; half filling
    by default."""
    if nel is None:
        nel = norb
    h, g = random_integrals(norb, seed)
    mol = Molecule()
    mol.sq_hamiltonian = sq_hamiltonian(h, g, 0.0)
    mol.hamiltonian = mol.sq_hamiltonian.jw_transform()
    mol.hf_reference = hf_reference(norb, nel)
    mol.orb_irreps_to_int = [0] * norb
    mol.orb_irreps = ["A"] * norb
    mol.one_body = h
    mol.two_body = g
    return mol


def create_external_mol(**kwargs):
    """JSON integral file -> Molecule (molecule_adapters.py:232-297)."""
    mol = Molecule(multiplicity=kwargs.get("multiplicity", 1), charge=kwargs.get("charge", 0),
                   filename=kwargs["filename"])
    with open(kwargs["filename"]) as f:
        data = json.load(f)
    try:
        pg = data["point_group"]["data"]
    except KeyError:
        pg = "C1"
    if pg != "C1":
        raise NotImplementedError("only C1 integral files are supported")
    nso = int(data["nso"]["data"])
    mol.point_group = ["C1", ["A"]]
    mol.orb_irreps = ["A"] * (nso // 2)
    mol.orb_irreps_to_int = [0] * (nso // 2)
    H = SQOperator()
    H.add(data["scalar_energy"]["data"], [], [])
    for p, q, hpq in data["oei"]["data"]:
        H.add(hpq, [p], [q])
    for p, q, r, s, v in data["tei"]["data"]:
        H.add(v / 4.0, [p, q], [s, r])
    ref = [0] * nso
    for a in range(data["na"]["data"]):
        ref[a * 2] = 1
    for b in range(data["nb"]["data"]):
        ref[b * 2 + 1] = 1
    mol.hf_reference = ref
    mol.sq_hamiltonian = H
    mol.hamiltonian = H.jw_transform()
    return mol


def create_TFIM(n, h, J):
    """1D transverse-field Ising model with open boundaries
    (adapters/model_adapters.py:5-31): H = -h sum_i Z_i - J sum_i X_i X_{i+1},
    reference |0...0>."""
    from .qubit_operator import QubitOperator
    from .utils import build_circuit
    tfim = Molecule()
    tfim.hamiltonian = QubitOperator()
    terms = [(-h, f"Z_{i}") for i in range(n)] + [(-J, f"X_{i} X_{i + 1}") for i in range(n - 1)]
    for coeff, op_str in terms:
        tfim.hamiltonian.add(coeff, build_circuit(op_str))
    tfim.hf_reference = [0] * n
    return tfim


def system_factory(system_type="molecule", build_type="external", **kwargs):
    """system/system_factory.py:5-57: molecules from external integrals (or,
    here, seeded random integrals; psi4 is not available) and the TFIM model."""
    if system_type == "model":
        if build_type != "TFIM":
            raise TypeError(f"build type {build_type} not supported, supported types are: TFIM")
        return create_TFIM(**kwargs)
    if system_type != "molecule":
        raise TypeError("system type not supported, supported types are 'molecule' and 'model'.")
    if build_type == "external":
        return create_external_mol(**kwargs)
    if build_type == "random":
        return random_molecule(kwargs["norb"], kwargs.get("nel"), kwargs.get("seed", 0))
    raise TypeError(f"build type {build_type} not supported, supported types are: external, "
                    "random")
