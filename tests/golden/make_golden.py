"""Generate the golden fixtures of tests/golden from the reference itself.

Run in a container that holds the reference sources (read where they lie) and
its compiled module (``make -C oracle ref``):

    python tests/golden/make_golden.py [--ref-src DIR] [--only FAMILY]

DIR defaults to $QFORTE_REF_SRC, else /root/reference/src/qforte.

Every output comes from the reference's own code path -- its C++ ``Computer``,
``SQOperator.jw_transform``, ``SQOpPool`` and its Python UCC drivers -- on
seeded synthetic inputs.  Integral files of the reference's tests are read
and stored as second-quantised term arrays (the test data the FCI pins in
tests/test_gpu_drivers.py refer to).
"""

import argparse
import json
import math
import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
warnings.filterwarnings("ignore")

from oracle import oracle as O  # noqa: E402
from qforte_b200.systems import hf_reference, random_integrals  # noqa: E402


def pauli_arrays(qo):
    """(coeff, x, z) arrays of a reference QubitOperator, circuits read as
    left-to-right products of single-qubit Paulis on distinct qubits."""
    c, xs, zs = [], [], []
    for coeff, circ in qo.terms():
        x = z = 0
        for g in circ.gates():
            b = 1 << g.target()
            lab = g.gate_id()
            if lab in ("X", "Y"):
                x |= b
            if lab in ("Y", "Z"):
                z |= b
        c.append(complex(coeff))
        xs.append(x)
        zs.append(z)
    return (np.array(c, dtype=np.complex128), np.array(xs, dtype=np.uint64),
            np.array(zs, dtype=np.uint64))


def sq_arrays(sqop):
    """Flatten SQOperator terms: coeff, cre/ann index lists padded with -1."""
    terms = sqop.terms()
    n = len(terms)
    coeff = np.array([complex(t[0]) for t in terms], dtype=np.complex128)
    w = max([len(t[1]) for t in terms] + [len(t[2]) for t in terms] + [1])
    cre = -np.ones((n, w), dtype=np.int32)
    ann = -np.ones((n, w), dtype=np.int32)
    for k, t in enumerate(terms):
        cre[k, :len(t[1])] = t[1]
        ann[k, :len(t[2])] = t[2]
    return coeff, cre, ann


def ref_sq_ham(qf, h, g):
    norb = h.shape[0]
    H = qf.SQOperator()
    H.add(0.0, [], [])
    for i in range(norb):
        ia, ib = 2 * i, 2 * i + 1
        for j in range(norb):
            ja, jb = 2 * j, 2 * j + 1
            H.add(h[i, j], [ia], [ja])
            H.add(h[i, j], [ib], [jb])
            for k in range(norb):
                ka, kb = 2 * k, 2 * k + 1
                for l in range(norb):
                    la, lb = 2 * l, 2 * l + 1
                    v = g[i, l, k, j] / 2
                    if ia != jb and kb != la:
                        H.add(v, [ia, jb], [kb, la])
                    if ib != ja and ka != lb:
                        H.add(v, [ib, ja], [ka, lb])
                    if ia != ja and ka != la:
                        H.add(v, [ia, ja], [ka, la])
                    if ib != jb and kb != lb:
                        H.add(v, [ib, jb], [kb, lb])
    return H


class _Sys:
    pass


def make_alg(qf, H, ref, pool_type):
    s = _Sys()
    s.hamiltonian = H
    s.hf_reference = ref
    s.hf_energy = 0.0
    alg = qf.UCCNVQE(s)
    alg._pool_type = pool_type
    alg.fill_pool()
    return alg


def ucc_fixture(qf, norb, seed, out):
    h, g = random_integrals(norb, seed)
    H = ref_sq_ham(qf, h, g).jw_transform()
    ref = hf_reference(norb, norb)
    nq = 2 * norb
    hc, hx, hz = pauli_arrays(H)
    rng = np.random.default_rng(1000 + seed)
    # dUCCSD: every SD operator, amplitudes U(-0.1, 0.1)
    alg = make_alg(qf, H, ref, "SD")
    M = len(alg._pool_obj)
    amps = rng.uniform(-0.1, 0.1, M)
    alg._tops = list(range(M))
    alg._tamps = list(amps)
    E = alg.energy_feval(list(amps))
    qc = qf.Computer(nq)
    qc.apply_circuit(alg.build_Uvqc(list(amps)))
    psi = np.array(qc.get_coeff_vec())
    grad = np.array(alg.measure_gradient(list(amps)))
    # ADAPT pool gradients: GSD pool, 12 operators drawn from it
    algg = make_alg(qf, H, ref, "GSD")
    P = len(algg._pool_obj)
    tops = [int(t) for t in rng.choice(P, 12, replace=False)]
    gamps = rng.uniform(-0.1, 0.1, 12)
    algg._tops = tops
    algg._tamps = list(gamps)
    pool_grads = np.array(algg.measure_gradient3())
    # spin-adapted pool: multi-excitation operators (abc/ansatz.py:38-55)
    alsa = make_alg(qf, H, ref, "sa_SD")
    S = len(alsa._pool_obj)
    sa_amps = rng.uniform(-0.1, 0.1, S)
    alsa._tops = list(range(S))
    alsa._tamps = list(sa_amps)
    sa_E = alsa.energy_feval(list(sa_amps))
    sa_grad = np.array(alsa.measure_gradient(list(sa_amps)))
    np.savez_compressed(out, norb=norb, seed=seed, nqubit=nq, ref=np.array(ref),
                        h=h, g=g, ham_c=hc, ham_x=hx, ham_z=hz, amps=amps, energy=E, psi=psi,
                        grad=grad, gsd_tops=np.array(tops), gsd_amps=gamps,
                        pool_grads=pool_grads, sa_amps=sa_amps, sa_energy=sa_E,
                        sa_grad=sa_grad)
    print(f"{out}: {nq} q, {len(hc)} H terms, {M} SD params, {P} GSD ops, E = {E:.12f}")


def pqe_fixture(qf, norb, seed, out):
    """UCCNPQE (ucc/uccnpqe.py): excited determinants and phase factors, and
    the residual vector at seeded dUCCSD amplitudes."""
    h, g = random_integrals(norb, seed)
    H = ref_sq_ham(qf, h, g).jw_transform()
    ref = hf_reference(norb, norb)
    rng = np.random.default_rng(1000 + seed)
    s = _Sys()
    s.hamiltonian = H
    s.hf_reference = ref
    s.hf_energy = 0.0
    alg = qf.UCCNPQE(s)
    alg._pool_type = "SD"
    alg._noise_factor = 0.0
    alg._res_vec_evals = 0
    alg._res_m_evals = 0
    alg._excited_dets = []
    alg._tops, alg._tamps = [], []
    alg.fill_pool()
    alg.initialize_ansatz()
    alg.fill_excited_dets()
    M = len(alg._tops)
    amps = rng.uniform(-0.1, 0.1, M)
    res = np.array(alg.get_residual_vector(list(amps)))
    dets = np.array([d for d, _ in alg._excited_dets], dtype=np.uint64)
    phases = np.array([complex(p) for _, p in alg._excited_dets], dtype=np.complex128)
    np.savez_compressed(out, norb=norb, seed=seed, amps=amps, residuals=res, dets=dets,
                        phases=phases)
    print(f"{out}: {M} residuals")


def compact_fixture(qf, norb, seed, out):
    """Compact (FEB / QEB) excitation circuits (utils/compact_excitation_circuits.py):
    each pool operator's gate list at a seeded amplitude, and the state of the
    whole compact ansatz on the reference, for SD, GSD and sa_SD pools with
    fermionic and qubit excitations."""
    from qforte.utils.compact_excitation_circuits import compact_excitation_circuit
    ref = hf_reference(norb, norb)
    rng = np.random.default_rng(2000 + seed)
    arrs = {}
    for pt in ("SD", "GSD", "sa_SD"):
        pool = qf.SQOpPool()
        pool.set_orb_spaces(ref)
        pool.fill_pool(pt)
        temp = []
        for c, op in pool:
            if pt == "sa_SD":
                terms = op.terms()
                for coeff, cr, an in terms[:len(terms) // 2]:
                    s = qf.SQOperator()
                    s.add_term(coeff, cr, an)
                    s.add_term(-coeff, an, cr)
                    temp.append(s)
            else:
                temp.append(op)
        amps = rng.uniform(-0.5, 0.5, len(temp))
        for qe in (False, True):
            key = f"{pt}_{'qe' if qe else 'fe'}"
            ids, tg, ct, pr, owner = [], [], [], [], []
            U = qf.Circuit()
            for k, (t, op) in enumerate(zip(amps, temp)):
                e = op.terms()[1]
                circ = compact_excitation_circuit(t * e[0], e[1], e[2], qe)
                U.add(circ)
                for g in circ.gates():
                    ids.append(g.gate_id())
                    tg.append(g.target())
                    ct.append(g.control())
                    pr.append(float(g.parameter()) if g.has_parameter() else 0.0)
                    owner.append(k)
            qc = qf.Computer(2 * norb)
            prep = qf.Circuit()
            for j, occ in enumerate(ref):
                if occ:
                    prep.add(qf.gate("X", j, j))
            qc.apply_circuit(prep)
            qc.apply_circuit(U)
            arrs[f"{key}_ids"] = np.array(ids)
            arrs[f"{key}_target"] = np.array(tg, dtype=np.int32)
            arrs[f"{key}_control"] = np.array(ct, dtype=np.int32)
            arrs[f"{key}_owner"] = np.array(owner, dtype=np.int32)
            arrs[f"{key}_param"] = np.array(pr)
            arrs[f"{key}_psi"] = np.array(qc.get_coeff_vec())
            arrs[f"{key}_cnots"] = U.get_num_cnots()
        arrs[f"{pt}_amps"] = amps
    np.savez_compressed(out, norb=norb, **arrs)
    print(f"{out}: compact circuits of {[k for k in arrs if k.endswith('_cnots')]}")


def pools_fixture(qf, norb, out):
    ref = hf_reference(norb, norb)
    arrs = {}
    rng = np.random.default_rng(7)
    for pt in ("SD", "GSD", "sa_SD", "SDTQ"):
        pool = qf.SQOpPool()
        pool.set_orb_spaces(ref)
        pool.fill_pool(pt)
        cs, cr, an, owner = [], [], [], []
        for k, (c, op) in enumerate(pool):
            a, b, d = sq_arrays(op)
            cs.append(a)
            cr.append(b)
            an.append(d)
            owner += [k] * len(a)
        w = max(x.shape[1] for x in cr)
        pad = lambda m: np.pad(m, ((0, 0), (0, w - m.shape[1])), constant_values=-1)
        arrs[f"{pt}_coeff"] = np.concatenate(cs)
        arrs[f"{pt}_cre"] = np.concatenate([pad(m) for m in cr])
        arrs[f"{pt}_ann"] = np.concatenate([pad(m) for m in an])
        arrs[f"{pt}_owner"] = np.array(owner, dtype=np.int32)
        if pt != "sa_SD":
            amps = rng.uniform(-0.1, 0.1, len(pool))
            tmp = qf.SQOpPool()
            for t, (c, op) in zip(amps, pool):
                tmp.add(t, op)
            A = tmp.get_qubit_operator("commuting_grp_lex")
            ac, ax, az = pauli_arrays(A)
            arrs[f"{pt}_amps"] = amps
            arrs[f"{pt}_A_c"], arrs[f"{pt}_A_x"], arrs[f"{pt}_A_z"] = ac, ax, az
    np.savez_compressed(out, norb=norb, **arrs)
    print(f"{out}: pools {[k for k in arrs if k.endswith('_owner')]}")


def gates_fixture(qf, out, n=6, ngates=300, seed=5):
    rng = np.random.default_rng(seed)
    one = ["X", "Y", "Z", "H", "R", "Rx", "Ry", "Rz", "V", "S", "T", "I"]
    two = ["A", "cX", "acX", "cY", "cZ", "cR", "cV", "cRz", "SWAP", "CNOT", "aCNOT"]
    kinds, tg, ct, pr = [], [], [], []
    qc = qf.Computer(n)
    circ = qf.Circuit()
    for _ in range(ngates):
        if rng.random() < 0.5:
            k = one[rng.integers(len(one))]
            t = int(rng.integers(n))
            c = t
        else:
            k = two[rng.integers(len(two))]
            t, c = (int(v) for v in rng.choice(n, 2, replace=False))
        p = float(rng.uniform(0, 4 * math.pi))
        circ.add(qf.gate(k, t, c, p))
        kinds.append(k)
        tg.append(t)
        ct.append(c)
        pr.append(p)
    qc.apply_circuit(circ)
    psi = np.array(qc.get_coeff_vec())
    # an operator application and its expectation value on that state
    op = qf.build_operator("0.5, X_0 Z_2; 0.3j, Y_1 X_3; -0.7, Z_0 Z_5; 0.2, X_1 X_1; "
                           "0.1, Y_2 Z_2 X_4; -0.25j, Z_3")
    qc2 = qf.Computer(qc)
    qc2.apply_operator(op)
    ev = qc.direct_op_exp_val(op)
    pev = [qc.direct_pauli_circ_exp_val(qf.build_circuit(s))
           for s in ("X_0 Y_1", "Y_2", "Y_1 Y_3 Z_0", "X_5 X_5 Y_4", "Z_1 X_1")]
    pmc = qc.perfect_measure_circuit(qf.build_circuit("X_0 Y_2 Z_4"))
    np.savez_compressed(out, n=n, kinds=np.array(kinds), target=np.array(tg),
                        control=np.array(ct), param=np.array(pr), psi=psi,
                        op_psi=np.array(qc2.get_coeff_vec()), op_expval=ev,
                        pauli_expvals=np.array(pev), perfect_measure=pmc)
    print(f"{out}: {ngates} gates on {n} qubits")


def integrals_fixture(path, out):
    with open(path) as f:
        data = json.load(f)
    oei = np.array(data["oei"]["data"], dtype=np.float64)
    tei = np.array(data["tei"]["data"], dtype=np.float64)
    np.savez_compressed(out, nso=data["nso"]["data"], na=data["na"]["data"],
                        nb=data["nb"]["data"], scalar=data["scalar_energy"]["data"],
                        oei=oei, tei=tei)
    print(f"{out}: {len(oei)} one-body, {len(tei)} two-body integrals")


def _test_qubit_system(test_file):
    """The qubit Hamiltonian (coef_vec, circ_vec), reference determinant and FCI
    energy that one of the reference's algorithm tests builds, read from its
    source (tests/test_qite.py:6-59: H2/STO-3G; tests/test_fast_qk.py:9-392:
    H4/STO-6G)."""
    import ast
    tree = ast.parse(open(test_file).read())
    found = {}
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            if name in ("E_fci", "coef_vec", "ref"):
                found[name] = ast.literal_eval(node.value)
            elif name == "circ_vec":
                found[name] = [c.args[0].value if c.args else "" for c in node.value.elts]
    return found


def qite_fixture(qf, test_file, norb, seed, out):
    """QITE (ite/qite.py) run by the reference: the H2 case of its own test
    (beta = 18, Lanczos every 49 steps), the same H2 with the dense cqoy
    expansion, and a seeded random-integral system with the sparse SD
    expansion and with the GSD one at two Trotter steps."""
    h2 = _test_qubit_system(test_file)
    H = qf.QubitOperator()
    for c, s in zip(h2["coef_vec"], h2["circ_vec"]):
        H.add(c, qf.build_circuit(s) if s else qf.Circuit())
    mol = qf.Molecule()
    mol.hamiltonian = H
    alg = qf.QITE(mol, reference=h2["ref"])
    alg.run(beta=18.0, do_lanczos=True, lanczos_gap=49)
    res = {"h2_coeffs": np.array(h2["coef_vec"]), "h2_circs": np.array(h2["circ_vec"]),
           "h2_ref": np.array(h2["ref"]), "h2_efci": h2["E_fci"],
           "h2_ekb": np.array(alg._Ekb), "h2_lanczos": complex(alg._Egs_lanczos)}
    h, g = random_integrals(norb, seed)
    Hq = ref_sq_ham(qf, h, g).jw_transform()
    s = _Sys()
    s.hamiltonian = Hq
    s.hf_reference = hf_reference(norb, norb)
    s.hf_energy = 0.0
    alg = qf.QITE(s)
    alg.run(beta=0.6, db=0.2, expansion_type="SD", sparseSb=True)
    res["rand_sd_ekb"] = np.array(alg._Ekb)
    res["rand_sd_nparams"] = alg._n_classical_params
    alg = qf.QITE(s, trotter_number=2)
    alg.run(beta=0.4, db=0.2, expansion_type="GSD", sparseSb=True)
    res["rand_gsd_ekb"] = np.array(alg._Ekb)
    res["rand_gsd_nparams"] = alg._n_classical_params
    # the transverse-field Ising model (adapters/model_adapters.py), cqoy expansion
    from qforte.adapters.model_adapters import create_TFIM
    alg = qf.QITE(create_TFIM(4, 1.0, 0.7))
    alg.run(beta=0.6, db=0.2, expansion_type="cqoy", sparseSb=True)
    res["tfim_ekb"] = np.array(alg._Ekb)
    res["tfim_nparams"] = alg._n_classical_params
    alg = qf.QITE(mol, reference=h2["ref"])
    alg.run(beta=0.6, db=0.2, expansion_type="cqoy", sparseSb=False)
    res["h2_cqoy_ekb"] = np.array(alg._Ekb)
    res["h2_cqoy_nparams"] = alg._n_classical_params
    np.savez_compressed(out, norb=norb, seed=seed, **res)
    print(f"{out}: H2 QITE E = {res['h2_ekb'][-1]}, random SD E = {res['rand_sd_ekb'][-1]}")


def srqk_fixture(qf, test_file, norb, seed, out):
    """SRQK (qkd/srqk.py:103-204 with abc/qsdabc.py:87-115) and NTSRQK
    (qkd/nt_srqk.py) run by the reference: the H4 cases of its own test
    (SRQK: trotter_number = 100, s = 6; NTSRQK: s = 4, dt = 0.8) and a seeded
    random-integral system (s = 3, dt = 0.5, one Trotter step)."""
    h4 = _test_qubit_system(test_file)
    H = qf.QubitOperator()
    for c, s in zip(h4["coef_vec"], h4["circ_vec"]):
        H.add(c, qf.build_circuit(s) if s else qf.Circuit())
    mol = qf.Molecule()
    mol.hamiltonian = H
    alg = qf.SRQK(mol, reference=h4["ref"], trotter_number=100)
    alg.run(s=6)
    res = {"h4_coeffs": np.array(h4["coef_vec"]), "h4_circs": np.array(h4["circ_vec"]),
           "h4_ref": np.array(h4["ref"]), "h4_efci": h4["E_fci"], "h4_S": alg._S,
           "h4_H": alg._Hbar, "h4_evals": np.array(alg._eigenvalues), "h4_egs": alg._Egs}
    h, g = random_integrals(norb, seed)
    s = _Sys()
    s.hamiltonian = ref_sq_ham(qf, h, g).jw_transform()
    s.hf_reference = hf_reference(norb, norb)
    s.hf_energy = 0.0
    alg = qf.SRQK(s)
    alg.run(s=3, dt=0.5)
    res.update({"rand_S": alg._S, "rand_H": alg._Hbar,
                "rand_evals": np.array(alg._eigenvalues), "rand_egs": alg._Egs})
    alg = qf.SRQK(s, trotter_number=2)
    # the per-step printout indexes root 1 of a 1x1 problem: run without it
    alg.run(s=3, dt=0.5, target_root=1, diagonalize_each_step=False)
    res.update({"rand_t2_S": alg._S, "rand_t2_H": alg._Hbar, "rand_t2_egs": alg._Egs,
                "rand_t2_ets": alg._Ets})
    # non-Trotterized SRQK (qkd/nt_srqk.py): the H4 case of the same test
    # (s = 4, dt = 0.8) and the random system
    alg = qf.NTSRQK(mol, reference=h4["ref"])
    alg.run(s=4, dt=0.8)
    res.update({"h4_nt_S": alg._S, "h4_nt_H": alg._Hbar, "h4_nt_egs": alg._Egs})
    alg = qf.NTSRQK(s)
    alg.run(s=3, dt=0.5)
    res.update({"rand_nt_S": alg._S, "rand_nt_H": alg._Hbar, "rand_nt_egs": alg._Egs})
    np.savez_compressed(out, norb=norb, seed=seed, **res)
    print(f"{out}: H4 NTSRQK E = {res['h4_nt_egs']}, cond S = "
          f"{np.linalg.cond(res['h4_nt_S']):.2e}; random NTSRQK cond S = "
          f"{np.linalg.cond(res['rand_nt_S']):.2e}")
    print(f"{out}: H4 SRQK E = {res['h4_egs']} (FCI {h4['E_fci']}), cond S = "
          f"{np.linalg.cond(res['h4_S']):.2e}; random E = {res['rand_egs']}, cond S = "
          f"{np.linalg.cond(res['rand_S']):.2e}")


def spqe_fixture(qf, tests_dir, norb, seed, out):
    """SPQE (ucc/spqe.py) run by the reference: the H4/STO-6G case of its own
    test (tests/test_spqe.py:11-39: external integrals, zero terms dropped,
    spqe_thresh 1e-4, dt 1e-4) and a seeded random-integral system."""
    mol = qf.system_factory(stytem_type="molecule", build_type="external", basis="sto-6g",
                            filename=os.path.join(tests_dir, "H4-sto6g-075a.json"))
    Hnz = qf.QubitOperator()
    for c, circ in mol._hamiltonian.terms():
        if abs(c) > 1.0e-14:
            Hnz.add(c, circ)
    mol._hamiltonian = Hnz
    alg = qf.SPQE(mol, print_summary_file=False)
    alg.run(spqe_maxiter=20, spqe_thresh=1.0e-4, opt_thresh=1.0e-5, dt=0.0001)
    res = {"h4_egs": alg.get_gs_energy(), "h4_energies": np.array(alg._energies),
           "h4_nparams": np.array(alg._n_classical_params_lst), "h4_npool": len(alg._pool_obj),
           "h4_tops": np.array(alg._tops),
           "h4_orb_e": np.array(alg._orb_e)}
    h, g = random_integrals(norb, seed)
    s = _Sys()
    s.hamiltonian = ref_sq_ham(qf, h, g).jw_transform()
    s.hf_reference = hf_reference(norb, norb)
    s.hf_energy = 0.0
    s.orb_irreps_to_int = [0] * norb
    s.point_group = ["c1", ["A"]]
    alg = qf.SPQE(s)
    alg.run(spqe_maxiter=10, spqe_thresh=1.0e-3, opt_thresh=1.0e-7, opt_maxiter=60, dt=0.001)
    res.update({"rand_egs": alg.get_gs_energy(), "rand_energies": np.array(alg._energies),
                "rand_nparams": np.array(alg._n_classical_params_lst),
                "rand_tops": np.array(alg._tops), "rand_npool": len(alg._pool_obj)})
    # moment energy corrections (utils/moment_energy_corrections.py) on H4:
    # UCCNPQE with the SD pool and SPQE, moments up to quadruples
    alg = qf.UCCNPQE(mol, max_moment_rank=4, moment_dt=0.001)
    alg.run(pool_type="SD", opt_thresh=1.0e-7, opt_maxiter=60)
    res.update({"mmcc_pqe_egs": alg.get_gs_energy(), "mmcc_pqe_mp": np.array(alg._E_mmcc_mp),
                "mmcc_pqe_en": np.array(alg._E_mmcc_en),
                "mmcc_pqe_en_diag": np.real(np.array(alg._epstein_nesbet)),
                "mmcc_pqe_mpdenom": np.array(alg._mpdenom)})
    alg = qf.SPQE(mol, max_moment_rank=4, moment_dt=0.001)
    alg.run(spqe_maxiter=20, spqe_thresh=1.0e-2, opt_thresh=1.0e-5, dt=0.0001)
    res.update({"mmcc_spqe_mp": np.array(alg._E_mmcc_mp), "mmcc_spqe_en": np.array(alg._E_mmcc_en)})
    np.savez_compressed(out, norb=norb, seed=seed, **res)
    print(f"{out}: H4 SPQE E = {res['h4_egs']} ({len(res['h4_energies'])} macro-iterations, "
          f"params {res['h4_nparams']}); random E = {res['rand_egs']}, params {res['rand_nparams']}")


def mrsqk_fixture(qf, test_file, norb, seed, out):
    """MRSQK (qkd/mrsqk.py) run by the reference: the H4 case of its own test
    (tests/test_fast_qk.py:401-405: trotter_number = 100, s = 3, d = 3) and a
    seeded random-integral system with and without spin-adapted references."""
    h4 = _test_qubit_system(test_file)
    H = qf.QubitOperator()
    for c, s in zip(h4["coef_vec"], h4["circ_vec"]):
        H.add(c, qf.build_circuit(s) if s else qf.Circuit())
    mol = qf.Molecule()
    mol.hamiltonian = H
    res = {"h4_coeffs": np.array(h4["coef_vec"]), "h4_circs": np.array(h4["circ_vec"]),
           "h4_ref": np.array(h4["ref"]), "h4_efci": h4["E_fci"]}

    def record(tag, alg):
        res[f"{tag}_egs"] = alg._Egs
        res[f"{tag}_evals"] = np.array(alg._eigenvalues)
        res[f"{tag}_single_refs"] = np.array(alg._single_det_refs)
        if alg._use_spin_adapted_refs:
            res[f"{tag}_sa_ndet"] = np.array([len(r) for r in alg._sa_ref_lst])
            res[f"{tag}_sa_flat_dets"] = np.array([d for r in alg._sa_ref_lst for _, d in r])
            res[f"{tag}_sa_flat_coeffs"] = np.array([c for r in alg._sa_ref_lst for c, _ in r])

    alg = qf.MRSQK(mol, reference=h4["ref"], trotter_number=100)
    alg.run(s=3, d=3)
    record("h4", alg)
    h, g = random_integrals(norb, seed)
    sy = _Sys()
    sy.hamiltonian = ref_sq_ham(qf, h, g).jw_transform()
    sy.hf_reference = hf_reference(norb, norb)
    sy.hf_energy = 0.0
    alg = qf.MRSQK(sy)
    alg.run(s=2, d=2, mr_dt=0.4)
    record("rand_sa", alg)
    alg = qf.MRSQK(sy)
    alg.run(s=2, d=2, mr_dt=0.4, use_spin_adapted_refs=False)
    record("rand", alg)
    np.savez_compressed(out, norb=norb, seed=seed, **res)
    print(f"{out}: H4 MRSQK E = {res['h4_egs']} (FCI {h4['E_fci']}); random SA E = "
          f"{res['rand_sa_egs']}, single-reference E = {res['rand_egs']}")


def oppl_fixture(qf, norb, seed, out):
    """Computer.direct_oppl_exp_val / direct_idxd_oppl_exp_val (computer.cc:773-806)
    on the commutator pool of UCCVQE.fill_commutator_pool (uccvqeabc.py:85-89):
    every [H, A_k] of the GSD pool at a seeded 3-operator dUCC state, and an
    indexed subset in a scrambled order."""
    h, g = random_integrals(norb, seed)
    H = ref_sq_ham(qf, h, g).jw_transform()
    ref = hf_reference(norb, norb)
    rng = np.random.default_rng(3000 + seed)
    alg = make_alg(qf, H, ref, "GSD")
    P = len(alg._pool_obj)
    tops = [int(t) for t in rng.choice(P, 3, replace=False)]
    amps = rng.uniform(-0.2, 0.2, 3)
    alg._tops, alg._tamps = tops, list(amps)
    comm = alg._pool_obj.get_qubit_op_pool()
    comm.join_as_commutator(H)
    qc = qf.Computer(2 * norb)
    qc.apply_circuit(alg.build_Uvqc(list(amps)))
    psi = np.array(qc.get_coeff_vec())
    vals = np.array(qc.direct_oppl_exp_val(comm))
    idxs = [int(i) for i in rng.permutation(P)[:P // 3]]
    ivals = np.array(qc.direct_idxd_oppl_exp_val(comm, idxs))
    np.savez_compressed(out, norb=norb, seed=seed, tops=np.array(tops), amps=amps, psi=psi,
                        oppl=vals, idxs=np.array(idxs), idxd_oppl=ivals)
    print(f"{out}: {P} commutators, max |<[H,A]>| = {np.max(np.abs(vals)):.3e}")


def bench_ucc_fixture(qf, norb, seed, batch, rows, out):
    """The default benchmark's problem: dUCCSD energy (AnsatzAlgorithm.energy_feval,
    algorithm.py:458-474) and adjoint gradient (UCCVQE.measure_gradient,
    uccvqeabc.py:122-251) of the listed rows of the benchmark's parameter matrix,
    default_rng(seed + 1).uniform(-0.1, 0.1, (batch, M))."""
    h, g = random_integrals(norb, seed)
    H = ref_sq_ham(qf, h, g).jw_transform()
    ref = hf_reference(norb, norb)
    alg = make_alg(qf, H, ref, "SD")
    M = len(alg._pool_obj)
    P = np.random.default_rng(seed + 1).uniform(-0.1, 0.1, (batch, M))
    alg._tops = list(range(M))
    E, G = [], []
    for r in rows:
        alg._tamps = list(P[r])
        E.append(alg.energy_feval(list(P[r])))
        G.append(np.array(alg.measure_gradient(list(P[r]))))
    np.savez_compressed(out, norb=norb, seed=seed, batch=batch, rows=np.array(rows),
                        nterms=len(H.terms()), energies=np.array(E), grads=np.array(G))
    print(f"{out}: rows {rows}: E = {E}, |g|max = {[float(np.max(np.abs(x))) for x in G]}")


def grad_fixture(qf, norb, seed, out):
    """Adjoint dUCCSD gradient at 2 norb qubits (UCCVQE.measure_gradient) at row
    0 of default_rng(seed + norb).uniform(-0.1, 0.1, (B, M)), the amplitudes
    the differentiation workload starts from, with its energy."""
    h, g = random_integrals(norb, seed)
    H = ref_sq_ham(qf, h, g).jw_transform()
    ref = hf_reference(norb, norb)
    alg = make_alg(qf, H, ref, "SD")
    M = len(alg._pool_obj)
    amps = np.random.default_rng(seed + norb).uniform(-0.1, 0.1, (1, M))[0]
    alg._tops = list(range(M))
    alg._tamps = list(amps)
    E = alg.energy_feval(list(amps))
    G = np.array(alg.measure_gradient(list(amps)))
    np.savez_compressed(out, norb=norb, seed=seed, nterms=len(H.terms()), amps=amps,
                        energy=E, grad=G)
    print(f"{out}: {M} parameters, E = {E:.12f}, |g|max = {np.max(np.abs(G)):.3e}")


def adapt_fixture(qf, norb, seed, out):
    """ADAPT pool gradients 2 Re <H psi|A_k psi> (UCCVQE.measure_gradient3,
    uccvqeabc.py:253-283) of the whole GSD pool at the 12-operator dUCC state
    of the pool-gradient workload: operators rng.choice(P, 12) and amplitudes
    U(-0.1, 0.1) from default_rng(seed + 7)."""
    h, g = random_integrals(norb, seed)
    H = ref_sq_ham(qf, h, g).jw_transform()
    ref = hf_reference(norb, norb)
    alg = make_alg(qf, H, ref, "GSD")
    P = len(alg._pool_obj)
    rng = np.random.default_rng(seed + 7)
    tops = [int(v) for v in rng.choice(P, 12, replace=False)]
    amps = rng.uniform(-0.1, 0.1, 12)
    alg._tops, alg._tamps = tops, list(amps)
    G = np.array(alg.measure_gradient3())
    np.savez_compressed(out, norb=norb, seed=seed, tops=np.array(tops), amps=amps,
                        pool_grads=G)
    print(f"{out}: {P} pool gradients, |g|max = {np.max(np.abs(G)):.3e}")


def sweep_fixture(qf, n, layers, seed, out):
    """The gate-application sweep (Computer.apply_circuit, computer.cc:93-114) of
    qforte_b200.workloads.layered_random_circuit(n, layers, seed) from |0...0>:
    the state's norm, 4,096 amplitudes at seeded indices, <Z_k> for every qubit
    and the probability mass of each value of the top 8 qubits."""
    from qforte_b200.workloads import layered_random_circuit
    _, spec = layered_random_circuit(n, layers, seed)
    circ = qf.Circuit()
    for k, t, c, p in spec:
        circ.add(qf.gate(k, t, c, p))
    qc = qf.Computer(n)
    qc.apply_circuit(circ)
    psi = np.array(qc.get_coeff_vec())
    del qc
    prob = psi.real ** 2 + psi.imag ** 2
    idx = np.sort(np.random.default_rng(seed + 500).choice(1 << n, 4096, replace=False))
    zk = np.array([prob.reshape(-1, 2, 1 << k)[:, 0, :].sum() -
                   prob.reshape(-1, 2, 1 << k)[:, 1, :].sum() for k in range(n)])
    top = prob.reshape(256, -1).sum(axis=1)
    np.savez_compressed(out, n=n, layers=layers, seed=seed, ngates=len(spec),
                        norm=np.sqrt(prob.sum()), idx=idx, amps=psi[idx], z=zk, top8=top)
    print(f"{out}: {len(spec)} gates on {n} qubits, norm - 1 = {np.sqrt(prob.sum()) - 1:.2e}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-src", default=os.environ.get("QFORTE_REF_SRC",
                                                        "/root/reference/src/qforte"))
    ap.add_argument("--only", default=None,
                    help="one fixture family (pqe, compact, qite, srqk, spqe, mrsqk, oppl, "
                         "bench16, grad20, adapt20, sweep20, sweep24)")
    a = ap.parse_args()
    qf = O.load_reference(a.ref_src)
    tests_dir = os.path.join(os.path.dirname(a.ref_src.rstrip("/")), "..", "tests")
    if a.only in ("compact", None):
        compact_fixture(qf, 4, 11, os.path.join(HERE, "compact_norb4.npz"))
    if a.only in ("pqe", None):
        pqe_fixture(qf, 4, 11, os.path.join(HERE, "pqe_norb4_seed11.npz"))
        pqe_fixture(qf, 6, 11, os.path.join(HERE, "pqe_norb6_seed11.npz"))
    if a.only in ("qite", None):
        qite_fixture(qf, os.path.join(tests_dir, "test_qite.py"), 3, 11,
                     os.path.join(HERE, "qite_norb3_seed11.npz"))
    if a.only in ("srqk", None):
        srqk_fixture(qf, os.path.join(tests_dir, "test_fast_qk.py"), 3, 11,
                     os.path.join(HERE, "srqk_norb3_seed11.npz"))
    if a.only in ("spqe", None):
        spqe_fixture(qf, tests_dir, 3, 11, os.path.join(HERE, "spqe_norb3_seed11.npz"))
    if a.only in ("mrsqk", None):
        mrsqk_fixture(qf, os.path.join(tests_dir, "test_fast_qk.py"), 3, 11,
                      os.path.join(HERE, "mrsqk_norb3_seed11.npz"))
    if a.only in ("oppl", None):
        oppl_fixture(qf, 4, 11, os.path.join(HERE, "oppl_norb4_seed11.npz"))
    # the benchmarked configurations themselves (minutes to an hour each on one core)
    if a.only == "bench16":
        bench_ucc_fixture(qf, 8, 11, 256, (0, 255), os.path.join(HERE, "bench_ucc16_seed11.npz"))
    if a.only == "grad20":
        grad_fixture(qf, 10, 11, os.path.join(HERE, "grad_ucc20_seed11.npz"))
    if a.only == "adapt20":
        adapt_fixture(qf, 10, 11, os.path.join(HERE, "adapt_gsd20_seed11.npz"))
    for n in (20, 24, 28):
        if a.only == f"sweep{n}":
            sweep_fixture(qf, n, 100, 11 + n, os.path.join(HERE, f"sweep{n}_seed{11 + n}.npz"))
    if a.only is not None:
        return
    ucc_fixture(qf, 4, 11, os.path.join(HERE, "ucc_norb4_seed11.npz"))
    ucc_fixture(qf, 6, 11, os.path.join(HERE, "ucc_norb6_seed11.npz"))
    pools_fixture(qf, 4, os.path.join(HERE, "pools_norb4.npz"))
    gates_fixture(qf, os.path.join(HERE, "gates_n6.npz"))
    integrals_fixture(os.path.join(tests_dir, "He-ccpvdz.json"),
                      os.path.join(HERE, "he_ccpvdz_integrals.npz"))
    integrals_fixture(os.path.join(tests_dir, "H4-sto6g-075a.json"),
                      os.path.join(HERE, "h4_sto6g_integrals.npz"))


if __name__ == "__main__":
    main()
