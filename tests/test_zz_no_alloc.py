"""The allocation-free expectation-value entry point.

qfb_sum_expval_noalloc computes what qfb_sum_expval computes, for callers that
must not allocate device memory while they run (a request loop holding a
fixed HBM budget, or code running while other work may hold every free byte).
Its scratch is a fixed array inside the library, so the test calls it twice in
a row (the second call sees the first call's leftovers) and checks both calls
against the allocating entry point, at the energy tolerance of the parity
tests.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E_TOL = 1e-10


def _expvals(lib, ds, bra, ket, n):
    a = np.zeros(n, dtype=np.complex128)
    b = np.zeros(n, dtype=np.complex128)
    from qforte_b200._lib import check, ptr
    check(lib.qfb_sum_expval(ds.h, bra, ket, ptr(a)), "qfb_sum_expval")
    check(lib.qfb_sum_expval_noalloc(ds.h, bra, ket, ptr(b)), "qfb_sum_expval_noalloc")
    return a, b


def test_noalloc_expval_matches_allocating_entry_point(cuda):
    import qforte_b200 as qb
    from qforte_b200._lib import check, lib, ptr
    from qforte_b200.device import sum_from_terms
    L = lib()

    # a Hamiltonian's energy on a random 10-qubit state
    mol = qb.random_molecule(5, 5, seed=3)
    rng = np.random.default_rng(1)
    psi = rng.normal(size=1024) + 1j * rng.normal(size=1024)
    psi /= np.linalg.norm(psi)
    qc = qb.Computer(10)
    qc.set_coeff_vec(psi)
    ham = sum_from_terms(mol.hamiltonian._pauli_terms())
    for _ in range(2):
        a, b = _expvals(L, ham, qc._h, qc._h, 1)
        assert abs(a[0] - b[0]) < E_TOL

    # a pool of operators (one result per operator) between two different
    # states of a batch of three, twice in a row
    pool = qb.SQOpPool()
    pool.set_orb_spaces(mol.hf_reference)
    pool.fill_pool("GSD")
    terms, seg = [], []
    for k, (c, op) in enumerate(pool):
        s = qb.SQOperator()
        s.add_op(op)
        pt = s.jw_transform()._pauli_terms()
        terms += pt
        seg += [k] * len(pt)
    psum = sum_from_terms(terms, seg, len(pool))
    bra, ket = ctypes.c_void_p(), ctypes.c_void_p()
    check(L.qfb_state_create(10, 3, ctypes.byref(bra)))
    check(L.qfb_state_create(10, 3, ctypes.byref(ket)))
    try:
        for b in range(3):
            v = rng.normal(size=1024) + 1j * rng.normal(size=1024)
            w = rng.normal(size=1024) + 1j * rng.normal(size=1024)
            check(L.qfb_state_upload(bra, b, ptr(v), 1024))
            check(L.qfb_state_upload(ket, b, ptr(w), 1024))
        for _ in range(2):
            a, b = _expvals(L, psum, bra, ket, 3 * len(pool))
            assert np.max(np.abs(a - b)) < E_TOL
    finally:
        L.qfb_state_destroy(bra)
        L.qfb_state_destroy(ket)


def test_noalloc_refuses_work_beyond_its_fixed_scratch(cuda):
    import qforte_b200 as qb
    from qforte_b200._lib import QFB_EINVAL, last_error, lib, ptr
    from qforte_b200.device import sum_from_terms
    L = lib()
    op = qb.build_operator("0.5, X_0 Z_2; 0.25, Y_1; -0.3, Z_3")
    ds = sum_from_terms(op._pauli_terms())  # 3 x-groups
    st = ctypes.c_void_p()
    assert L.qfb_state_create(4, 30000, ctypes.byref(st)) == 0
    try:
        out = np.zeros(30000, dtype=np.complex128)
        rc = L.qfb_sum_expval_noalloc(ds.h, st, st, ptr(out))
        assert rc == QFB_EINVAL
        assert "fixed scratch" in last_error()
    finally:
        L.qfb_state_destroy(st)
